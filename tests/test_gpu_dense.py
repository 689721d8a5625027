"""GPU tests of the exact modular GEMM D <- (D - A B) mod p (gbgpu_dense_submul):
the int8 tensor-core form and the CUDA-core form against an exact CPU
evaluation, bit for bit, over every limb count and ragged shapes."""
import ctypes as C

import numpy as np
import pytest

from gb_b200 import _lib

pytestmark = pytest.mark.gpu


def exact_submul(D, A, B, p):
    """(D - A B) mod p exactly: B split into 16-bit halves keeps int64 sums exact
    for the sizes used here (K * (p-1) * 2^16 < 2^63)."""
    A = A.astype(np.int64)
    B = B.astype(np.int64)
    lo = (A @ (B & 0xFFFF)) % p
    hi = (A @ (B >> 16)) % p
    prod = (lo + ((hi << 16) % p)) % p
    return ((D.astype(np.int64) - prod) % p).astype(np.uint32)


def run(form, p, A, B, D):
    lib = _lib.load()
    M, K = A.shape
    N = B.shape[1]
    A = np.ascontiguousarray(A, dtype=np.uint32)
    B = np.ascontiguousarray(B, dtype=np.uint32)
    out = np.ascontiguousarray(D, dtype=np.uint32).copy()
    opt = _lib.Options(form, 0, 1, 0, None)
    _lib.check(lib.gbgpu_dense_submul_host(p, M, N, K, A.ctypes.data, K, B.ctypes.data, N,
                                           out.ctypes.data, N, C.byref(opt)))
    return out


CASES = [
    # (p, M, N, K): one per limb count, tile-aligned and ragged
    (251, 128, 256, 128),
    (251, 300, 520, 700),
    (32003, 128, 128, 256),
    (65521, 257, 130, 333),
    (65521, 512, 384, 2048),
    (1000003, 200, 96, 500),  # three limbs
    (16777213, 130, 70, 129),
    (2147483647, 128, 64, 128),
    (2147483647, 333, 200, 1000),
    (3, 100, 100, 100),
    (65537, 129, 129, 129),
]


@pytest.mark.parametrize("p,M,N,K", CASES)
@pytest.mark.parametrize("form", [_lib.FORM_TENSOR, _lib.FORM_PLAIN])
def test_dense_submul_exact(form, p, M, N, K):
    rng = np.random.default_rng(p % 1000 + M + N + K)
    A = rng.integers(0, p, size=(M, K), dtype=np.int64)
    B = rng.integers(0, p, size=(K, N), dtype=np.int64)
    D = rng.integers(0, p, size=(M, N), dtype=np.int64)
    got = run(form, p, A, B, D)
    want = exact_submul(D, A, B, p)
    assert np.array_equal(got, want)


def test_dense_submul_extreme_values_multi_panel():
    # all residues p-1 maximise every limb product; K spans several K panels
    for p, K in ((251, 33024 + 640), (65521, 16384 + 256), (2147483647, 8192 + 384)):
        M, N = 128, 64
        A = np.full((M, K), p - 1, dtype=np.int64)
        B = np.full((K, N), p - 1, dtype=np.int64)
        D = np.zeros((M, N), dtype=np.int64)
        want = exact_submul(D, A, B, p)
        for form in (_lib.FORM_TENSOR, _lib.FORM_PLAIN):
            assert np.array_equal(run(form, p, A, B, D), want), (p, form)


def test_dense_submul_rejects_bad_arguments():
    lib = _lib.load()
    opt = _lib.Options(_lib.FORM_TENSOR, 0, 1, 0, None)
    buf = np.zeros(16, dtype=np.uint32)
    rc = lib.gbgpu_dense_submul_host(2, 2, 2, 2, buf.ctypes.data, 2, buf.ctypes.data, 2,
                                     buf.ctypes.data, 2, C.byref(opt))
    assert rc == _lib.GBGPU_EINVAL  # even prime on the tensor-core form
    rc = lib.gbgpu_dense_submul_host(101, 2, 2, 4, buf.ctypes.data, 2, buf.ctypes.data, 2,
                                     buf.ctypes.data, 2, C.byref(opt))
    assert rc == _lib.GBGPU_EINVAL  # lda < K


def cpu_rref(D, p):
    """Reduced row echelon form over GF(p) (numpy int64, exact)."""
    A = np.array(D, dtype=np.int64) % p
    rows, cols = A.shape
    r = 0
    piv = []
    for c in range(cols):
        nz = np.nonzero(A[r:, c])[0]
        if nz.size == 0:
            continue
        i = r + nz[0]
        A[[r, i]] = A[[i, r]]
        inv = pow(int(A[r, c]), p - 2, p)
        A[r] = (A[r] * inv) % p
        others = np.nonzero(A[:, c])[0]
        for o in others:
            if o != r:
                A[o] = (A[o] - A[o, c] * A[r]) % p
        piv.append(c)
        r += 1
        if r == rows:
            break
    return A[:r].astype(np.uint32), piv


@pytest.mark.parametrize("p,rows,cols,rank", [
    (251, 200, 260, 120), (65521, 300, 300, 300), (65521, 520, 300, 170),
    (2147483647, 260, 400, 200), (3, 150, 200, 60), (1000003, 129, 1030, 100)])
@pytest.mark.parametrize("form", [_lib.FORM_TENSOR, _lib.FORM_PLAIN])
def test_dense_rref_exact(form, p, rows, cols, rank):
    torch = pytest.importorskip("torch")
    from gb_b200 import synth
    D = synth.dense_lowrank(rows, cols, rank, p, seed=rows + cols)
    want, piv = cpu_rref(D, p)
    lib = _lib.load()
    dev = torch.from_numpy(D.astype(np.uint32).view(np.int32)).cuda()
    pc = torch.zeros(min(rows, cols), dtype=torch.int32, device="cuda")
    rk = C.c_int32()
    opt = _lib.Options(form, 0, 1, 0, None)
    _lib.check(lib.gbgpu_dense_rref(p, rows, cols, dev.data_ptr(), cols, C.byref(rk),
                                    pc.data_ptr(), C.byref(opt)))
    got = dev.cpu().numpy().view(np.uint32)
    assert rk.value == len(piv)
    assert pc.cpu().numpy()[: rk.value].tolist() == piv
    assert np.array_equal(got[: rk.value], want)
    assert not got[rk.value:].any()


def test_autotune_writes_a_cache_and_keeps_results_exact(tmp_path, monkeypatch):
    """gbgpu_autotune times the tile shapes on this GPU, writes one valid line
    per (limbs, K band) it tuned, and the GEMMs after it stay exact."""
    lib = _lib.load()
    path = tmp_path / "shapes.txt"
    _lib.check(lib.gbgpu_autotune(0, str(path).encode()))
    lines = [l.split() for l in path.read_text().splitlines() if not l.startswith("#")]
    assert len(lines) >= 9
    for L, kmax, shape in lines:
        assert int(L) in (1, 2) and int(shape) in (0, 1, 2)
        if int(shape) == 1:
            assert int(kmax) <= 256
        if int(shape) == 2:
            assert int(L) == 2
    for p, M, N, K in [(251, 300, 520, 700), (65521, 257, 130, 333), (65521, 200, 300, 2000)]:
        rng = np.random.default_rng(K)
        A = rng.integers(0, p, size=(M, K), dtype=np.int64)
        B = rng.integers(0, p, size=(K, N), dtype=np.int64)
        D = rng.integers(0, p, size=(M, N), dtype=np.int64)
        got = run(_lib.FORM_TENSOR, p, A, B, D)
        assert np.array_equal(got, exact_submul(D, A, B, p))
