"""GPU parity at the sizes the workloads name (the reference's own la, or an
exact CPU evaluation, as the checker):

* the 20000 x 5000 A|B/C|D staircase over p = 65521 (the bench matrix), whole,
  against the reference la (src/la_ff_32.c:1804, option 1, all host threads);
* the exact modular GEMM D - A B mod p on 8192 x 8192 blocks for p = 251,
  65521, 2^31 - 1 and on 16384 x 16384 for p = 65521: sampled output rows
  evaluated exactly on the CPU and a Freivalds check of every row with random
  vectors (false-accept chance below p^-3);
* the dense RREF of a rank-6144 8192 x 8192 block (gbgpu_dense_rref) for the
  three primes, against the reference's dense echelon and interreduction
  (exact_dense_linear_algebra + interreduce_dense_matrix, src/la_ff_32.c:1217
  and :1181, src/la_ff_16.c:873-989 and :837-871 for p = 251) run on the
  same block through a Macaulay matrix whose Schur complement is the block;
* the step after the linear algebra (src/convert.c:137-280) on the answer of
  the 20000 x 5000 staircase: the same new basis elements, basis hash table
  size and hash-map layout as the reference's own conversion.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from gb_b200 import _lib, la, synth
from helpers import dense_rref_rows, matvec_mod, vecmat_mod

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")


@needs_ref
def test_staircase_20000x5000_matches_reference_whole():
    mat = synth.staircase(20000, 5000, 20000, 65521, 0.02, 0.05, seed=1)
    got = la.linear_algebra(mat, form=_lib.FORM_TENSOR)
    want, _ = oracle.ref_la(mat, 1, nthreads=THREADS)
    assert got.np == want.np and got.nnz == want.nnz
    assert got.equals(want), got.first_difference(want)


@needs_ref
def test_basis_conversion_of_the_staircase_answer_matches_reference():
    mat = synth.staircase(20000, 5000, 20000, 65521, 0.02, 0.05, seed=1)
    exps = synth.distinct_monomials(mat.ncl + mat.ncr, 8, seed=5)
    want = oracle.basis_bench(mat, exps, nthreads=THREADS)
    got = oracle.basis_bench(
        mat, exps, keep_fn=la.function_address("gbgpu_linear_algebra_keep"),
        convert_fn=la.function_address("gbgpu_convert_sparse_matrix_rows_to_basis_elements"))
    assert got["np"] == want["np"] == 5000
    assert got["eld"] == want["eld"]
    assert got["digest"] == want["digest"]
    assert got["map_digest"] == want["map_digest"]


def _uniform(torch, p, shape, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.randint(0, p, shape, device="cuda", dtype=torch.int64,
                         generator=g).to(torch.int32)


@pytest.mark.parametrize("n,p", [(8192, 251), (8192, 65521), (8192, 2147483647),
                                 (16384, 65521)])
def test_dense_submul_at_size_exact(n, p):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    A, B, D = (_uniform(torch, p, (n, n), s) for s in (1, 2, 3))
    out = D.clone()
    opt = _lib.Options(_lib.FORM_TENSOR, 0, 1, 0, None)
    _lib.check(lib.gbgpu_dense_submul(p, n, n, n, A.data_ptr(), n, B.data_ptr(), n,
                                      out.data_ptr(), n, C.byref(opt)))
    torch.cuda.synchronize()
    A, B, D, out = (t.cpu().numpy() for t in (A, B, D, out))
    assert out.min() >= 0 and out.max() < p
    rng = np.random.default_rng(n + p)
    # sampled rows, exactly
    for i in rng.choice(n, size=4, replace=False):
        want = (D[i].astype(np.int64) - vecmat_mod(A[i], B, p)) % p
        assert np.array_equal(out[i].astype(np.int64), want), f"row {i}"
    # every row, Freivalds: out x == D x - A (B x)  (mod p)
    for _ in range(3):
        x = rng.integers(0, p, size=n, dtype=np.int64)
        lhs = matvec_mod(out, x, p)
        rhs = (matvec_mod(D, x, p) - matvec_mod(A, matvec_mod(B, x, p), p)) % p
        assert np.array_equal(lhs, rhs)


@needs_ref
@pytest.mark.parametrize("p", [251, 65521, 2147483647])
def test_dense_rref_8192_matches_reference(p):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    n, r = 8192, 6144
    L, R = _uniform(torch, p, (n, r), 11), _uniform(torch, p, (r, n), 12)
    Rn = torch.remainder(p - R.to(torch.int64), p).to(torch.int32)
    D = torch.zeros(n, n, device="cuda", dtype=torch.int32)
    opt = _lib.Options(_lib.FORM_TENSOR, 0, 1, 0, None)
    _lib.check(lib.gbgpu_dense_submul(p, n, n, r, L.data_ptr(), r, Rn.data_ptr(), n,
                                      D.data_ptr(), n, C.byref(opt)))  # D = L R
    torch.cuda.synchronize()
    D0 = D.cpu().numpy()
    piv = torch.empty(n, device="cuda", dtype=torch.int32)
    rank = C.c_int32()
    _lib.check(lib.gbgpu_dense_rref(p, n, n, D.data_ptr(), n, C.byref(rank), piv.data_ptr(),
                                    C.byref(opt)))
    torch.cuda.synchronize()
    got = dense_rref_rows(D.cpu().numpy(), rank.value, piv.cpu().numpy(), n)
    want, _ = oracle.ref_la(synth.dense_block_macaulay(D0, p), 1, nthreads=THREADS)
    assert rank.value == want.np == r
    assert got.equals(want), got.first_difference(want)


@needs_ref
def test_f4_dense_cubic_10_p31_every_la_call_matches_reference(tmp_path):
    """F4 on the dense cubic system in 10 variables (10 polynomials, all 286
    monomials of degree <= 3, p = 2^31 - 1, la option 1) with gb's own host
    code: every la call (src/f4.c:306) goes to libgbgpu.so and, on a copy of
    the matrix, to the reference la; the answers must agree bit for bit.  The
    run is compared round by round until the reference calls have used 40 s
    (the reference cannot finish this system); the largest matrix reached is
    checked to be at least 40000 rows (round 8: 42358 x 72876 with this seed)."""
    import subprocess
    import sys
    from oracle.f4_compare import parse_log
    log = tmp_path / "calls.log"
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run([sys.executable, "-m", "oracle.f4_compare", "--nvars", "10", "--ngens", "10",
                    "--maxdeg", "3", "--p", "2147483647", "--la-option", "1", "--seed", "10",
                    "--budget", "40", "--log", str(log), "--impl", "gpu"],
                   check=True, cwd=repo, timeout=1500)
    res = parse_log(str(log))
    calls = res["calls"]
    assert calls, res
    bad = [c for c in calls if not c["equal"]]
    assert not bad, bad
    assert max(c["nr"] for c in calls) >= 40000, calls
