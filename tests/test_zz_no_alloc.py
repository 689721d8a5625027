"""GPU test of gbgpu_dense_submul_noalloc, the entry point that allocates
nothing, for callers that must not call cudaMalloc/cudaFree once they run (a
device-memory budget reserved up front, or a host allocator that owns all
device memory).  It must return exactly what gbgpu_dense_submul returns on the
same inputs, on two calls in a row (the second call reuses the fixed scratch
array the first one left behind), leave the device's allocations as they were,
and reject work larger than its fixed scratch.  The file name makes pytest
collect it last."""
import ctypes as C

import numpy as np
import pytest

from gb_b200 import _lib

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 32 << 20  # the library's fixed scratch array


def _device_mats(torch, p, M, N, K, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    mk = lambda r, c: torch.randint(0, p, (r, c), device="cuda", dtype=torch.int64,
                                    generator=g).to(torch.int32)
    return mk(M, K), mk(K, N), mk(M, N)


def _pool_used_bytes(device: int):
    """Bytes in use in the device's default stream-ordered memory pool (the
    pool cudaMallocAsync draws from), or None where cuda-python is absent."""
    try:
        from cuda.bindings import runtime as rt
    except ImportError:
        return None
    err, pool = rt.cudaDeviceGetDefaultMemPool(device)
    if err != rt.cudaError_t.cudaSuccess:
        return None
    err, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    return int(used) if err == rt.cudaError_t.cudaSuccess else None


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    opt = _lib.Options(_lib.FORM_TENSOR, 0, 1, 0, None)
    for call, (p, M, N, K) in enumerate([(65521, 300, 260, 700), (2147483647, 257, 130, 1111)]):
        A, B, D = _device_mats(torch, p, M, N, K, seed=11 + call)
        D_ref = D.clone()
        _lib.check(lib.gbgpu_dense_submul(p, M, N, K, A.data_ptr(), K, B.data_ptr(), N,
                                          D_ref.data_ptr(), N, C.byref(opt)))
        D_new = D.clone()
        torch.cuda.synchronize()
        torch_before = torch.cuda.memory_allocated()
        free_before = torch.cuda.mem_get_info()[0]
        pool_before = _pool_used_bytes(0)
        _lib.check(lib.gbgpu_dense_submul_noalloc(p, M, N, K, A.data_ptr(), K, B.data_ptr(), N,
                                                  D_new.data_ptr(), N, 0, None))
        torch.cuda.synchronize()
        # nothing was allocated: torch's allocator and the stream-ordered pool
        # read as before the call.  The driver's free memory may drop once, by
        # at most the library's fixed 32 MiB scratch array, when the first call
        # makes the driver load that array on this GPU (lazy module loading);
        # after that it must not move.
        assert torch.cuda.memory_allocated() == torch_before
        assert _pool_used_bytes(0) == pool_before
        drop = free_before - torch.cuda.mem_get_info()[0]
        if call == 0:
            assert 0 <= drop <= SCRATCH_BYTES + (2 << 20), drop
        else:
            assert drop == 0, drop
        assert torch.equal(D_new, D_ref), f"call {call}: results differ"
        assert not torch.equal(D_new, D)  # the update did something


def test_noalloc_rejects_work_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    # L = 2 limb planes of (M + N) x K bytes: 2 * (8192 + 8192) * 4096 = 128 MiB > 32 MiB
    rc = lib.gbgpu_dense_submul_noalloc(65521, 8192, 8192, 4096, buf.data_ptr(), 4096,
                                        buf.data_ptr(), 8192, buf.data_ptr(), 8192, 0, None)
    assert rc == _lib.GBGPU_ERANGE
    assert "scratch" in _lib.last_error()
    rc = lib.gbgpu_dense_submul_noalloc(65522, 4, 4, 4, buf.data_ptr(), 4, buf.data_ptr(), 4,
                                        buf.data_ptr(), 4, 0, None)
    assert rc == _lib.GBGPU_EINVAL  # even modulus
