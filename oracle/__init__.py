"""TEST INFRASTRUCTURE ONLY: Python bindings of the CPU oracle and of the
reference build.

* ``liboracle.so`` -- the plain-C restatement in ``gbla_oracle.c``.
* ``_ref/libgbref.so`` -- the reference gb library compiled from its own
  sources by ``ref/Makefile`` (present only where it was built; it travels
  with the repository snapshot as a built file).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, always as the checker or the timed baseline,
never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

from gb_b200.matrix import MacaulayMatrix, ReducedRows

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgbref.so")
# gb compiled with its two linear-algebra call sites rerouted to libgbgpu.so (linked to it)
GB_GPU_SO = os.path.join(HERE, "_ref", "libgb_gpu.so")
# the same with the hash -> column mapping and row sort rerouted too (ref/gb_gpu_full.c)
GB_GPU_FULL_SO = os.path.join(HERE, "_ref", "libgb_gpu_full.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_PI64 = C.POINTER(C.c_int64)
_PI32 = C.POINTER(C.c_int32)

_oracle = None
_ref = None


def build(reference: Optional[str] = None) -> None:
    """Compile liboracle.so and, when the reference sources exist, _ref/."""
    env = dict(os.environ)
    if reference:
        env["REFERENCE"] = reference
    subprocess.run(["make", "-s", "-C", HERE], check=True, env=env)


def _load_oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = C.CDLL(ORACLE_SO)
        lib.oracle_la_csr.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                      _i64p, _i32p, _i32p, _PI32, C.POINTER(_PI64),
                                      C.POINTER(_PI32), C.POINTER(_PI32), _PI64]
        lib.oracle_interreduce_csr.argtypes = [C.c_int32, C.c_int32, C.c_int32, _i64p, _i32p,
                                               _i32p, C.POINTER(_PI64), C.POINTER(_PI32),
                                               C.POINTER(_PI32), _PI64]
        lib.oracle_free.argtypes = [C.c_void_p]
        lib.oracle_inverse.argtypes = [C.c_int32, C.c_int32]
        lib.oracle_inverse.restype = C.c_int32
        lib.oracle_normalize_row.argtypes = [_i32p, C.c_int64, C.c_int32]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _load_ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference build oracle/_ref/libgbref.so is absent")
        lib = C.CDLL(REF_SO)
        lib.gbref_la_csr.argtypes = [C.c_int32] * 8 + [
            _i64p, _i32p, _i32p, _PI32, C.POINTER(_PI64), C.POINTER(_PI32),
            C.POINTER(_PI32), C.POINTER(C.c_double)]
        lib.gbref_interreduce_csr.argtypes = [C.c_int32, C.c_int32, C.c_int32, _i64p, _i32p,
                                              _i32p, C.POINTER(_PI64), C.POINTER(_PI32),
                                              C.POINTER(_PI32), C.POINTER(C.c_double)]
        lib.gbref_free.argtypes = [C.c_void_p]
        lib.gbref_set_la.argtypes = [C.c_void_p, C.c_void_p]
        lib.gbref_set_capture.argtypes = [C.c_char_p]
        lib.gbref_layout.argtypes = [_i64p, C.c_int]
        lib.gbref_layout.restype = C.c_int
        lib.gbref_hook_calls.restype = C.c_int64
        lib.gbref_hook_seconds.restype = C.c_double
        lib.gbref_basis_bench.argtypes = [C.c_int32] * 8 + [
            _i64p, _i32p, _i32p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
            _PI32, _PI32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        lib.f4_julia.restype = C.c_int64
        lib.f4_julia.argtypes = [_PI32, C.POINTER(_PI32), C.POINTER(_PI32), C.POINTER(C.c_void_p),
                                 _i32p, _i32p, _i32p] + [C.c_int32] * 12
        lib.free_julia_data.argtypes = [C.POINTER(_PI32), C.POINTER(_PI32),
                                        C.POINTER(C.c_void_p), C.c_int64, C.c_int64]
        _ref = lib
    return _ref


def _take(free, n: int, ptr, cols, vals) -> ReducedRows:
    optr = np.ctypeslib.as_array(ptr, shape=(n + 1,)).copy()
    nnz = int(optr[-1])
    oc = np.ctypeslib.as_array(cols, shape=(max(nnz, 1),))[:nnz].copy()
    ov = np.ctypeslib.as_array(vals, shape=(max(nnz, 1),))[:nnz].copy()
    for x in (ptr, cols, vals):
        free(C.cast(x, C.c_void_p))
    return ReducedRows(optr, oc, ov)


def oracle_la(mat: MacaulayMatrix, laopt: Optional[int] = None, with_work: bool = False):
    """The oracle's answer for one Macaulay matrix and its work count W
    (pivot-row entries applied, single-threaded order).  With ``with_work``
    W is split as (known pivots, new pivots)."""
    lib = _load_oracle()
    npv = C.c_int32()
    ptr, cols, vals = _PI64(), _PI32(), _PI32()
    work = (C.c_int64 * 2)()
    rc = lib.oracle_la_csr(mat.p, mat.laopt if laopt is None else laopt, mat.nr, mat.ncl,
                           mat.ncr, mat.row_ptr, mat.cols, mat.vals, C.byref(npv),
                           C.byref(ptr), C.byref(cols), C.byref(vals),
                           C.cast(work, _PI64))
    if rc != 0:
        raise ValueError(f"oracle rejected the matrix (rc={rc})")
    rows = _take(lib.oracle_free, npv.value, ptr, cols, vals)
    if with_work:
        return rows, (work[0], work[1])
    return rows, work[0] + work[1]


def oracle_interreduce(p: int, nc: int, rows: ReducedRows) -> Tuple[ReducedRows, int]:
    lib = _load_oracle()
    ptr, cols, vals = _PI64(), _PI32(), _PI32()
    work = (C.c_int64 * 2)()
    rc = lib.oracle_interreduce_csr(p, rows.np, nc, rows.row_ptr, rows.cols, rows.vals,
                                    C.byref(ptr), C.byref(cols), C.byref(vals),
                                    C.cast(work, _PI64))
    if rc != 0:
        raise ValueError(f"oracle rejected the rows (rc={rc})")
    return _take(lib.oracle_free, rows.np, ptr, cols, vals), work[0] + work[1]


def oracle_normalize(row: np.ndarray, p: int) -> np.ndarray:
    r = np.ascontiguousarray(row, dtype=np.int32).copy()
    _load_oracle().oracle_normalize_row(r, r.shape[0], p)
    return r


def ref_la(mat: MacaulayMatrix, laopt: Optional[int] = None, nthreads: int = 1
           ) -> Tuple[ReducedRows, float]:
    """The reference's own la on one matrix: (answer, seconds of the la call)."""
    lib = _load_ref()
    nru, nrl = mat.split_counts()
    npv = C.c_int32()
    ptr, cols, vals = _PI64(), _PI32(), _PI32()
    secs = C.c_double()
    rc = lib.gbref_la_csr(mat.p, mat.laopt if laopt is None else laopt, nthreads, mat.nr,
                          nru, nrl, mat.ncl, mat.ncr, mat.row_ptr, mat.cols, mat.vals,
                          C.byref(npv), C.byref(ptr), C.byref(cols), C.byref(vals),
                          C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"reference la failed (rc={rc})")
    return _take(lib.gbref_free, npv.value, ptr, cols, vals), secs.value


def ref_interreduce(p: int, nc: int, rows: ReducedRows) -> Tuple[ReducedRows, float]:
    lib = _load_ref()
    ptr, cols, vals = _PI64(), _PI32(), _PI32()
    secs = C.c_double()
    rc = lib.gbref_interreduce_csr(p, rows.np, nc, rows.row_ptr, rows.cols, rows.vals,
                                   C.byref(ptr), C.byref(cols), C.byref(vals), C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"reference interreduce failed (rc={rc})")
    return _take(lib.gbref_free, rows.np, ptr, cols, vals), secs.value


def basis_bench(mat: MacaulayMatrix, exps: np.ndarray, keep_fn: Optional[int] = None,
                convert_fn: Optional[int] = None, nthreads: int = 1) -> dict:
    """One matrix through the la and then src/convert.c:137-280 (the answer
    turned into basis elements of a fresh basis and basis hash table), with
    the reference's own functions or, when given, the raw addresses of
    gbgpu_linear_algebra_keep / gbgpu_convert_sparse_matrix_rows_to_basis_
    elements.  ``exps`` (nc x nv int16, distinct rows) are the column
    monomials.  Returns the conversion's seconds, np, bht->eld and digests of
    the new basis elements and of the table's hash map."""
    lib = _load_ref()
    nru, nrl = mat.split_counts()
    exps = np.ascontiguousarray(exps, dtype=np.int16)
    secs = C.c_double()
    npv, eld = C.c_int32(), C.c_int32()
    dig, mdig = C.c_uint64(), C.c_uint64()
    rc = lib.gbref_basis_bench(mat.p, int(exps.shape[1]), nthreads, mat.nr, nru, nrl, mat.ncl,
                               mat.ncr, mat.row_ptr, mat.cols, mat.vals, exps.ctypes.data,
                               keep_fn, convert_fn, C.byref(secs), C.byref(npv), C.byref(eld),
                               C.byref(dig), C.byref(mdig))
    if rc != 0:
        raise RuntimeError(f"basis bench failed (rc={rc})")
    return {"seconds": secs.value, "np": npv.value, "eld": eld.value, "digest": dig.value,
            "map_digest": mdig.value}


def ref_layout() -> np.ndarray:
    out = np.zeros(64, dtype=np.int64)
    n = _load_ref().gbref_layout(out, 64)
    return out[:n]


def _f4_binding(lib):
    lib.f4_julia.restype = C.c_int64
    lib.f4_julia.argtypes = [_PI32, C.POINTER(_PI32), C.POINTER(_PI32), C.POINTER(C.c_void_p),
                             _i32p, _i32p, _i32p] + [C.c_int32] * 12
    lib.free_julia_data.argtypes = [C.POINTER(_PI32), C.POINTER(_PI32),
                                    C.POINTER(C.c_void_p), C.c_int64, C.c_int64]
    return lib


def _run_f4(lib, case: dict):
    bld = C.c_int32()
    blen, bexp = _PI32(), _PI32()
    bcf = C.c_void_p()
    lens = np.ascontiguousarray(case["lens"], dtype=np.int32)
    exps = np.ascontiguousarray(case["exps"], dtype=np.int32)
    cfs = np.ascontiguousarray(case["cfs"], dtype=np.int32)
    lib.f4_julia(C.byref(bld), C.byref(blen), C.byref(bexp), C.byref(bcf), lens, exps, cfs,
                 case["field_char"], case["mon_order"], case["nr_vars"], case["nr_gens"],
                 case["ht_size"], case["nr_threads"], case["max_nr_pairs"],
                 case["reset_hash_table"], case["la_option"], case["reduce_gb"], 0, 0)
    n = bld.value
    lens_out = np.ctypeslib.as_array(blen, shape=(n,)).copy()
    nterms = int(lens_out.sum())
    cf_ptr = C.cast(bcf, _PI32)
    cfs_out = np.ctypeslib.as_array(cf_ptr, shape=(max(nterms, 1),))[:nterms].copy()
    exps_out = np.ctypeslib.as_array(bexp, shape=(max(nterms * case["nr_vars"], 1),))[
        : nterms * case["nr_vars"]].copy()
    lib.free_julia_data(C.byref(blen), C.byref(bexp), C.byref(bcf), n, case["field_char"])
    return lens_out, cfs_out, exps_out


_gb_gpu = None


def gb_gpu_available() -> bool:
    return os.path.exists(GB_GPU_SO)


def gb_gpu_f4(case: dict):
    """F4 of gb compiled with the two-macro drop-in recipe: every linear-algebra
    call goes to libgbgpu.so.  Returns (lens, cfs, exps) of the basis."""
    global _gb_gpu
    if _gb_gpu is None:
        _gb_gpu = _f4_binding(C.CDLL(GB_GPU_SO))
    return _run_f4(_gb_gpu, case)


_gb_gpu_full = None


def gb_gpu_full_available() -> bool:
    return os.path.exists(GB_GPU_FULL_SO)


def gb_gpu_full_f4(case: dict):
    """F4 of gb with the linear algebra AND the conversion / row sort before it
    on libgbgpu.so (ref/gb_gpu_full.c).  Returns (lens, cfs, exps)."""
    global _gb_gpu_full
    if _gb_gpu_full is None:
        _gb_gpu_full = _f4_binding(C.CDLL(GB_GPU_FULL_SO))
    return _run_f4(_gb_gpu_full, case)


def ref_f4(case: dict, la_fn=None, ir_fn=None, capture_dir: Optional[str] = None):
    """Run the reference's F4 (f4_julia, src/f4.c:190) on a golden case.

    ``la_fn`` / ``ir_fn`` are raw C function addresses with the reference's
    linear_algebra / interreduce_matrix_rows signatures (for example the GPU
    library's ``gbgpu_linear_algebra``); None keeps the reference's own.
    Returns (lens, cfs, exps) of the exported basis."""
    lib = _load_ref()
    lib.gbref_set_la(la_fn, ir_fn)
    lib.gbref_set_capture(capture_dir.encode() if capture_dir else None)
    try:
        return _run_f4(lib, case)
    finally:
        lib.gbref_set_la(None, None)
        lib.gbref_set_capture(None)


def ref_convert(nv: int, exps: np.ndarray, deg: np.ndarray, idx: np.ndarray, mo: int,
                row_ptr: np.ndarray, hashes: np.ndarray):
    """The reference's convert_hashes_to_columns + sort_matrix_rows
    (src/convert.c:30-135, src/order.c:125-131) on one round's flat data.
    Returns (hcm, ncl, row_order, out_cols, seconds)."""
    lib = _load_ref()
    n = int(exps.shape[0])
    nr = int(row_ptr.shape[0] - 1)
    exps = np.ascontiguousarray(exps, dtype=np.int16)
    deg = np.ascontiguousarray(deg, dtype=np.int32)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    hashes = np.ascontiguousarray(hashes, dtype=np.int32)
    hcm = np.zeros(max(n, 1), dtype=np.int32)
    order = np.zeros(max(nr, 1), dtype=np.int32)
    cols = np.zeros(max(int(row_ptr[-1]), 1), dtype=np.int32)
    ncl = C.c_int32()
    secs = C.c_double()
    lib.gbref_convert_csr.argtypes = [C.c_int32, C.c_int32] + [C.c_void_p] * 3 + [
        C.c_int32, C.c_int32] + [C.c_void_p] * 2 + [C.c_void_p, C.POINTER(C.c_int32)] + [
        C.c_void_p] * 2 + [C.POINTER(C.c_double)]
    rc = lib.gbref_convert_csr(nv, n, exps.ctypes.data, deg.ctypes.data, idx.ctypes.data, mo, nr,
                               row_ptr.ctypes.data, hashes.ctypes.data, hcm.ctypes.data,
                               C.byref(ncl), order.ctypes.data, cols.ctypes.data, C.byref(secs))
    if rc != 0:
        raise RuntimeError("reference conversion failed")
    return hcm[:n], ncl.value, order[:nr], cols[:int(row_ptr[-1])], secs.value
