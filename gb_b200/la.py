"""Host-side mirror of the reference's linear-algebra interface.

``linear_algebra(mat)`` and ``interreduce_matrix_rows(p, nc, rows)`` take
the same arguments and return the same rows as gb's
``linear_algebra(mat, bs, st)`` (src/la_ff_16.c:1430-1507 and twins) and
``interreduce_matrix_rows(mat, bs, st)`` (src/la_ff_16.c:1605-1673), on flat
CSR matrices, computed by libgbgpu.so on the GPU.  Errors raise
:class:`gb_b200._lib.GbgpuError` (the reference has no error path; invalid
input is rejected with GBGPU_EINVAL instead of being reduced into garbage).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .matrix import MacaulayMatrix, ReducedRows


def _options(form: int = _lib.FORM_AUTO, device: int = 0, stream: Optional[int] = None,
             profile: bool = False):
    return _lib.Options(form, device, 1, 1 if profile else 0, stream)


def _csr(mat: MacaulayMatrix) -> _lib.Csr:
    return _lib.Csr(mat.p, mat.laopt, mat.nr, mat.ncl, mat.ncr,
                    mat.row_ptr.ctypes.data, mat.cols.ctypes.data, mat.vals.ctypes.data)


def _take(lib, rows: _lib.Rows) -> ReducedRows:
    n, nnz = rows.np, rows.nnz
    ptr = np.ctypeslib.as_array(rows.row_ptr, shape=(n + 1,)).copy()
    cols = np.ctypeslib.as_array(rows.cols, shape=(max(nnz, 1),))[:nnz].copy()
    vals = np.ctypeslib.as_array(rows.vals, shape=(max(nnz, 1),))[:nnz].copy()
    lib.gbgpu_rows_free(C.byref(rows))
    return ReducedRows(ptr, cols, vals)


def linear_algebra(mat: MacaulayMatrix, form: int = _lib.FORM_AUTO, device: int = 0
                   ) -> ReducedRows:
    """New pivots of one Macaulay matrix (descending lead, monic, columns >= ncl)."""
    lib = _lib.load()
    out = _lib.Rows()
    opt = _options(form, device)
    _lib.check(lib.gbgpu_reduce(C.byref(_csr(mat)), C.byref(opt), C.byref(out)))
    return _take(lib, out)


def interreduce_matrix_rows(p: int, nc: int, rows: ReducedRows, device: int = 0
                            ) -> ReducedRows:
    """Full interreduction of rows with distinct leads (ascending lead order)."""
    lib = _lib.load()
    out = _lib.Rows()
    opt = _options(_lib.FORM_AUTO, device)
    _lib.check(lib.gbgpu_interreduce(p, rows.np, nc, rows.row_ptr.ctypes.data,
                                     rows.cols.ctypes.data, rows.vals.ctypes.data,
                                     C.byref(opt), C.byref(out)))
    return _take(lib, out)


def reduce_batch(mats: Sequence[MacaulayMatrix], form: int = _lib.FORM_AUTO, device: int = 0
                 ) -> Tuple[List[Optional[ReducedRows]], List[int]]:
    """Reduce independent matrices in one call; a failing matrix yields None
    and its status code, the others are unaffected."""
    lib = _lib.load()
    n = len(mats)
    csrs = (_lib.Csr * max(n, 1))(*[_csr(m) for m in mats])
    outs = (_lib.Rows * max(n, 1))()
    status = (C.c_int32 * max(n, 1))()
    opt = _options(form, device)
    _lib.check(lib.gbgpu_reduce_batch(n, csrs, C.byref(opt), outs,
                                      C.cast(status, C.POINTER(C.c_int32))))
    res = []
    for i in range(n):
        res.append(_take(lib, outs[i]) if status[i] == 0 else None)
    return res, [int(status[i]) for i in range(n)]


class Plan:
    """Device-resident copy of one matrix for repeated runs (benchmarks)."""

    def __init__(self, mat: MacaulayMatrix, form: int = _lib.FORM_AUTO, device: int = 0,
                 profile: bool = False):
        self._lib = _lib.load()
        self._mat = mat  # keep host arrays alive until the upload finished
        self._h = C.c_void_p()
        opt = _options(form, device, profile=profile)
        _lib.check(self._lib.gbgpu_plan_create(C.byref(_csr(mat)), C.byref(opt),
                                               C.byref(self._h)))

    def run(self) -> None:
        _lib.check(self._lib.gbgpu_plan_run(self._h))

    def result(self) -> ReducedRows:
        out = _lib.Rows()
        _lib.check(self._lib.gbgpu_plan_result(self._h, C.byref(out)))
        return _take(self._lib, out)

    def first_entry(self) -> np.ndarray:
        """Per right column j: the position of its first entry in the answer's
        entry array (-1: none) -- the order in which src/hash.c:604-669
        inserts the answer's monomials into the basis hash table."""
        n = int(self._mat.ncr)
        out = np.empty(max(n, 1), dtype=np.int64)
        _lib.check(self._lib.gbgpu_plan_first_entry(self._h, out.ctypes.data, n))
        return out[:n]

    def map_columns(self, mapping: np.ndarray) -> None:
        """Rewrite the answer on the device: column ncl + j becomes mapping[j]."""
        m = np.ascontiguousarray(mapping, dtype=np.int32)
        if m.shape[0] != self._mat.ncr:
            raise ValueError("mapping needs ncr entries")
        _lib.check(self._lib.gbgpu_plan_map_columns(self._h, m.ctypes.data, int(m.shape[0])))

    def stats(self) -> dict:
        st = _lib.Stats()
        _lib.check(self._lib.gbgpu_plan_stats(self._h, C.byref(st)))
        return st.as_dict()

    def close(self) -> None:
        if self._h:
            self._lib.gbgpu_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def layout() -> np.ndarray:
    out = np.zeros(64, dtype=np.int64)
    n = _lib.load().gbgpu_layout(out.ctypes.data_as(C.POINTER(C.c_int64)), 64)
    return out[:n]


def function_address(name: str) -> int:
    """Raw address of an exported C function (to hand to the reference's hooks)."""
    return C.cast(getattr(_lib.load(), name), C.c_void_p).value
