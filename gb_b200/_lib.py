"""ctypes binding of libgbgpu.so (include/gbgpu.h).

The shared object is built in-tree by :mod:`gb_b200.build`.  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgbgpu.so")

GBGPU_OK = 0
GBGPU_EINVAL = -22
GBGPU_ENOMEM = -12
GBGPU_ENODEV = -19
GBGPU_ECUDA = -5
GBGPU_ETIMEDOUT = -110
GBGPU_ERANGE = -34

FORM_AUTO, FORM_PLAIN, FORM_TENSOR, FORM_BLOCKED_PLAIN = 0, 1, 2, 3

_PI64 = C.POINTER(C.c_int64)
_PI32 = C.POINTER(C.c_int32)


class Csr(C.Structure):
    _fields_ = [("p", C.c_int32), ("laopt", C.c_int32), ("nr", C.c_int32), ("ncl", C.c_int32),
                ("ncr", C.c_int32), ("row_ptr", C.c_void_p), ("cols", C.c_void_p),
                ("vals", C.c_void_p), ("val_bytes", C.c_int32)]


class Rows(C.Structure):
    _fields_ = [("np", C.c_int32), ("nnz", C.c_int64), ("row_ptr", _PI64), ("cols", _PI32),
                ("vals", _PI32)]


class Options(C.Structure):
    _fields_ = [("form", C.c_int32), ("device", C.c_int32), ("check", C.c_int32),
                ("profile", C.c_int32), ("stream", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_schur", C.c_double), ("ms_echelon", C.c_double),
                ("ms_rref", C.c_double), ("ms_compact", C.c_double),
                ("rows_reduced", C.c_int64), ("dense_rows", C.c_int64), ("rank", C.c_int64),
                ("echelon_rounds", C.c_int64), ("kernel_launches", C.c_int64),
                ("work_schur", C.c_int64), ("work_dense", C.c_int64),
                ("gemm_launches", C.c_int64), ("gemm_ms", C.c_double),
                ("gemm_int8_ops", C.c_double), ("form_used", C.c_int64),
                ("ms_classify", C.c_double), ("ms_check", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GbgpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gbgpu error {code}: {msg}")
        self.code = code


# every entry point declared in include/gbgpu.h
EXPORTS = [
    "gbgpu_linear_algebra", "gbgpu_interreduce_matrix_rows", "gbgpu_linear_algebra_status",
    "gbgpu_interreduce_matrix_rows_status", "gbgpu_reduce", "gbgpu_interreduce",
    "gbgpu_rows_free", "gbgpu_plan_create", "gbgpu_plan_run", "gbgpu_plan_result",
    "gbgpu_plan_stats", "gbgpu_plan_destroy", "gbgpu_reduce_batch", "gbgpu_layout",
    "gbgpu_last_error", "gbgpu_kernel_launches", "gbgpu_dense_submul", "gbgpu_dense_submul_host",
    "gbgpu_dense_submul_noalloc", "gbgpu_plan_result_into", "gbgpu_dense_rref",
    "gbgpu_plan_result_into_v", "gbgpu_plan_run_into_v", "gbgpu_autotune",
    "gbgpu_convert_hashes_to_columns_flat", "gbgpu_convert_hashes_to_columns",
    "gbgpu_sort_matrix_rows", "gbgpu_linear_algebra_keep", "gbgpu_linear_algebra_keep_status",
    "gbgpu_kept_answer", "gbgpu_convert_sparse_matrix_rows_to_basis_elements",
    "gbgpu_convert_sparse_matrix_rows_to_basis_elements_status", "gbgpu_plan_first_entry",
    "gbgpu_plan_map_columns", "gbgpu_symbolic_preprocessing",
    "gbgpu_symbolic_preprocessing_status",
]

_lib = None


def load(path: str = LIB_PATH):
    """Load the library (once).  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m gb_b200.build` "
                           "(the GPU path has no CPU fallback)")
    lib = C.CDLL(path)
    lib.gbgpu_reduce.argtypes = [C.POINTER(Csr), C.POINTER(Options), C.POINTER(Rows)]
    lib.gbgpu_interreduce.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.POINTER(Options), C.POINTER(Rows)]
    lib.gbgpu_rows_free.argtypes = [C.POINTER(Rows)]
    lib.gbgpu_rows_free.restype = None
    lib.gbgpu_plan_create.argtypes = [C.POINTER(Csr), C.POINTER(Options), C.POINTER(C.c_void_p)]
    lib.gbgpu_plan_run.argtypes = [C.c_void_p]
    lib.gbgpu_plan_result.argtypes = [C.c_void_p, C.POINTER(Rows)]
    lib.gbgpu_plan_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
    lib.gbgpu_plan_result_into.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_int64, C.c_int64, _PI32, _PI64]
    lib.gbgpu_plan_result_into_v.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_int32, C.c_int64, C.c_int64, _PI32, _PI64]
    lib.gbgpu_plan_run_into_v.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_int32, C.c_int64, C.c_int64, _PI32, _PI64]
    lib.gbgpu_plan_first_entry.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.gbgpu_plan_map_columns.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.gbgpu_plan_destroy.argtypes = [C.c_void_p]
    lib.gbgpu_plan_destroy.restype = None
    lib.gbgpu_reduce_batch.argtypes = [C.c_int32, C.POINTER(Csr), C.POINTER(Options),
                                       C.POINTER(Rows), _PI32]
    lib.gbgpu_layout.argtypes = [_PI64, C.c_int32]
    dense = [C.c_int32] * 4 + [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                               C.c_int64, C.POINTER(Options)]
    lib.gbgpu_dense_submul.argtypes = dense
    lib.gbgpu_dense_submul_host.argtypes = dense
    lib.gbgpu_dense_submul_noalloc.argtypes = [C.c_int32] * 4 + [
        C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32,
        C.c_void_p]
    lib.gbgpu_dense_rref.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int64,
                                     _PI32, C.c_void_p, C.POINTER(Options)]
    lib.gbgpu_autotune.argtypes = [C.c_int32, C.c_char_p]
    lib.gbgpu_convert_hashes_to_columns_flat.argtypes = [C.c_int32, C.c_int32] + [
        C.c_void_p] * 3 + [C.c_int32, C.c_int32] + [C.c_void_p] * 7 + [C.c_int32]
    lib.gbgpu_last_error.restype = C.c_char_p
    lib.gbgpu_kernel_launches.restype = C.c_int64
    _lib = lib
    return lib


def last_error() -> str:
    return load().gbgpu_last_error().decode(errors="replace")


def check(code: int) -> None:
    if code != GBGPU_OK:
        raise GbgpuError(code, last_error())
