"""The product path has no CPU fallback: without a CUDA device every compute
entry point of libgbgpu.so returns an error instead of computing on the host,
and no product source refers to the oracle (the CPU restatement that the
tests check against)."""
import ctypes as C
import os
import re

import numpy as np
import pytest
import torch

from gb_b200 import _lib, la, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

no_gpu = pytest.mark.skipif(torch.cuda.is_available(), reason="needs a host without a GPU")


@no_gpu
def test_plan_fails_loudly_without_a_device():
    m = synth.staircase(60, 20, 50, 65521, seed=1)
    with pytest.raises(_lib.GbgpuError) as e:
        p = la.Plan(m)
        p.run()
    assert e.value.code == _lib.GBGPU_ENODEV


@no_gpu
@pytest.mark.parametrize("p", [251, 65521, 2147483647])
def test_one_shot_entry_points_fail_loudly_without_a_device(p):
    m = synth.staircase(40, 12, 30, p, seed=2)
    with pytest.raises(_lib.GbgpuError) as e:
        la.linear_algebra(m)
    assert e.value.code == _lib.GBGPU_ENODEV
    # a batch runs no matrix: the call fails with the device error
    with pytest.raises(_lib.GbgpuError) as e:
        la.reduce_batch([m, m])
    assert e.value.code == _lib.GBGPU_ENODEV


@no_gpu
@pytest.mark.parametrize("form", [_lib.FORM_TENSOR, _lib.FORM_PLAIN])
def test_dense_product_fails_loudly_without_a_device(form):
    lib = _lib.load()
    a = np.ones((4, 4), dtype=np.uint32)
    out = np.zeros((4, 4), dtype=np.uint32)
    opt = _lib.Options(form, 0, 1, 0, None)
    rc = lib.gbgpu_dense_submul_host(101, 4, 4, 4, a.ctypes.data, 4, a.ctypes.data, 4,
                                     out.ctypes.data, 4, C.byref(opt))
    assert rc == _lib.GBGPU_ENODEV
    assert not out.any()  # nothing computed on the host


@no_gpu
def test_column_conversion_fails_loudly_without_a_device():
    lib = _lib.load()
    nv, n, nr = 2, 3, 2
    exps = np.array([[2, 0], [1, 1], [0, 2]], dtype=np.int16)
    deg = np.full(n, 2, dtype=np.int32)
    idx = np.array([2, 1, 1], dtype=np.int32)
    row_ptr = np.array([0, 2, 4], dtype=np.int64)
    hashes = np.array([1, 2, 2, 3], dtype=np.int32)
    hcm = np.zeros(n, np.int32)
    order = np.zeros(nr, np.int32)
    optr = np.zeros(nr + 1, np.int64)
    cols = np.zeros(4, np.int32)
    ncl = C.c_int32()
    rc = lib.gbgpu_convert_hashes_to_columns_flat(
        nv, n, exps.ctypes.data, deg.ctypes.data, idx.ctypes.data, 0, nr, row_ptr.ctypes.data,
        hashes.ctypes.data, hcm.ctypes.data, C.byref(ncl), order.ctypes.data, optr.ctypes.data,
        cols.ctypes.data, 0)
    assert rc == _lib.GBGPU_ENODEV


def _product_sources():
    for sub in ("gb_b200", "include"):
        for dirpath, _, files in os.walk(os.path.join(ROOT, sub)):
            for f in files:
                if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp", ".c")):
                    yield os.path.join(dirpath, f)


def test_no_product_source_refers_to_the_oracle():
    bad = []
    pat = re.compile(r"\boracle\b|gbla_oracle|libgbref|oracle/_ref")
    for path in _product_sources():
        with open(path, encoding="utf-8", errors="replace") as fh:
            for n, line in enumerate(fh, 1):
                if pat.search(line):
                    bad.append(f"{os.path.relpath(path, ROOT)}:{n}: {line.strip()}")
    assert not bad, "product sources mention the oracle:\n" + "\n".join(bad)
