"""The product path has no CPU fallback: without a CUDA device every compute
entry point of libgbgpu.so returns an error instead of computing on the host,
and no product source refers to the oracle (the CPU restatement that the
tests check against)."""
import os
import re

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
