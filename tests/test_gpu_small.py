"""GPU tests of the one-pass small-matrix path (gb_b200/csrc/small.cu): the
la calls gbgpu_reduce and the drop-in gbgpu_linear_algebra route there when a
matrix is small.  Its answers must equal the oracle's and the general plan
path's, bit for bit, for every kernel family, across growing sizes (the
session's buffers grow), from several host threads at once, and it must
reject contract violations like the general path."""
import threading

import numpy as np
import pytest

import oracle
from gb_b200 import _lib, la, synth
from gb_b200.matrix import MacaulayMatrix, load_captures
from helpers import capture_files

pytestmark = pytest.mark.gpu

PRIMES = [2, 3, 7, 101, 127, 251, 32003, 65521, 65537, 1000003, 2147483647]


def _plan_answer(m):
    plan = la.Plan(m, form=_lib.FORM_PLAIN)
    plan.run()
    try:
        return plan.result()
    finally:
        plan.close()


@pytest.mark.parametrize("p", PRIMES)
def test_small_path_matches_oracle_and_plan(p):
    for k, (nru, nrl, ncr) in enumerate([(5, 3, 4), (40, 30, 60), (120, 90, 200),
                                         (300, 80, 140), (30, 200, 40)]):
        m = synth.random_macaulay(nru, nrl, ncr, p, density=0.15, seed=k + p % 97,
                                  dup_rows=min(5, nrl))
        want, _ = oracle.oracle_la(m)
        got = la.linear_algebra(m)
        assert got.equals(want), (p, k, got.first_difference(want))
        assert _plan_answer(m).equals(got)


def test_small_path_on_every_captured_call():
    for f in capture_files():
        for c in load_captures(f):
            if c.kind != 0:
                continue
            got = la.linear_algebra(c.mat)
            assert got.equals(c.answer), (f, got.first_difference(c.answer))


def test_small_path_from_several_threads():
    mats = [synth.random_macaulay(60 + 10 * i, 40, 80, [101, 32003, 2147483647][i % 3],
                                  density=0.2, seed=i) for i in range(12)]
    want = [oracle.oracle_la(m)[0] for m in mats]
    errors = []

    def work(idx):
        try:
            for _ in range(3):
                for i in idx:
                    if not la.linear_algebra(mats[i]).equals(want[i]):
                        errors.append(i)
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(repr(e))

    ts = [threading.Thread(target=work, args=(list(range(j, 12, 4)),)) for j in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors


def test_small_path_rejects_contract_violations():
    m = synth.random_macaulay(10, 8, 12, 101, seed=6)
    bad = MacaulayMatrix(m.p, m.ncl, m.ncr, m.row_ptr, m.cols, m.vals.copy())
    bad.vals[bad.row_ptr[3] + 1] = 101  # coefficient == p
    with pytest.raises(_lib.GbgpuError) as ei:
        la.linear_algebra(bad)
    assert ei.value.code == _lib.GBGPU_EINVAL and "coefficient" in str(ei.value)
    # a good matrix right after a rejected one is reduced correctly
    assert la.linear_algebra(m).equals(oracle.oracle_la(m)[0])


def test_batch_of_small_matrices_is_one_launch():
    """A batch of small matrices (uneven shapes, several primes, one that
    breaks the contract) is reduced in ONE persistent launch with a device
    work queue; every answer equals the oracle's, the bad matrix alone fails."""
    lib = _lib.load()
    mats = []
    for i in range(40):
        p = PRIMES[i % len(PRIMES)]
        mats.append(synth.random_macaulay(20 + 7 * i, 10 + 3 * i, 30 + 5 * i, p, density=0.15,
                                          seed=100 + i, dup_rows=min(3, 10 + 3 * i)))
    bad = mats[7]
    mats[7] = MacaulayMatrix(bad.p, bad.ncl, bad.ncr, bad.row_ptr, bad.cols, bad.vals.copy())
    mats[7].vals[mats[7].row_ptr[2] + 1] = 0  # zero coefficient
    before = lib.gbgpu_kernel_launches()
    outs, status = la.reduce_batch(mats)
    assert lib.gbgpu_kernel_launches() - before == 1
    for i, m in enumerate(mats):
        if i == 7:
            assert status[i] == _lib.GBGPU_EINVAL and outs[i] is None
            continue
        assert status[i] == 0, (i, status[i])
        want, _ = oracle.oracle_la(m)
        assert outs[i].equals(want), (i, outs[i].first_difference(want))


def test_batch_mixed_small_and_blocked():
    mats = [synth.random_macaulay(30, 20, 40, 32003, density=0.2, seed=1),
            synth.staircase(1200, 400, 1500, 65521, seed=2),
            synth.random_macaulay(50, 30, 60, 2147483647, density=0.2, seed=3),
            synth.staircase(900, 300, 1000, 2147483647, seed=4)]
    outs, status = la.reduce_batch(mats)
    assert list(status) == [0, 0, 0, 0]
    for m, o in zip(mats, outs):
        assert o.equals(oracle.oracle_la(m)[0])
