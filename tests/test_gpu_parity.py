"""GPU parity tests: libgbgpu.so (called through its C ABI) against the oracle
and the reference's captured answers, bit-exact (integer work: no tolerance).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from gb_b200 import _lib, la, synth
from gb_b200.matrix import MacaulayMatrix, ReducedRows
from tests.helpers import all_captures, as_rows, f4_cases

pytestmark = pytest.mark.gpu

CAPTURES = all_captures()
FORMS = [_lib.FORM_PLAIN, _lib.FORM_TENSOR, _lib.FORM_BLOCKED_PLAIN]


def check_same(got: ReducedRows, want: ReducedRows):
    assert got.equals(want), got.first_difference(want)


@pytest.mark.parametrize("name,k,cap", CAPTURES, ids=[f"{n}-{k}" for n, k, _ in CAPTURES])
def test_gpu_matches_reference_capture(name, k, cap):
    if cap.kind == 0:
        for form in FORMS:
            check_same(la.linear_algebra(cap.mat, form=form), cap.answer)
    else:
        got = la.interreduce_matrix_rows(cap.mat.p, cap.mat.nc, as_rows(cap.mat))
        check_same(got, cap.answer)


PRIMES = [2, 3, 101, 127, 251, 32003, 65521, 65537, 131071, 1000003, 2147483647]


@pytest.mark.parametrize("p", PRIMES)
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_gpu_matches_oracle_random(p, seed):
    m = synth.random_macaulay(40, 60, 50, p, density=0.08, seed=seed, dup_rows=5,
                              right_only_frac=0.3)
    want, _ = oracle.oracle_la(m)
    for form in FORMS:
        check_same(la.linear_algebra(m, form=form), want)


@pytest.mark.parametrize("p", [251, 32003, 65521, 2147483647])
def test_gpu_matches_oracle_staircase(p):
    m = synth.staircase(1500, 400, 1500, p, seed=7)
    want, _ = oracle.oracle_la(m, 1)
    for form in FORMS:
        check_same(la.linear_algebra(m, form=form), want)


def test_gpu_wide_matrix_global_accumulators():
    # nc and ncr beyond the shared-memory accumulator: global scratch path
    m = synth.random_macaulay(400, 40, 60000, 65521, density=0.0015, seed=11, dup_rows=3)
    want, _ = oracle.oracle_la(m)
    for form in FORMS:
        check_same(la.linear_algebra(m, form=form), want)
    m = synth.random_macaulay(300, 30, 70000, 2147483647, density=0.001, seed=12)
    want, _ = oracle.oracle_la(m)
    for form in FORMS:
        check_same(la.linear_algebra(m, form=form), want)


def test_gpu_small_path_repeatable_on_wide_blocks():
    """The one-CTA echelon of the small-matrix path on 100 x 300 right blocks
    (several load passes per thread before the lead inverses are taken): every
    run, single and batched, equals the oracle, for primes near 2^31 and 2^16."""
    base = synth.integer_staircase(400, 100, 300, bound=1 << 6, dmin=0.02, dmax=0.05, seed=1)
    primes = synth.largest_primes_below(1 << 31, 12) + synth.largest_primes_below(1 << 16, 4)
    imgs = [synth.image_mod(base, p) for p in primes]
    wants = [oracle.oracle_la(m)[0] for m in imgs]
    for _ in range(3):
        for m, want in zip(imgs, wants):
            check_same(la.linear_algebra(m), want)
        got, status = la.reduce_batch(imgs)
        assert status == [0] * len(imgs)
        for g, want in zip(got, wants):
            check_same(g, want)


@pytest.mark.parametrize("p", [251, 65521, 1000003, 2147483647])
def test_gpu_blocked_many_rounds(p):
    # many C|D rows on few leads with a rank-deficient right block: several
    # claiming rounds and pivot blocks that span more than one 128-block
    m = synth.random_macaulay(300, 700, 400, p, density=0.05, seed=21, dup_rows=40)
    want, _ = oracle.oracle_la(m)
    for form in FORMS:
        check_same(la.linear_algebra(m, form=form), want)


def test_gpu_edge_cases():
    for form in FORMS:
        # no rows to reduce
        m = synth.random_macaulay(20, 0, 10, 101, seed=1)
        want, _ = oracle.oracle_la(m)
        assert want.np == 0
        check_same(la.linear_algebra(m, form=form), want)
        # every lower row is a copy of a known pivot: everything reduces to zero
        m = synth.random_macaulay(20, 12, 10, 32003, seed=2, dup_rows=12)
        assert la.linear_algebra(m, form=form).np == 0
        # empty right block
        m = synth.random_macaulay(15, 10, 0, 65521, seed=3, density=0.3)
        assert la.linear_algebra(m, form=form).np == 0
        # one right column
        m = synth.random_macaulay(15, 10, 1, 65521, seed=4, density=0.3)
        want, _ = oracle.oracle_la(m)
        check_same(la.linear_algebra(m, form=form), want)
        # many rows colliding on few leads, rank-deficient right block
        m = synth.random_macaulay(3, 80, 20, 7, seed=5, density=0.5)
        want, _ = oracle.oracle_la(m)
        check_same(la.linear_algebra(m, form=form), want)


def _expect_einval(m):
    with pytest.raises(_lib.GbgpuError) as ei:
        la.linear_algebra(m)
    assert ei.value.code == _lib.GBGPU_EINVAL


def test_gpu_rejects_contract_violations():
    m = synth.random_macaulay(10, 8, 12, 101, seed=6)
    bad = MacaulayMatrix(m.p, m.ncl, m.ncr, m.row_ptr, m.cols, m.vals.copy())
    bad.vals[0] = 2
    _expect_einval(bad)  # not monic
    _expect_einval(MacaulayMatrix(m.p, m.ncl + 1, m.ncr - 1, m.row_ptr, m.cols, m.vals))
    bad = MacaulayMatrix(m.p, m.ncl, m.ncr, m.row_ptr, m.cols, m.vals.copy())
    bad.vals[-1] = m.p
    _expect_einval(bad)  # coefficient out of range
    bad = MacaulayMatrix(m.p, m.ncl, m.ncr, m.row_ptr, m.cols.copy(), m.vals)
    bad.cols[-1] = m.nc + 5
    _expect_einval(bad)  # column out of range
    # the library still works after rejecting input
    want, _ = oracle.oracle_la(m)
    check_same(la.linear_algebra(m), want)


def test_gpu_batch_isolates_failures():
    mats = [synth.random_macaulay(30, 20, 30, p, seed=s, density=0.1)
            for s, p in enumerate([101, 32003, 65521, 2147483647, 251])]
    bad = MacaulayMatrix(mats[2].p, mats[2].ncl, mats[2].ncr, mats[2].row_ptr, mats[2].cols,
                         mats[2].vals.copy())
    bad.vals[0] = 3
    mats[2] = bad
    outs, status = la.reduce_batch(mats)
    assert status[2] == _lib.GBGPU_EINVAL and outs[2] is None
    for i in (0, 1, 3, 4):
        assert status[i] == 0
        want, _ = oracle.oracle_la(mats[i])
        check_same(outs[i], want)


def test_gpu_plan_reruns_identically():
    m = synth.staircase(800, 200, 800, 65521, seed=9)
    want, _ = oracle.oracle_la(m)
    plan = la.Plan(m)
    for _ in range(3):
        plan.run()
        check_same(plan.result(), want)
    st = plan.stats()
    assert st["rank"] == want.np and st["rows_reduced"] == 200
    assert st["ms_total"] > 0 and st["kernel_launches"] > 0
    plan.close()


def test_gpu_interreduce_random():
    rng = np.random.default_rng(5)
    for p in (101, 65521, 2147483647):
        leads = np.sort(rng.choice(300, size=120, replace=False))
        ptr, cols, vals = [0], [], []
        for l in leads:
            k = min(15, 299 - l)
            tail = np.sort(rng.choice(np.arange(l + 1, 300), size=k, replace=False)) if k else []
            cols += [int(l)] + list(map(int, tail))
            vals += [1] + rng.integers(1, p, size=len(tail)).tolist()
            ptr.append(len(cols))
        perm = rng.permutation(len(leads))  # any row order
        rows = ReducedRows(np.array(ptr), np.array(cols), np.array(vals))
        sel = [np.arange(rows.row_ptr[i], rows.row_ptr[i + 1]) for i in perm]
        lens = np.array([len(s) for s in sel])
        rows_p = ReducedRows(np.concatenate([[0], np.cumsum(lens)]),
                             rows.cols[np.concatenate(sel)], rows.vals[np.concatenate(sel)])
        want, _ = oracle.oracle_interreduce(p, 300, rows)
        check_same(la.interreduce_matrix_rows(p, 300, rows_p), want)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("case", f4_cases(), ids=[c["name"] for c in f4_cases()])
def test_f4_with_gpu_linear_algebra_matches_golden(case):
    """gb's own F4 (host code of the reference build) with both linear-algebra
    call sites pointed at libgbgpu.so reproduces the golden basis."""
    la_fn = la.function_address("gbgpu_linear_algebra")
    ir_fn = la.function_address("gbgpu_interreduce_matrix_rows")
    lens, cfs, exps = oracle.ref_f4(case, la_fn=la_fn, ir_fn=ir_fn)
    exp = case["expected"]
    assert lens.shape[0] == exp["bld"]
    assert int(lens.sum()) == exp["nterms"]
    assert lens.tolist() == exp["tlen"]
    assert cfs.tolist() == exp["tcf"]
    assert exps.tolist() == exp["texp"]


@pytest.mark.skipif(not oracle.gb_gpu_available(), reason="integration build absent")
@pytest.mark.parametrize("case", f4_cases(), ids=[c["name"] for c in f4_cases()])
def test_integration_recipe_build_matches_golden(case):
    """gb compiled with the two-macro drop-in recipe (two -D macros, no source
    edit, linked against libgbgpu.so) reproduces every golden basis."""
    lens, cfs, exps = oracle.gb_gpu_f4(case)
    exp = case["expected"]
    assert lens.tolist() == exp["tlen"]
    assert cfs.tolist() == exp["tcf"]
    assert exps.tolist() == exp["texp"]


def test_plan_result_into_caller_buffers():
    m = synth.staircase(600, 150, 600, 32003, seed=4)
    want, _ = oracle.oracle_la(m)
    lib = _lib.load()
    plan = la.Plan(m)
    plan.run()
    npv, nnz = C.c_int32(), C.c_int64()
    rc = lib.gbgpu_plan_result_into(plan._h, None, None, None, 0, 0, C.byref(npv), C.byref(nnz))
    assert rc == _lib.GBGPU_ERANGE and npv.value == want.np and nnz.value == want.nnz
    rp = np.zeros(npv.value + 1, dtype=np.int64)
    cols = np.zeros(nnz.value, dtype=np.int32)
    vals = np.zeros(nnz.value, dtype=np.int32)
    _lib.check(lib.gbgpu_plan_result_into(plan._h, rp.ctypes.data, cols.ctypes.data,
                                          vals.ctypes.data, rp.shape[0], cols.shape[0],
                                          C.byref(npv), C.byref(nnz)))
    check_same(ReducedRows(rp, cols, vals), want)
    plan.close()


@pytest.mark.parametrize("p,vb", [(251, 1), (32003, 2), (65521, 2)])
@pytest.mark.parametrize("form", [_lib.FORM_PLAIN, _lib.FORM_TENSOR])
def test_narrow_values_in_and_out(form, p, vb):
    """Values at the reference's coefficient width (cf_8 / cf_16) on the way in
    (gbgpu_csr.val_bytes) and out (gbgpu_plan_result_into_v): same answer as
    the oracle."""
    m = synth.staircase(700, 180, 650, p, seed=9)
    want, _ = oracle.oracle_la(m)
    lib = _lib.load()
    vdt = np.uint8 if vb == 1 else np.uint16
    vals_in = np.ascontiguousarray(m.vals.astype(vdt))
    csr = _lib.Csr(m.p, m.laopt, m.nr, m.ncl, m.ncr, m.row_ptr.ctypes.data, m.cols.ctypes.data,
                   vals_in.ctypes.data, vb)
    opt = _lib.Options(form, 0, 1, 0, None)
    h = C.c_void_p()
    _lib.check(lib.gbgpu_plan_create(C.byref(csr), C.byref(opt), C.byref(h)))
    try:
        _lib.check(lib.gbgpu_plan_run(h))
        npv, nnz = C.c_int32(), C.c_int64()
        rc = lib.gbgpu_plan_result_into_v(h, None, None, None, vb, 0, 0, C.byref(npv),
                                          C.byref(nnz))
        assert rc == _lib.GBGPU_ERANGE and npv.value == want.np and nnz.value == want.nnz
        rp = np.zeros(npv.value + 1, dtype=np.int64)
        cols = np.zeros(max(nnz.value, 1), dtype=np.int32)
        vals = np.zeros(max(nnz.value, 1), dtype=vdt)
        _lib.check(lib.gbgpu_plan_result_into_v(h, rp.ctypes.data, cols.ctypes.data,
                                                vals.ctypes.data, vb, rp.shape[0], cols.shape[0],
                                                C.byref(npv), C.byref(nnz)))
        check_same(ReducedRows(rp, cols[:nnz.value], vals[:nnz.value].astype(np.int32)), want)
        # a width too narrow for the prime is rejected
        if p > 255:
            rc = lib.gbgpu_plan_result_into_v(h, rp.ctypes.data, cols.ctypes.data,
                                              vals.ctypes.data, 1, rp.shape[0], cols.shape[0],
                                              C.byref(npv), C.byref(nnz))
            assert rc == _lib.GBGPU_EINVAL
    finally:
        lib.gbgpu_plan_destroy(h)
    bad = _lib.Csr(m.p, m.laopt, m.nr, m.ncl, m.ncr, m.row_ptr.ctypes.data, m.cols.ctypes.data,
                   vals_in.ctypes.data, 3)
    assert lib.gbgpu_plan_create(C.byref(bad), C.byref(opt), C.byref(h)) == _lib.GBGPU_EINVAL


@pytest.mark.parametrize("p,vb", [(65521, 2), (2147483647, 4)])
def test_run_into_streams_the_answer(p, vb):
    """gbgpu_plan_run_into_v: the answer copied block by block during the
    back substitution equals the oracle's; too-small arrays give ERANGE with the
    sizes; after a streamed run the result calls refuse until the next run."""
    m = synth.staircase(1500, 700, 1400, p, seed=13)
    want, _ = oracle.oracle_la(m)
    lib = _lib.load()
    vdt = np.uint16 if vb == 2 else np.int32
    plan = la.Plan(m, form=_lib.FORM_TENSOR)
    npv, nnz = C.c_int32(), C.c_int64()
    rc = lib.gbgpu_plan_run_into_v(plan._h, None, None, None, vb, 0, 0, C.byref(npv), C.byref(nnz))
    assert rc == _lib.GBGPU_ERANGE and npv.value == want.np and nnz.value == want.nnz
    rp = np.zeros(npv.value + 1, dtype=np.int64)
    cols = np.zeros(nnz.value, dtype=np.int32)
    vals = np.zeros(nnz.value, dtype=vdt)
    small = np.zeros(4, dtype=np.int32)
    rc = lib.gbgpu_plan_run_into_v(plan._h, rp.ctypes.data, small.ctypes.data, small.ctypes.data,
                                   vb, rp.shape[0], 1, C.byref(npv), C.byref(nnz))
    assert rc == _lib.GBGPU_ERANGE and nnz.value == want.nnz
    for _ in range(2):
        _lib.check(lib.gbgpu_plan_run_into_v(plan._h, rp.ctypes.data, cols.ctypes.data,
                                             vals.ctypes.data, vb, rp.shape[0], cols.shape[0],
                                             C.byref(npv), C.byref(nnz)))
        check_same(ReducedRows(rp, cols, vals.astype(np.int64).astype(np.int32)), want)
    with pytest.raises(_lib.GbgpuError):
        plan.result()
    plan.run()
    check_same(plan.result(), want)
    plan.close()
