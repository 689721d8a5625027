"""GPU tests of the step before the linear algebra on the device:
convert_hashes_to_columns + sort_matrix_rows (src/convert.c:30-135,
src/order.c:98-131) through gbgpu_convert_hashes_to_columns_flat, against the
reference's own functions (the test build, oracle/_ref) on the same rounds:
the column map (hcm), the number of pivot columns and the rows' columns must
be equal, and the row order equal up to the order of rows that tie on
(lead column, length), which the reference's qsort leaves unspecified.  And
end to end: gb's F4 with the conversion, the row sort and the linear algebra
all on the GPU (oracle/ref/gb_gpu_full.c) reproduces every golden basis."""
import ctypes as C

import numpy as np
import pytest

import oracle
from gb_b200 import _lib, synth
from helpers import f4_cases

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")]


def device_convert(r, mo):
    lib = _lib.load()
    n, nr = r["exps"].shape[0], r["row_ptr"].shape[0] - 1
    nnz = int(r["row_ptr"][-1])
    hcm = np.zeros(max(n, 1), np.int32)
    order = np.zeros(max(nr, 1), np.int32)
    optr = np.zeros(nr + 1, np.int64)
    cols = np.zeros(max(nnz, 1), np.int32)
    ncl = C.c_int32()
    _lib.check(lib.gbgpu_convert_hashes_to_columns_flat(
        r["nv"], n, r["exps"].ctypes.data, r["deg"].ctypes.data, r["idx"].ctypes.data, mo, nr,
        r["row_ptr"].ctypes.data, r["hashes"].ctypes.data, hcm.ctypes.data, C.byref(ncl),
        order.ctypes.data, optr.ctypes.data, cols.ctypes.data, 0))
    return hcm[:n], ncl.value, order[:nr], optr, cols[:nnz]


def rows_by_key(order, cols, optr, row_ptr):
    """{(lead column, length): sorted list of the rows' column tuples}, the
    rows' keys in output order."""
    groups, keys = {}, []
    for k, i in enumerate(order):
        c = tuple(cols[optr[k]:optr[k + 1]].tolist()) if optr is not None else None
        keys.append((c[0], len(c)))
        groups.setdefault(keys[-1], []).append(c)
    return {k: sorted(v) for k, v in groups.items()}, keys


@pytest.mark.parametrize("mo", [0, 1])
@pytest.mark.parametrize("nv,maxdeg,n_cols,nr,n_piv,row_len", [
    (4, 5, 100, 60, 30, 10), (7, 6, 1500, 2500, 1200, 40), (12, 6, 15000, 12000, 6000, 60),
    (3, 40, 800, 900, 300, 25)])
def test_device_conversion_matches_reference(mo, nv, maxdeg, n_cols, nr, n_piv, row_len):
    r = synth.f4_round(nv, maxdeg, n_cols, nr, n_piv, row_len, seed=nv + mo)
    hcm, ncl, order, optr, cols = device_convert(r, mo)
    rh, rncl, rorder, rcols, _ = oracle.ref_convert(r["nv"], r["exps"], r["deg"], r["idx"], mo,
                                                    r["row_ptr"], r["hashes"])
    assert np.array_equal(hcm, rh) and ncl == rncl
    roptr = np.zeros(nr + 1, np.int64)
    np.cumsum(np.diff(r["row_ptr"])[rorder], out=roptr[1:])
    g_dev, k_dev = rows_by_key(order, cols, optr, r["row_ptr"])
    g_ref, k_ref = rows_by_key(rorder, rcols, roptr, r["row_ptr"])
    assert k_dev == k_ref and k_dev == sorted(k_dev)  # same (lead, length) sequence
    assert g_dev == g_ref  # same rows in every tie group
    # ties keep their input order on the device
    for a in range(nr - 1):
        if k_dev[a] == k_dev[a + 1]:
            assert order[a] < order[a + 1]


@pytest.mark.skipif(not oracle.gb_gpu_full_available(), reason="full GPU build absent")
@pytest.mark.parametrize("case", f4_cases(), ids=[c["name"] for c in f4_cases()])
def test_f4_with_conversion_on_gpu_matches_golden(case):
    lens, cfs, exps = oracle.gb_gpu_full_f4(case)
    exp = case["expected"]
    assert lens.tolist() == exp["tlen"]
    assert cfs.tolist() == exp["tcf"]
    assert exps.tolist() == exp["texp"]


def _first_entries_host(rr, ncl, ncr):
    first = np.full(ncr, -1, dtype=np.int64)
    cols = np.asarray(rr.cols, dtype=np.int64) - ncl
    seen = np.zeros(ncr, dtype=bool)
    for e, j in enumerate(cols.tolist()):
        if not seen[j]:
            seen[j] = True
            first[j] = e
    return first


@pytest.mark.gpu
@pytest.mark.parametrize("p,form", [(65521, _lib.FORM_TENSOR), (2147483647, _lib.FORM_AUTO),
                                    (32003, _lib.FORM_PLAIN)])
def test_plan_first_entry_and_column_map(p, form):
    """The device side of src/convert.c:137-280: the first entry of every
    right column in the answer and the rewrite of every entry through a
    column map, against the host answer."""
    from gb_b200 import la
    m = synth.staircase(900, 300, 700, p, seed=11)
    plan = la.Plan(m, form=form)
    plan.run()
    rr = plan.result()
    first = plan.first_entry()
    assert first.tolist() == _first_entries_host(rr, m.ncl, m.ncr).tolist()
    rng = np.random.default_rng(5)
    mapping = rng.permutation(m.ncr).astype(np.int32) + 7
    plan.map_columns(mapping)
    mapped = plan.result()
    assert np.array_equal(mapped.row_ptr, rr.row_ptr)
    assert np.array_equal(mapped.vals, rr.vals)
    want = mapping[np.asarray(rr.cols, dtype=np.int64) - m.ncl]
    assert np.array_equal(np.asarray(mapped.cols), want)
    # the mapped answer no longer counts from ncl: a second map or a first-
    # entry query is refused, and the answer stays as mapped
    with pytest.raises(_lib.GbgpuError):
        plan.map_columns(mapping)
    with pytest.raises(_lib.GbgpuError):
        plan.first_entry()
    assert np.array_equal(np.asarray(plan.result().cols), want)
    # a new run starts from ncl-based columns again
    plan.run()
    assert plan.first_entry().tolist() == first.tolist()
    plan.close()


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("p", [251, 32003, 65521, 2147483647])
def test_basis_conversion_matches_reference(p):
    """src/f4.c:306-311 on one matrix with a fresh basis: the reference's la
    and convert_sparse_matrix_rows_to_basis_elements against
    gbgpu_linear_algebra_keep + gbgpu_convert_sparse_matrix_rows_to_basis_
    elements -- the same new basis elements (table indices, monomials,
    coefficients), the same table size and the same hash-map layout."""
    from gb_b200 import la
    m = synth.staircase(1500, 500, 1200, p, seed=21)
    exps = synth.distinct_monomials(m.ncl + m.ncr, 7, seed=3)
    want = oracle.basis_bench(m, exps)
    got = oracle.basis_bench(
        m, exps, keep_fn=la.function_address("gbgpu_linear_algebra_keep"),
        convert_fn=la.function_address("gbgpu_convert_sparse_matrix_rows_to_basis_elements"))
    assert got["np"] == want["np"] > 0
    assert got["eld"] == want["eld"]
    assert got["digest"] == want["digest"]
    assert got["map_digest"] == want["map_digest"]
