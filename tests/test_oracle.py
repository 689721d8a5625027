"""CPU tests: the oracle pinned against the reference's golden data.

* every matrix captured from the reference's own F4 golden programs
  (tests/golden/mats, with the reference's answer) is answered identically
  by the oracle, for la options 1 and 2;
* the known-answer test of test/normalize_row.c;
* the reference's F4 golden bases (tests/golden/f4) are reproduced by the
  reference build, and the oracle agrees with the reference build on seeded
  synthetic matrices (when oracle/_ref was built here).
"""
import os

import numpy as np
import pytest

import oracle
from gb_b200 import synth
from gb_b200.matrix import MacaulayMatrix
from tests.helpers import all_captures, as_rows, f4_cases, kat_normalize

CAPTURES = all_captures()


def test_captures_present():
    assert len(CAPTURES) > 200
    kinds = {c.kind for _, _, c in CAPTURES}
    assert kinds == {0, 1}
    primes = {c.mat.p for _, _, c in CAPTURES}
    assert {101, 127, 32003, 65521, 2147483647} <= primes


@pytest.mark.parametrize("name,k,cap", CAPTURES, ids=[f"{n}-{k}" for n, k, _ in CAPTURES])
def test_oracle_matches_reference_capture(name, k, cap):
    if cap.kind == 0:
        cap.mat.validate()
        for laopt in (1, 2):
            got, _ = oracle.oracle_la(cap.mat, laopt)
            assert got.equals(cap.answer), got.first_difference(cap.answer)
    else:
        got, _ = oracle.oracle_interreduce(cap.mat.p, cap.mat.nc, as_rows(cap.mat))
        assert got.equals(cap.answer), got.first_difference(cap.answer)


def test_normalize_row_known_answer():
    kat = kat_normalize()
    row = oracle.oracle_normalize(np.array(kat["row"]), kat["p"])
    for idx, want in kat["checks"]:
        assert row[idx] == want
    assert row[0] == 1


def test_inverse():
    lib = oracle._load_oracle()
    for p in (101, 32003, 65521, 2147483647):
        for a in (1, 2, 3, p - 1, p // 2):
            inv = lib.oracle_inverse(a, p)
            assert (a * inv) % p == 1


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("case", f4_cases(), ids=[c["name"] for c in f4_cases()])
def test_reference_build_reproduces_golden_basis(case):
    if case["name"] == "cyclic_7":
        pytest.skip("cyclic_7 takes tens of seconds on one core")
    lens, cfs, exps = oracle.ref_f4(case)
    exp = case["expected"]
    assert lens.shape[0] == exp["bld"]
    assert int(lens.sum()) == exp["nterms"]
    if "tlen" in exp:
        assert lens.tolist() == exp["tlen"]
    if "tcf" in exp:
        assert cfs.tolist() == exp["tcf"]
    if "texp" in exp:
        assert exps.tolist() == exp["texp"]


PRIMES = [2, 3, 101, 127, 251, 32003, 65521, 131071, 2147483647]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("p", PRIMES)
@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_matches_reference_build_synthetic(p, seed):
    m = synth.random_macaulay(25, 30, 35, p, density=0.1, seed=seed, dup_rows=2,
                              right_only_frac=0.3)
    m.validate()
    # 42/43/44 are Monte Carlo in the reference (random combinations drawn
    # with rand() % p, src/la_ff_16.c:449-451): a block combination misses
    # rank with probability about 1/p and the reference then returns other
    # rows, so they are compared only where p is large (one thread keeps the
    # rand() stream deterministic)
    for laopt in ((1, 2, 42, 43, 44) if p > 65000 else (1, 2)):
        want, _ = oracle.ref_la(m, laopt, nthreads=1 if laopt > 2 else 2)
        got, _ = oracle.oracle_la(m, laopt)
        assert got.equals(want), (laopt, got.first_difference(want))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_oracle_matches_reference_build_staircase():
    m = synth.staircase(600, 150, 600, 65521, seed=5)
    m.validate()
    want, _ = oracle.ref_la(m, 1, nthreads=4)
    got, _ = oracle.oracle_la(m, 2)
    assert got.equals(want), got.first_difference(want)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_oracle_interreduce_matches_reference_build():
    rng = np.random.default_rng(3)
    for p in (101, 65521, 2147483647):
        # echelon rows with distinct leads over 60 columns
        leads = np.sort(rng.choice(60, size=25, replace=False))
        ptr, cols, vals = [0], [], []
        for l in leads:
            tail = np.sort(rng.choice(np.arange(l + 1, 60), size=min(8, 59 - l), replace=False)) \
                if l < 59 else np.zeros(0, int)
            cols += [int(l)] + tail.tolist()
            vals += [1] + rng.integers(1, p, size=tail.shape[0]).tolist()
            ptr.append(len(cols))
        from gb_b200.matrix import ReducedRows
        rows = ReducedRows(np.array(ptr), np.array(cols), np.array(vals))
        want, _ = oracle.ref_interreduce(p, 60, rows)
        got, _ = oracle.oracle_interreduce(p, 60, rows)
        assert got.equals(want), got.first_difference(want)


def test_oracle_rejects_contract_violations():
    m = synth.random_macaulay(6, 4, 8, 101, seed=1)
    bad = MacaulayMatrix(m.p, m.ncl, m.ncr, m.row_ptr, m.cols, m.vals.copy())
    bad.vals[0] = 2  # rows must be monic
    with pytest.raises(ValueError):
        bad.validate()
    with pytest.raises(ValueError):
        oracle.oracle_la(bad, 1)
    nopiv = MacaulayMatrix(m.p, m.ncl + 1, m.ncr - 1, m.row_ptr, m.cols, m.vals)
    with pytest.raises(ValueError):
        nopiv.validate()
    with pytest.raises(ValueError):
        oracle.oracle_la(nopiv, 1)


def _rref_python(D, p):
    """Gauss-Jordan over GF(p) in plain Python (small blocks only)."""
    R = [list(map(int, row)) for row in D]
    piv, r = [], 0
    for c in range(len(R[0]) if R else 0):
        k = next((i for i in range(r, len(R)) if R[i][c] % p), None)
        if k is None:
            continue
        R[r], R[k] = R[k], R[r]
        inv = pow(R[r][c], p - 2, p)
        R[r] = [v * inv % p for v in R[r]]
        for i in range(len(R)):
            if i != r and R[i][c]:
                f = R[i][c]
                R[i] = [(a - f * b) % p for a, b in zip(R[i], R[r])]
        piv.append(c)
        r += 1
    return np.array(R, dtype=np.int64), r, piv


@pytest.mark.parametrize("p", [101, 65521, 2147483647])
def test_dense_block_embedding_yields_the_rref(p):
    """The Macaulay embedding of a dense block (used to run the reference's dense
    echelon on D blocks) has the block's RREF as its answer, in the oracle and
    in the reference build."""
    from gb_b200 import synth
    from helpers import dense_rref_rows
    D = synth.dense_lowrank(24, 30, 17, p, seed=4)
    R, rank, piv = _rref_python(D, p)
    want = dense_rref_rows(R, rank, piv, 24)
    m = synth.dense_block_macaulay(D, p)
    got, _ = oracle.oracle_la(m)
    assert rank == 17 and got.equals(want), got.first_difference(want)
    if oracle.ref_available():
        ref, _ = oracle.ref_la(m, 1, nthreads=2)
        assert ref.equals(want)


def test_f4_compare_harness_self_check_and_budget(tmp_path):
    """The round-by-round comparison harness (oracle/f4_compare.py, the
    reference hook's compare mode): comparing the reference with itself logs
    every la call as equal, and a budget stops the run after the call that
    exceeds it."""
    import subprocess
    import sys
    from oracle.f4_compare import parse_log
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    args = [sys.executable, "-m", "oracle.f4_compare", "--nvars", "4", "--ngens", "4",
            "--maxdeg", "3", "--p", "65521", "--la-option", "2", "--seed", "3",
            "--impl", "reference", "--threads", "2"]
    full = tmp_path / "full.log"
    subprocess.run(args + ["--budget", "1000", "--log", str(full)], check=True, cwd=repo,
                   timeout=300)
    res = parse_log(str(full))
    assert res["end"] == "done" and len(res["calls"]) >= 5
    assert all(c["equal"] == 1 and c["np"] == c["ref_np"] for c in res["calls"])
    cut = tmp_path / "cut.log"
    subprocess.run(args + ["--budget", "1e-9", "--log", str(cut)], check=True, cwd=repo,
                   timeout=300)
    res = parse_log(str(cut))
    assert len(res["calls"]) == 1 and res["end"].startswith("stop budget")


@pytest.mark.parametrize("mo", [0, 1])
def test_reference_conversion_matches_restated_order(mo):
    """The reference's convert_hashes_to_columns + sort_matrix_rows (through
    the test build) orders columns as the restated comparator of
    synth.column_order_key says and rows by (lead column, length); this pins
    the order the device conversion reproduces."""
    from gb_b200 import synth
    r = synth.f4_round(5, 6, 300, 200, 80, 20, seed=mo + 1)
    hcm, ncl, order, cols, _ = oracle.ref_convert(r["nv"], r["exps"], r["deg"], r["idx"], mo,
                                                  r["row_ptr"], r["hashes"])
    keys = synth.column_order_key(r["exps"], r["deg"], r["idx"], mo)
    want = [h + 1 for h in sorted(range(len(keys)), key=lambda h: keys[h])]
    assert hcm.tolist() == want and ncl == int((r["idx"] == 2).sum())
    col_of = np.empty(len(keys) + 1, dtype=np.int64)
    col_of[hcm] = np.arange(len(keys))
    ptr = r["row_ptr"]
    lead = col_of[r["hashes"][ptr[:-1]]]
    lens = np.diff(ptr)
    got_keys = [(int(lead[i]), int(lens[i])) for i in order]
    assert got_keys == sorted(got_keys) and sorted(order.tolist()) == list(range(len(lens)))
    off = 0
    for i in order:
        seg = r["hashes"][ptr[i]:ptr[i + 1]]
        assert cols[off:off + seg.shape[0]].tolist() == col_of[seg].tolist()
        off += seg.shape[0]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_basis_bench_harness_inserts_each_answer_column_once():
    """The basis-conversion harness (reference functions only): the fresh
    basis hash table ends with one element per distinct column of the answer
    (src/hash.c:604-669 inserts a monomial at its first entry and finds it
    afterwards), and two runs give the same digests."""
    from gb_b200 import synth
    m = synth.staircase(300, 100, 250, 65521, seed=4)
    exps = synth.distinct_monomials(m.ncl + m.ncr, 6, seed=2)
    a = oracle.basis_bench(m, exps)
    b = oracle.basis_bench(m, exps)
    want, _ = oracle.ref_la(m)
    assert a["np"] == want.np
    assert a["eld"] == 1 + len(np.unique(want.cols))
    assert a == {**b, "seconds": a["seconds"]}
