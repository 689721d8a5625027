"""The multi-modular driver's host logic (no GPU): GF(p) images of integer
matrices, the lucky-pattern choice, CRT + rational reconstruction, and the
lifted answer against an exact rational elimination.  The per-prime answers
come from the oracle here; the GPU path is tested in test_gpu_multimod.py."""
from fractions import Fraction

import numpy as np

import oracle
from gb_b200 import multimod, synth
from gb_b200.matrix import ReducedRows
from tests.helpers import exact_answer, small_integer_matrix


def oracle_answers(mat, primes):
    ps, ans = [], []
    for p in primes:
        img = multimod.image(mat, p)
        if img is None:
            continue
        r, _ = oracle.oracle_la(img)
        ps.append(p)
        ans.append(r)
    return ps, ans


def test_image_is_monic_and_drops_vanishing_entries():
    mat = multimod.IntegerMacaulay(
        2, 2, np.array([0, 2, 5], dtype=np.int64), np.array([0, 2, 1, 2, 3], dtype=np.int32),
        np.array([3, 7, 5, 10, 11], dtype=np.int64))
    img = multimod.image(mat, 5)
    assert img is None  # 5 divides the lead of row 1
    img = multimod.image(mat, 7)  # row 0: 3, 7 -> 1, 0 (dropped)
    assert list(img.row_ptr) == [0, 1, 4] and list(img.vals[img.row_ptr[:-1]]) == [1, 1]
    assert list(img.cols) == [0, 1, 2, 3]
    # row 1 scaled by 5^-1 mod 7 = 3: 5, 10, 11 -> 1, 2, 5
    assert list(img.vals[1:]) == [1, 2, 5]


def test_ratrecon_and_crt_round_trip():
    from gb_b200.matrix import ReducedRows
    primes = list(synth.largest_primes_below(1 << 31, 4))
    fracs = [(3, 7), (-22, 9), (123456789, 987654), (-1, 2 ** 40 + 15)]
    # one answer row [1, f_0, f_1, ...] at columns 10, 11, ... per prime
    lifter = None
    for p in primes:
        vals = [1] + [a * pow(b, p - 2, p) % p for a, b in fracs]
        ans = ReducedRows(np.array([0, len(vals)]), np.arange(10, 10 + len(vals)),
                          np.array(vals))
        if lifter is None:
            lifter = multimod.Lifter(ans, p)
        else:
            lifter.add(ans, p)
    got = lifter.lift()
    assert got.fractions() == [[(10, Fraction(1))] +
                               [(11 + k, Fraction(a, b)) for k, (a, b) in enumerate(fracs)]]
    assert multimod._ratrecon(0, lifter.m, 10) == (0, 1)


def test_lift_matches_exact_rational_answer():
    mat = small_integer_matrix()
    want = exact_answer(mat)
    primes = list(synth.largest_primes_below(1 << 31, 40))
    ps, ans = oracle_answers(mat, primes)
    got = None
    for k in range(2, len(ps) + 1):
        got = multimod.combine(ps[:k], ans[:k])
        if got is not None and got.image(ps[-1]).equals(ans[-1]):
            break
    assert got is not None
    assert got.fractions() == want
    # every image of the lifted answer is the GF(p) answer
    for p, a in zip(ps, ans):
        assert got.image(p).equals(a)


def test_lucky_pattern_skips_a_rank_deficient_prime():
    p0 = 2147483647
    # known pivot [1 | 0 0]; C rows [1 | 1 0], [1 | 5 p0]: the Schur complement
    # [[1, 0], [5, p0]] has determinant p0 -- rank 2 over Q, 1 mod p0
    mat = multimod.IntegerMacaulay(
        1, 2, np.array([0, 1, 3, 6], dtype=np.int64),
        np.array([0, 0, 1, 0, 1, 2], dtype=np.int32),
        np.array([1, 1, 1, 1, 5, p0], dtype=np.int64))
    primes = [p0] + list(synth.largest_primes_below(p0, 3))
    ps, ans = oracle_answers(mat, primes)
    assert [len(multimod._pattern(a)) for a in ans] == [1, 2, 2, 2]
    pat = multimod.lucky_pattern(ans)
    assert pat == (1, 2)
    sel = [i for i, a in enumerate(ans) if multimod._pattern(a) == pat]
    got = multimod.combine([ps[i] for i in sel], [ans[i] for i in sel])
    assert got.fractions() == [[(2, Fraction(1))], [(1, Fraction(1))]]
    assert got.fractions() == exact_answer(mat)


def test_unreconstructible_residues_ask_for_more_primes():
    mat = small_integer_matrix(seed=2, bound=1 << 20)
    ps, ans = oracle_answers(mat, list(synth.largest_primes_below(1 << 31, 2)))
    # one 31-bit prime cannot hold the answer's fractions
    assert multimod.combine(ps[:1], ans[:1]) is None


def _oracle_batch(mats, form=0, device=0):
    out = [oracle.oracle_la(m)[0] for m in mats]
    return out, [0] * len(out)


def test_driver_loop_with_oracle_images(monkeypatch):
    """reduce_over_q's batching, pattern choice, incremental lift and check,
    with the GPU batch call replaced by the oracle (host logic only)."""
    from gb_b200 import la
    monkeypatch.setattr(la, "reduce_batch", _oracle_batch)
    mat = small_integer_matrix()
    got = multimod.reduce_over_q(mat, batch=5)
    assert got.fractions() == exact_answer(mat)
    p0 = 2147483647  # the first prime tried is rank deficient for this matrix
    mat = multimod.IntegerMacaulay(
        1, 2, np.array([0, 1, 3, 6], dtype=np.int64),
        np.array([0, 0, 1, 0, 1, 2], dtype=np.int32),
        np.array([1, 1, 1, 1, 5, p0], dtype=np.int64))
    for batch in (1, 2, 4):
        got = multimod.reduce_over_q(mat, batch=batch)
        assert got.fractions() == [[(2, Fraction(1))], [(1, Fraction(1))]]


def test_native_crt_matches_python_integers():
    """libgblift.so's x <- x + M ((r - x) M^-1 mod p) against Python integers,
    across limb boundaries and with residues at both ends of [0, p)."""
    rng = np.random.default_rng(5)
    primes = synth.largest_primes_below(1 << 31, 12)
    n = 257
    want = [0] * n
    lifter = None
    m = 1
    for k, p in enumerate(primes):
        r = rng.integers(0, p, size=n)
        r[:3] = [0, p - 1, 1]
        ans = ReducedRows(np.arange(n + 1), np.arange(10, 10 + n), r.astype(np.int32))
        # one answer row per entry keeps the pattern fixed: leads 10 .. 10 + n - 1
        if lifter is None:
            lifter = multimod.Lifter(ans, p)
        else:
            lifter.add(ans, p)
        want = [w + m * (((int(ri) - w) * pow(m, -1, p)) % p) for w, ri in zip(want, r)]
        m *= p
        # answer row i (lead 10 + i) is row n - 1 - i of the lift (descending
        # leads), its entry column i of the support
        got = [int.from_bytes(lifter.x[n - 1 - i, i].tobytes(), "little") for i in range(n)]
        assert got == want, f"after {k + 1} primes"
    assert lifter.m == m and lifter.nl * 64 >= m.bit_length() + 64


def test_native_crt_threads_over_many_entries():
    """gblift_crt_add on 20000 entries (split over host threads) equals the
    Python integer update, entry for entry."""
    rng = np.random.default_rng(9)
    lib = multimod._lift_lib()
    n, nl = 20000, 4
    x = np.zeros((n, nl), dtype=np.uint64)
    want = [0] * n
    m = 1
    for p in synth.largest_primes_below(1 << 31, 5):
        r = rng.integers(0, p, size=n).astype(np.int64)
        m_len = max(1, (m.bit_length() + 63) // 64)
        ml = np.frombuffer(m.to_bytes(8 * m_len, "little"), dtype=np.uint64).copy()
        assert lib.gblift_crt_add(n, nl, x.ctypes.data, ml.ctypes.data, m_len, r.ctypes.data,
                                  p, pow(m % p, p - 2, p)) == 0
        want = [w + m * (((int(ri) - w) * pow(m, -1, p)) % p) for w, ri in zip(want, r)]
        m *= p
    got = [int.from_bytes(x[i].tobytes(), "little") for i in range(n)]
    assert got == want
    assert lib.gblift_crt_add(n, 1, x.ctypes.data, ml.ctypes.data, 1, r.ctypes.data, 7, 1) == -1


def test_lifter_grows_its_columns_when_an_entry_vanishes_mod_p():
    """An entry that is 0 modulo the first prime (absent from that answer) and
    nonzero modulo the next ones is lifted from residue 0 at the first prime."""
    primes = synth.largest_primes_below(1 << 31, 6)
    frac = Fraction(primes[0] * 5, 7)  # vanishes modulo primes[0]
    lifter = None
    for p in primes:
        v = frac.numerator * pow(frac.denominator, p - 2, p) % p
        cols, vals = ([20, 21], [1, v]) if v else ([20], [1])
        ans = ReducedRows(np.array([0, len(cols)]), np.array(cols), np.array(vals))
        if lifter is None:
            lifter = multimod.Lifter(ans, p)
            assert list(lifter.support) == [20]
        else:
            lifter.add(ans, p)
    assert list(lifter.support) == [20, 21]
    assert lifter.lift().fractions() == [[(20, Fraction(1)), (21, frac)]]
