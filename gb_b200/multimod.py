"""Multi-modular reduction of an integer Macaulay matrix: the linear-algebra
step over the rationals, computed as many GF(p) reductions on the GPU and
combined on the host.

The reference has no such driver: its rational path (src/la_qq.c) works on
GMP numbers and is outside the GPU build.  What it shares with the modular
path is the answer: for a matrix M = [A|B ; C|D] with the known pivots A|B,
the new pivots are the reduced row echelon form of

    rowspace(M) over Q  intersected with  {x : x vanishes on the left block},

restricted to the right block, rows monic and in descending lead order --
the same rows `linear_algebra` returns over GF(p) (src/la_ff_32.c:1804-1851
and twins), now with rational entries.  For all but finitely many primes
("lucky" primes) the answer modulo p is the image of the rational answer,
with the same pivot columns.  So:

1. the integer rows are mapped to GF(p) for a batch of primes (the largest
   primes below 2^31) and normalised to lead 1 there (a row multiple, which
   changes no row space); a prime that divides a lead coefficient is
   skipped;
2. the images are reduced in one `gbgpu_reduce_batch` call on the GPU;
3. among the answers, the pivot pattern of a lucky prime is the one of
   largest rank and, at equal rank, the lexicographically smallest pivot
   columns (a prime can only lose rank or push pivots right); answers with
   another pattern are dropped;
4. the residues of every entry are combined by the Chinese remainder theorem,
   one prime at a time (x <- x + M ((r - x) M^-1 mod p)), and lifted to
   fractions a/b by rational reconstruction (half-extended Euclid,
   |a|, b <= sqrt(M/2) for the product M of the primes used);
5. the lifted answer is checked against the answer of one more prime that
   took no part in the lift; on a mismatch more primes are added.

Step 5 is the usual probabilistic certificate of multi-modular algorithms:
a wrong lift survives only if the extra prime divides the difference of
two bounded numbers.
"""
from __future__ import annotations

import dataclasses
import os
from fractions import Fraction
from math import gcd, isqrt
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

from .matrix import MacaulayMatrix, ReducedRows


@dataclasses.dataclass
class IntegerMacaulay:
    """A Macaulay matrix with integer coefficients (CSR, 0-based columns,
    leads first), in the layout of :class:`MacaulayMatrix` but with
    coefficients of any size (``vals`` may hold Python integers)."""

    ncl: int
    ncr: int
    row_ptr: np.ndarray  # int64 [nr + 1]
    cols: np.ndarray  # int32 [nnz]
    vals: np.ndarray  # int64 or object [nnz], nonzero

    @property
    def nr(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @staticmethod
    def from_matrix(m: MacaulayMatrix, vals: Optional[np.ndarray] = None) -> "IntegerMacaulay":
        return IntegerMacaulay(m.ncl, m.ncr, np.asarray(m.row_ptr, dtype=np.int64),
                               np.asarray(m.cols, dtype=np.int32),
                               np.asarray(m.vals if vals is None else vals))


@dataclasses.dataclass
class RationalRows:
    """The answer over Q: ``np`` rows in CSR form (columns as in
    :class:`ReducedRows`), entry k = num[k] / den[k] with den[k] > 0.  The
    entries of a row share denominators where they can, so a fraction need
    not be in lowest terms (``fractions()`` reduces them).  Leads are 1."""

    row_ptr: np.ndarray  # int64 [np + 1]
    cols: np.ndarray  # int32 [nnz]
    num: np.ndarray  # object [nnz]
    den: np.ndarray  # object [nnz]
    primes_used: int = 0

    @property
    def np(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    def fractions(self) -> List[List[Tuple[int, Fraction]]]:
        out = []
        for i in range(self.np):
            a, b = int(self.row_ptr[i]), int(self.row_ptr[i + 1])
            out.append([(int(self.cols[k]), Fraction(int(self.num[k]), int(self.den[k])))
                        for k in range(a, b)])
        return out

    def image(self, p: int) -> Optional[ReducedRows]:
        """These rows modulo p (None if p divides a denominator)."""
        den = np.array([int(d) % p for d in self.den], dtype=np.int64)
        if np.any(den == 0):
            return None
        num = np.array([int(a) % p for a in self.num], dtype=np.int64)
        inv = np.array([pow(int(d), p - 2, p) for d in den], dtype=np.int64)
        vals = (num * inv) % p
        keep = vals != 0
        counts = np.add.reduceat(keep.astype(np.int64), self.row_ptr[:-1]) if self.np and \
            self.row_ptr[-1] else np.zeros(self.np, dtype=np.int64)
        counts[np.diff(self.row_ptr) == 0] = 0
        ptr = np.zeros(self.np + 1, dtype=np.int64)
        np.cumsum(counts, out=ptr[1:])
        return ReducedRows(ptr, self.cols[keep], vals[keep].astype(np.int32))


def primes_below_2_31() -> Iterable[int]:
    """The primes below 2^31 in decreasing order (Miller-Rabin, exact for
    32-bit integers)."""
    n = (1 << 31) - 1
    while n > 2:
        if _is_prime(n):
            yield n
        n -= 2


def _is_prime(n: int) -> bool:
    if n < 2:
        return False
    for q in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % q == 0:
            return n == q
    d, r = n - 1, 0
    while d % 2 == 0:
        d //= 2
        r += 1
    for a in (2, 3, 5, 7):  # exact below 3.2e9
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(r - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def image(mat: IntegerMacaulay, p: int) -> Optional[MacaulayMatrix]:
    """The matrix over GF(p): coefficients mod p, every row scaled to lead 1,
    entries that vanish mod p dropped.  None when p divides a lead
    coefficient (the row's lead would move)."""
    vals = np.array([int(v) % p for v in mat.vals], dtype=np.int64) \
        if mat.vals.dtype == object else np.mod(mat.vals.astype(np.int64), p)
    nr = mat.nr
    if nr == 0:
        return MacaulayMatrix(p, mat.ncl, mat.ncr, mat.row_ptr, mat.cols, vals.astype(np.int32))
    lead_pos = mat.row_ptr[:-1]
    leads = vals[lead_pos]
    if np.any(leads == 0):
        return None
    inv = np.array([pow(int(x), p - 2, p) for x in leads], dtype=np.int64)
    lens = np.diff(mat.row_ptr)
    vals = (vals * np.repeat(inv, lens)) % p
    keep = vals != 0
    counts = np.add.reduceat(keep.astype(np.int64), lead_pos)
    ptr = np.zeros(nr + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    return MacaulayMatrix(p, mat.ncl, mat.ncr, ptr, mat.cols[keep], vals[keep].astype(np.int32))


def _pattern(rows: ReducedRows) -> Tuple[int, ...]:
    """Pivot columns of an answer, ascending."""
    leads = rows.cols[rows.row_ptr[:-1]] if rows.np else np.zeros(0, dtype=np.int32)
    return tuple(sorted(int(c) for c in leads))


def lucky_pattern(answers: Sequence[ReducedRows]) -> Tuple[int, ...]:
    """The pivot pattern of a lucky prime among the answers: the largest
    rank, then the lexicographically smallest pivot columns."""
    pats = [_pattern(r) for r in answers]
    return min(pats, key=lambda t: (-len(t), t))


def _dense(rows: ReducedRows, order: Sequence[int], support: np.ndarray) -> np.ndarray:
    """Answer rows as a dense array over the sorted column list ``support``
    (which holds every column of the answer), rows in the order of their
    pivot columns ``order``."""
    out = np.zeros((len(order), support.shape[0]), dtype=np.int64)
    if rows.np == 0:
        return out
    leads = rows.cols[rows.row_ptr[:-1]].astype(np.int64)
    order_arr = np.asarray(order, dtype=np.int64)
    # position of every answer row in `order` (descending leads)
    pos = np.searchsorted(-order_arr, -leads)
    nnz = rows.nnz
    row_of_entry = np.repeat(pos, np.diff(rows.row_ptr))
    out[row_of_entry, np.searchsorted(support, rows.cols[:nnz])] = rows.vals[:nnz]
    return out


def _ratrecon(x: int, m: int, bound: int) -> Optional[Tuple[int, int]]:
    """a/b with a = b x mod m, |a| <= bound, 0 < b <= bound (None if none)."""
    r0, r1 = m, x % m
    s0, s1 = 0, 1
    while r1 > bound:
        q = r0 // r1
        r0, r1 = r1, r0 - q * r1
        s0, s1 = s1, s0 - q * s1
    if s1 == 0 or abs(s1) > bound:
        return None
    a, b = (r1, s1) if s1 > 0 else (-r1, -s1)
    if gcd(a, b) != 1:
        return None
    return a, b


_lift = None


def _lift_lib():
    """libgblift.so (built with the package; compiled here if missing)."""
    global _lift
    if _lift is None:
        import ctypes as C
        from . import build
        if not os.path.exists(build.LIFT_LIB):
            build.build_lift()
        lib = C.CDLL(build.LIFT_LIB)
        lib.gblift_crt_add.argtypes = [C.c_int64, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                       C.c_void_p, C.c_uint32, C.c_uint32]
        lib.gblift_crt_add.restype = C.c_int
        _lift = lib
    return _lift


class Lifter:
    """Incremental Chinese remaindering of the answers of one pivot pattern:
    the residues of every entry (dense over the union of the answers'
    columns) as one integer in [0, M), M the product of the primes added,
    held as little-endian 64-bit limbs and updated by libgblift.so
    (x <- x + M ((r - x) M^-1 mod p))."""

    def __init__(self, answer: ReducedRows, p: int):
        self.pattern = _pattern(answer)
        self.order = sorted(self.pattern, reverse=True)  # answer rows: descending lead
        self.support = np.zeros(0, dtype=np.int64)  # sorted columns of the entries
        self.nl = 4  # limbs per entry
        self.x = np.zeros((len(self.order), 0, self.nl), dtype=np.uint64)
        self.m = 1
        self.primes: List[int] = []
        self.hard: Optional[Tuple[int, int]] = None  # the entry that failed to lift last
        self.add(answer, p)

    def _grow(self, answer: ReducedRows) -> None:
        cols = np.unique(answer.cols[: answer.nnz].astype(np.int64))
        new = np.setdiff1d(cols, self.support, assume_unique=True)
        if new.shape[0] == 0:
            return
        # a column no earlier answer had is 0 modulo every earlier prime
        support = np.union1d(self.support, new)
        keep = np.searchsorted(support, self.support)
        x = np.zeros((len(self.order), support.shape[0], self.nl), dtype=np.uint64)
        x[:, keep, :] = self.x
        self.support, self.x = support, x

    def add(self, answer: ReducedRows, p: int) -> None:
        """x <- the integer in [0, M p) that is x mod M and the answer mod p."""
        self._grow(answer)
        r = np.ascontiguousarray(_dense(answer, self.order, self.support), dtype=np.int64)
        m_len = max(1, (self.m.bit_length() + 63) // 64)
        if m_len + 1 > self.nl:  # room for M p
            x = np.zeros(self.x.shape[:2] + (2 * self.nl,), dtype=np.uint64)
            x[:, :, : self.nl] = self.x
            self.x, self.nl = x, 2 * self.nl
        mlimbs = np.frombuffer(self.m.to_bytes(8 * m_len, "little"), dtype=np.uint64).copy()
        n = int(r.size)
        if n:
            rc = _lift_lib().gblift_crt_add(n, self.nl, self.x.ctypes.data, mlimbs.ctypes.data,
                                            m_len, r.ctypes.data, p,
                                            pow(self.m % p, p - 2, p))
            if rc != 0:
                raise RuntimeError("gblift_crt_add rejected its arguments")
        self.m *= p
        self.primes.append(p)

    def _row_values(self, r: int) -> List[int]:
        raw = self.x[r].tobytes()
        w = 8 * self.nl
        return [int.from_bytes(raw[k * w:(k + 1) * w], "little")
                for k in range(self.support.shape[0])]

    def lift(self) -> Optional[RationalRows]:
        """Rational reconstruction of every entry, or None when some entry has
        none yet (more primes needed).

        Entries of an echelon form mostly share their denominators, so every
        entry first tries the denominators found so far (their lcm while it
        stays within the bound): y = x d mod M in the symmetric range with
        |y| <= sqrt(M/2) makes y/d the reconstruction (unique within those
        bounds; kept over d, not reduced), at the cost of one multiplication;
        only the others run the extended Euclid.  The entry that failed last time is tried first, then the
        rows from the last."""
        m = self.m
        bound = _isqrt((m - 1) // 2)
        half = m // 2
        nrows, ncols = len(self.order), int(self.support.shape[0])
        if self.hard is not None and self.hard[0] < nrows and self.hard[1] < ncols:
            v = int.from_bytes(self.x[self.hard].tobytes(), "little")
            if v and _ratrecon(v, m, bound) is None:
                return None
        # the last rows (smallest leads) carry the largest fractions: they go
        # first, so that a lift that needs more primes stops early
        per_row: List[Tuple[List[int], List[int], List[int]]] = [([], [], [])] * nrows
        d = 1
        for r in range(nrows - 1, -1, -1):
            xs = self._row_values(r)
            rc, rn, rd = [], [], []
            for k in range(ncols):
                v = xs[k]
                if v == 0:
                    continue
                y = v * d % m
                if y > half:
                    y -= m
                q = None
                if -bound <= y <= bound:
                    # y = d v (mod M) by construction, |y| and d within the
                    # bounds: the same number as the reconstruction of v,
                    # written over the shared denominator d
                    q = (y, d)
                if q is None:
                    q = _ratrecon(v, m, bound)
                    if q is None:
                        self.hard = (r, k)
                        return None
                    lcm = d // gcd(d, q[1]) * q[1]
                    d = lcm if lcm <= bound else q[1]
                rc.append(int(self.support[k]))
                rn.append(q[0])
                rd.append(q[1])
            per_row[r] = (rc, rn, rd)
        ptr = [0]
        cols, num, den = [], [], []
        for rc, rn, rd in per_row:
            cols += rc
            num += rn
            den += rd
            ptr.append(len(cols))
        return RationalRows(np.array(ptr, dtype=np.int64), np.array(cols, dtype=np.int32),
                            np.array(num, dtype=object), np.array(den, dtype=object),
                            primes_used=len(self.primes))


def combine(primes: Sequence[int], answers: Sequence[ReducedRows]) -> Optional[RationalRows]:
    """Lift answers of the same (lucky) pattern to Q.  Returns None when some
    entry has no rational reconstruction yet (more primes needed)."""
    lifter = Lifter(answers[0], primes[0])
    for p, a in zip(primes[1:], answers[1:]):
        lifter.add(a, p)
    return lifter.lift()


def _isqrt(n: int) -> int:
    return isqrt(n)


def reduce_over_q(mat: IntegerMacaulay, batch: int = 8, max_primes: int = 512,
                  device: int = 0, stats: Optional[dict] = None) -> RationalRows:
    """The linear-algebra step of an integer Macaulay matrix over Q: GF(p)
    images reduced on the GPU (`gbgpu_reduce_batch`, `batch` primes per
    call), combined on the host.  After every batch the residues collected
    so far (all but the newest prime of the lucky pattern) are lifted, and
    the lift is checked against that newest prime.  Raises RuntimeError when
    ``max_primes`` primes do not certify an answer.  With ``stats`` (a dict)
    the seconds spent in the gbgpu_reduce_batch calls, host CSR in and out
    ('batch_s'), in the images ('image_s'), in the lifts and checks
    ('lift_s'), the primes tried and the lift attempts are recorded there."""
    import time
    from . import la
    st = stats if stats is not None else {}
    for key in ("batch_s", "image_s", "lift_s"):
        st[key] = 0.0
    st["lifts"] = 0
    gen = primes_below_2_31()
    lifter: Optional[Lifter] = None
    held: Optional[Tuple[int, ReducedRows]] = None  # the check prime, not yet lifted
    tried = 0
    while tried < max_primes:
        ps, imgs = [], []
        t0 = time.perf_counter()
        while len(ps) < batch and tried < max_primes:
            p = next(gen)
            tried += 1
            m = image(mat, p)
            if m is not None:
                ps.append(p)
                imgs.append(m)
        st["primes_tried"] = tried
        t1 = time.perf_counter()
        st["image_s"] += t1 - t0
        if not imgs:
            continue
        answers, status = la.reduce_batch(imgs, device=device)
        t2 = time.perf_counter()
        st["batch_s"] += t2 - t1
        for p, a, code in zip(ps, answers, status):
            if code != 0 or a is None:
                raise RuntimeError(f"GF({p}) image failed with status {code}")
            pat = _pattern(a)
            best = held[1] if held is not None else None
            if best is not None and pat != _pattern(best):
                if (-len(pat), pat) < (-len(_pattern(best)), _pattern(best)):
                    lifter, held = None, None  # every earlier prime was unlucky
                else:
                    continue  # this prime is unlucky
            if held is not None:
                if lifter is None:
                    lifter = Lifter(held[1], held[0])
                else:
                    lifter.add(held[1], held[0])
            held = (p, a)
        if lifter is None or held is None:
            st["lift_s"] += time.perf_counter() - t2
            continue
        res = lifter.lift()
        st["lifts"] += 1
        ok = False
        if res is not None:
            img = res.image(held[0])
            ok = img is not None and img.equals(held[1])
        st["lift_s"] += time.perf_counter() - t2
        if ok:
            return res
    raise RuntimeError(f"no certified rational answer after {tried} primes")
