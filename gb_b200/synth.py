"""Seeded synthetic Macaulay matrices and dense blocks.

No public benchmark suite exists for this path: the reference ships input
systems without timings.  These generators stand in for the workloads,
with the shapes, sizes and value distributions the benchmark configurations
name.  Every generator is a pure function of its arguments and seed
(numpy PCG64).

* :func:`staircase` -- the standalone A|B/C|D matrix: ``nru = ncl`` known
  pivots (row i has lead i, coefficient 1), ``nrl`` rows to reduce with
  leads uniform in ``[0, ncl)``; each row holds a fraction U[dmin, dmax] of
  all columns, half in the left block inside a band right of its lead and
  half in the right block around column ``ncl + lead * ncr / ncl``
  (banded along the pivot staircase), coefficients uniform in [1, p-1],
  every row monic.  Rows are sorted by (lead, length) like
  ``sort_matrix_rows`` (src/order.c:98-131), with the known pivot first
  for its lead.
* :func:`random_macaulay` -- small irregular matrices for parity tests
  (sparse, with duplicated leads, empty-ish right blocks, rank deficiency).
* :func:`dense_lowrank` -- D = L * R mod p with L n x r, R r x n (rank <= r).
"""
from __future__ import annotations

import itertools

import numpy as np

from .matrix import MacaulayMatrix


def _band_sample(rng: np.random.Generator, lo: int, hi: int, k: int) -> np.ndarray:
    """k distinct integers from [lo, hi) (fewer if the range is short)."""
    n = hi - lo
    if n <= 0 or k <= 0:
        return np.zeros(0, dtype=np.int64)
    k = min(k, n)
    if k * 3 >= n:
        return lo + rng.permutation(n)[:k]
    out = np.unique(rng.integers(lo, hi, size=int(k * 1.3) + 8))
    while out.shape[0] < k:
        out = np.unique(np.concatenate([out, rng.integers(lo, hi, size=k)]))
    return rng.permutation(out)[:k]


def staircase(nru: int = 20000, nrl: int = 5000, ncr: int = 20000, p: int = 65521,
              dmin: float = 0.02, dmax: float = 0.05, band: float = 4.0,
              seed: int = 1, laopt: int = 1) -> MacaulayMatrix:
    """The banded A|B/C|D matrix described in the module docstring.

    ``band`` is the ratio of a band's width to the number of entries drawn
    in it (4 -> about a quarter of the band is filled)."""
    rng = np.random.default_rng(seed)
    ncl = nru
    nc = ncl + ncr
    leads = np.concatenate([np.arange(nru), rng.integers(0, ncl, size=nrl)])
    nnz = np.maximum(2, np.round(rng.uniform(dmin, dmax, size=nru + nrl) * nc)).astype(np.int64)
    rows_c, rows_v = [], []
    for i in range(nru + nrl):
        lead = int(leads[i])
        na = int(nnz[i] // 2)
        nb = int(nnz[i] - na)
        wa = max(1, int(band * na))
        a = _band_sample(rng, lead + 1, min(ncl, lead + 1 + wa), na - 1)
        center = ncl + (lead * ncr) // max(ncl, 1)
        wb = max(1, int(band * nb))
        b = _band_sample(rng, max(ncl, center - wb // 2), min(nc, center + wb - wb // 2), nb)
        c = np.concatenate([[lead], rng.permutation(np.concatenate([a, b]))])
        v = np.concatenate([[1], rng.integers(1, p, size=c.shape[0] - 1)])
        rows_c.append(c)
        rows_v.append(v)
    lens = np.array([r.shape[0] for r in rows_c], dtype=np.int64)
    is_lower = np.concatenate([np.zeros(nru, bool), np.ones(nrl, bool)])
    order = np.lexsort((lens, is_lower, leads))  # known pivot first per lead
    ptr = np.zeros(nru + nrl + 1, dtype=np.int64)
    np.cumsum(lens[order], out=ptr[1:])
    cols = np.concatenate([rows_c[i] for i in order]).astype(np.int32)
    vals = np.concatenate([rows_v[i] for i in order]).astype(np.int32)
    return MacaulayMatrix(p, ncl, ncr, ptr, cols, vals, laopt)


def integer_staircase(nru: int, nrl: int, ncr: int, bound: int = 1 << 20,
                      dmin: float = 0.02, dmax: float = 0.05, seed: int = 1) -> MacaulayMatrix:
    """The staircase structure with integer coefficients in [-bound, bound]
    without 0 (leads 1): one "system" whose images modulo many primes
    (``image_mod``) share their sparsity structure.  The returned matrix holds
    the integers in ``vals`` (int64) and ``p`` = 2 bound + 1."""
    m = staircase(nru, nrl, ncr, 2 * bound + 1, dmin, dmax, seed=seed)
    v = m.vals.astype(np.int64)
    ints = np.where(v > bound, v - (2 * bound + 1), v)  # [1, bound] U [-bound, -1]
    return MacaulayMatrix(m.p, m.ncl, m.ncr, m.row_ptr, m.cols, ints, m.laopt)


def image_mod(m: MacaulayMatrix, p: int) -> MacaulayMatrix:
    """The image of an integer matrix (``integer_staircase``) modulo a prime
    p > bound: every coefficient stays nonzero, leads stay 1."""
    vals = np.mod(np.asarray(m.vals, dtype=np.int64), p).astype(np.int32)
    return MacaulayMatrix(p, m.ncl, m.ncr, m.row_ptr, m.cols, vals, m.laopt)


def largest_primes_below(bound: int, count: int) -> list:
    """The `count` largest primes below `bound` (deterministic Miller-Rabin
    for 64-bit integers)."""
    def is_prime(n: int) -> bool:
        if n < 2:
            return False
        for q in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
            if n % q == 0:
                return n == q
        d, r = n - 1, 0
        while d % 2 == 0:
            d //= 2
            r += 1
        for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
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
    out, n = [], bound - 1
    while len(out) < count and n > 1:
        if is_prime(n):
            out.append(n)
        n -= 1
    return out


def random_macaulay(nru: int, nrl: int, ncr: int, p: int, density: float = 0.1,
                    seed: int = 0, laopt: int = 1, dup_rows: int = 0,
                    right_only_frac: float = 0.0) -> MacaulayMatrix:
    """Irregular matrix satisfying the mat_t contract.

    ``dup_rows`` lower rows are exact multiples-free copies of known pivots
    (they reduce to zero); ``right_only_frac`` of the lower rows have no
    left entries besides their lead."""
    rng = np.random.default_rng(seed)
    ncl = nru
    nc = ncl + ncr
    rows = []
    for i in range(nru):
        k = max(0, int(rng.binomial(nc - i - 1, density)))
        c = np.concatenate([[i], _band_sample(rng, i + 1, nc, k)])
        v = np.concatenate([[1], rng.integers(1, p, size=c.shape[0] - 1)])
        rows.append((i, 0, c, v))
    for j in range(nrl):
        lead = int(rng.integers(0, max(ncl, 1)))
        if j < dup_rows:
            c, v = rows[lead][2].copy(), rows[lead][3].copy()
        else:
            lo = ncl if rng.random() < right_only_frac else lead + 1
            k = max(0, int(rng.binomial(nc - lo, density)))
            c = np.concatenate([[lead], _band_sample(rng, lo, nc, k)])
            v = np.concatenate([[1], rng.integers(1, p, size=c.shape[0] - 1)])
        rows.append((lead, 1, c, v))
    rows.sort(key=lambda r: (r[0], r[1], r[2].shape[0]))
    lens = np.array([r[2].shape[0] for r in rows], dtype=np.int64)
    ptr = np.zeros(len(rows) + 1, dtype=np.int64)
    np.cumsum(lens, out=ptr[1:])
    cols = np.concatenate([r[2] for r in rows]).astype(np.int32) if rows else np.zeros(0, np.int32)
    vals = np.concatenate([r[3] for r in rows]).astype(np.int32) if rows else np.zeros(0, np.int32)
    return MacaulayMatrix(p, ncl, ncr, ptr, cols, vals, laopt)


def dense_lowrank(n_rows: int, n_cols: int, rank: int, p: int, seed: int = 0) -> np.ndarray:
    """Residue matrix L * R mod p (int64) of rank <= ``rank``, L and R uniform.

    Exact: the products are split into 16-bit halves of R so every partial
    sum stays far below 2^63."""
    rng = np.random.default_rng(seed)
    L = rng.integers(0, p, size=(n_rows, rank), dtype=np.int64)
    R = rng.integers(0, p, size=(rank, n_cols), dtype=np.int64)
    out = np.zeros((n_rows, n_cols), dtype=np.int64)
    r_lo, r_hi = R & 0xFFFF, R >> 16
    step = max(1, int((1 << 62) // (max(p - 1, 1) << 16)))
    for k0 in range(0, rank, step):
        lo = (L[:, k0:k0 + step] @ r_lo[k0:k0 + step, :]) % p
        hi = (L[:, k0:k0 + step] @ r_hi[k0:k0 + step, :]) % p
        out = (out + lo + ((hi << 16) % p)) % p
    return out


def dense_block_macaulay(D: np.ndarray, p: int, laopt: int = 1) -> MacaulayMatrix:
    """A Macaulay matrix whose answer is the reduced row echelon form of the
    dense residue block ``D`` (r x m): r known pivots [e_i | 0] followed by r
    rows [e_i | D_i] (lead i, coefficient 1).  Its Schur complement is D
    itself, so a la call on it runs exactly the dense echelon and
    interreduction of the D block (src/la_ff_32.c:1217 and :1181 for la option
    1); the answer's columns are those of D shifted by r."""
    D = np.asarray(D, dtype=np.int64)
    r, m = D.shape
    nz = D != 0
    lens = nz.sum(axis=1).astype(np.int64)
    ptr = np.zeros(2 * r + 1, dtype=np.int64)
    ptr[1:r + 1] = np.arange(1, r + 1)
    ptr[r + 1:] = r + np.cumsum(1 + lens)
    nnz = int(ptr[-1])
    cols = np.empty(nnz, dtype=np.int32)
    vals = np.empty(nnz, dtype=np.int32)
    cols[:r] = np.arange(r)
    vals[:r] = 1
    starts = ptr[r:2 * r]
    cols[starts] = np.arange(r)
    vals[starts] = 1
    ri, ci = np.nonzero(nz)
    # position of entry k of row i: starts[i] + 1 + (rank of k within row i)
    within = np.arange(ri.shape[0]) - np.repeat(np.concatenate(([0], np.cumsum(lens)[:-1])), lens)
    at = starts[ri] + 1 + within
    cols[at] = r + ci
    vals[at] = D[ri, ci]
    return MacaulayMatrix(p, r, m, ptr, cols, vals, laopt)


def monomials_drl_desc(nvars: int, maxdeg: int):
    """All exponent vectors of total degree <= maxdeg, in descending DRL order
    (degree first, then the smaller exponent of the last differing variable
    is larger, src/order.c:239-267) -- the term order gb's input expects."""
    mons = [e for d in range(maxdeg + 1)
            for e in itertools.product(range(d + 1), repeat=nvars) if sum(e) == d]
    return sorted(mons, key=lambda e: (sum(e), tuple(-x for x in reversed(e))), reverse=True)


def dense_system(nvars: int, ngens: int, maxdeg: int, p: int, seed: int):
    """`ngens` polynomials in `nvars` variables, each with every monomial of
    degree <= maxdeg and coefficients uniform in [1, p-1] (seeded), as gb's
    f4_julia takes them: (term counts, coefficients, exponent vectors)."""
    rng = np.random.default_rng(seed)
    mons = monomials_drl_desc(nvars, maxdeg)
    lens, cfs, exps = [], [], []
    for _ in range(ngens):
        lens.append(len(mons))
        cfs += rng.integers(1, p, size=len(mons)).tolist()
        for e in mons:
            exps += list(e)
    return lens, cfs, exps


def f4_case(name: str, nvars: int, ngens: int, maxdeg: int, p: int, la_option: int,
            seed: int, nr_threads: int = 1) -> dict:
    """The f4_julia arguments of a dense system (DRL, no final reduction)."""
    lens, cfs, exps = dense_system(nvars, ngens, maxdeg, p, seed)
    return {"name": name, "nr_vars": nvars, "nr_gens": ngens, "ht_size": 12, "field_char": p,
            "mon_order": 0, "nr_threads": nr_threads, "la_option": la_option, "reduce_gb": 0,
            "max_nr_pairs": 0, "reset_hash_table": 0, "lens": lens, "cfs": cfs, "exps": exps}



_SYNTH_LIB = None


def staircase_native(nru: int, nrl: int, ncr: int, p: int, dmin: float, dmax: float,
                     band: float = 4.0, seed: int = 1, laopt: int = 1,
                     threads: int = 0) -> MacaulayMatrix:
    """The banded A|B/C|D structure of ``staircase`` drawn by the host
    generator libgbsynth.so (gb_b200/csrc/synth.cpp; host threads, one random
    stream per row, so the matrix does not depend on the thread count): for
    the batched workloads, whose matrices reach hundreds of millions of
    entries.  Inside each band the columns are one draw per equal stratum."""
    import ctypes as C
    import os
    global _SYNTH_LIB
    if _SYNTH_LIB is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libgbsynth.so")
        lib = C.CDLL(path)
        lib.gbsynth_staircase_layout.restype = C.c_int64
        lib.gbsynth_staircase_layout.argtypes = [C.c_int32] * 3 + [C.c_double] * 3 + [
            C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p]
        lib.gbsynth_staircase_fill.argtypes = [C.c_int32] * 4 + [C.c_double] * 3 + [
            C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _SYNTH_LIB = lib
    lib = _SYNTH_LIB
    threads = threads or (os.cpu_count() or 1)
    nr = nru + nrl
    ptr = np.empty(nr + 1, dtype=np.int64)
    order = np.empty(max(nr, 1), dtype=np.int32)
    nnz = lib.gbsynth_staircase_layout(nru, nrl, ncr, dmin, dmax, band, seed, threads,
                                       ptr.ctypes.data, order.ctypes.data)
    if nnz < 0:
        raise ValueError("bad staircase parameters")
    cols = np.empty(max(nnz, 1), dtype=np.int32)
    vals = np.empty(max(nnz, 1), dtype=np.int32)
    if lib.gbsynth_staircase_fill(nru, nrl, ncr, p, dmin, dmax, band, seed, threads,
                                  ptr.ctypes.data, order.ctypes.data, cols.ctypes.data,
                                  vals.ctypes.data) != 0:
        raise ValueError("bad staircase parameters")
    return MacaulayMatrix(p, nru, ncr, ptr, cols[:nnz], vals[:nnz], laopt)


def f4_round(nv: int, maxdeg: int, n_cols: int, nr: int, n_piv: int, row_len: int,
             seed: int = 0):
    """Synthetic input of one F4 round's conversion step: n_cols distinct
    monomials in nv variables of degree <= maxdeg (the secondary hash table,
    hash index = position + 1), the first n_piv of them marked as lead
    monomials of known pivots (idx 2, the rest 1), and nr rows of about
    row_len distinct hash indices each whose first entry (the lead term) is a
    pivot monomial.  Returns dict(nv, exps [n][nv] int16, deg, idx, row_ptr,
    hashes)."""
    from math import comb
    if n_cols > comb(nv + maxdeg, maxdeg):
        raise ValueError("fewer monomials of that degree than columns asked for")
    rng = np.random.default_rng(seed)
    mons = set()
    for _ in range(64 * n_cols):
        if len(mons) >= n_cols:
            break
        d = int(rng.integers(0, maxdeg + 1))
        mons.add(tuple(int(x) for x in rng.multinomial(d, [1.0 / nv] * nv)))
    if len(mons) < n_cols:
        raise ValueError("could not draw enough distinct monomials")
    mons = sorted(mons)
    rng.shuffle(mons)
    exps = np.array(mons, dtype=np.int16).reshape(n_cols, nv)
    deg = exps.sum(axis=1).astype(np.int32)
    idx = np.ones(n_cols, dtype=np.int32)
    idx[:n_piv] = 2
    perm = rng.permutation(n_cols)  # table order differs from the pivot marks
    exps, deg, idx = exps[perm], deg[perm], idx[perm]
    piv_hashes = np.flatnonzero(idx == 2) + 1
    ptr = [0]
    hashes = []
    for i in range(nr):
        lead = int(piv_hashes[i]) if i < len(piv_hashes) else int(rng.choice(piv_hashes))
        k = max(1, int(rng.integers(max(1, row_len // 2), row_len + row_len // 2 + 1)))
        k = min(k, n_cols)
        cand = np.unique(rng.integers(1, n_cols + 1, size=2 * k + 8))
        cand = cand[cand != lead]
        rest = rng.permutation(cand)[:k - 1]
        hashes.append(np.concatenate([[lead], rest]))
        ptr.append(ptr[-1] + hashes[-1].shape[0])
    return {"nv": nv, "exps": np.ascontiguousarray(exps), "deg": deg, "idx": idx,
            "row_ptr": np.array(ptr, dtype=np.int64),
            "hashes": np.concatenate(hashes).astype(np.int32)}


def column_order_key(exps: np.ndarray, deg: np.ndarray, idx: np.ndarray, mo: int) -> list:
    """Sort keys of the reference's column order (hcm_cmp, src/order.c:153-235)
    for monomials given by rows of exps: pivot monomials (idx 2) first, then
    DRL (mo 0): higher degree first, then the smaller exponent of the last
    variable where they differ; LEX (mo 1): the larger exponent of the first
    variable where they differ."""
    keys = []
    for e, d, i in zip(exps.tolist(), deg.tolist(), idx.tolist()):
        if mo == 1:
            keys.append((-i,) + tuple(-x for x in e))
        else:
            keys.append((-i, -d) + tuple(reversed(e)))
    return keys


def distinct_monomials(n: int, nv: int, max_exp: int = 31, seed: int = 1) -> np.ndarray:
    """``n`` distinct exponent vectors of ``nv`` variables (int16, entries in
    [0, max_exp]): the monomials of a matrix's columns for the basis-
    conversion workloads."""
    rng = np.random.default_rng(seed)
    if (max_exp + 1) ** nv < 2 * n:
        raise ValueError("too few monomials of this shape")
    out = np.empty((0, nv), dtype=np.int16)
    while out.shape[0] < n:
        cand = rng.integers(0, max_exp + 1, size=(2 * n, nv)).astype(np.int16)
        out = np.unique(np.concatenate([out, cand]), axis=0)
    return rng.permutation(out)[:n]
