"""Shared fixtures data for the test-suite (golden files, small generators)."""
import glob
import json
import os

from fractions import Fraction

import numpy as np

from gb_b200 import multimod, synth
from gb_b200.matrix import ReducedRows, load_captures

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def f4_cases():
    out = []
    for f in sorted(glob.glob(os.path.join(GOLDEN, "f4", "*.json"))):
        with open(f) as fh:
            out.append(json.load(fh))
    return out


def capture_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "mats", "*.npz")))


def all_captures():
    """(file name, index, Capture) for every captured reference la call."""
    out = []
    for f in capture_files():
        for k, c in enumerate(load_captures(f)):
            out.append((os.path.basename(f)[:-4], k, c))
    return out


def as_rows(mat):
    return ReducedRows(mat.row_ptr, mat.cols, mat.vals)


def kat_normalize():
    with open(os.path.join(GOLDEN, "kat_normalize_row.json")) as fh:
        return json.load(fh)


def exact_answer(mat: multimod.IntegerMacaulay):
    """Rows of the reduced row echelon form over Q whose pivot lies in the
    right block, restricted to it, descending lead (pure Python, small cases)."""
    nr, nc = mat.nr, mat.ncl + mat.ncr
    M = [[Fraction(0)] * nc for _ in range(nr)]
    for i in range(nr):
        for k in range(int(mat.row_ptr[i]), int(mat.row_ptr[i + 1])):
            M[i][int(mat.cols[k])] = Fraction(int(mat.vals[k]))
    piv_row = 0
    pivots = []
    for c in range(nc):
        r = next((r for r in range(piv_row, nr) if M[r][c] != 0), None)
        if r is None:
            continue
        M[piv_row], M[r] = M[r], M[piv_row]
        inv = 1 / M[piv_row][c]
        M[piv_row] = [v * inv for v in M[piv_row]]
        for rr in range(nr):
            if rr != piv_row and M[rr][c] != 0:
                f = M[rr][c]
                M[rr] = [a - f * b for a, b in zip(M[rr], M[piv_row])]
        pivots.append((c, piv_row))
        piv_row += 1
    rows = [(c, M[r]) for c, r in pivots if c >= mat.ncl]
    rows.sort(key=lambda t: -t[0])
    return [[(j, v) for j, v in enumerate(row) if j >= mat.ncl and v != 0] for _, row in rows]


def small_integer_matrix(seed=1, bound=1 << 6):
    m = synth.integer_staircase(40, 15, 30, bound=bound, dmin=0.05, dmax=0.15, seed=seed)
    return multimod.IntegerMacaulay.from_matrix(m, vals=m.vals.astype(np.int64))


def matvec_mod(M, x, p: int, chunk: int = 1024) -> np.ndarray:
    """(M x) mod p exactly for residue matrices M (rows x n, any integer
    dtype, entries < p < 2^31) and residue vectors x: every product is
    reduced before the row sums (each < 2^62, sums of n < 2^32 of them stay
    below 2^63)."""
    M = np.asarray(M)
    x = np.asarray(x, dtype=np.int64)
    out = np.empty(M.shape[0], dtype=np.int64)
    for r0 in range(0, M.shape[0], chunk):
        blk = M[r0:r0 + chunk].astype(np.int64)
        out[r0:r0 + chunk] = ((blk * x[None, :]) % p).sum(axis=1) % p
    return out


def vecmat_mod(a, B, p: int, chunk: int = 512) -> np.ndarray:
    """(a B) mod p exactly for a residue vector a (K) and matrix B (K x N)."""
    a = np.asarray(a, dtype=np.int64)
    B = np.asarray(B)
    out = np.zeros(B.shape[1], dtype=np.int64)
    for k0 in range(0, B.shape[0], chunk):
        blk = B[k0:k0 + chunk].astype(np.int64)
        out = (out + ((blk * a[k0:k0 + chunk, None]) % p).sum(axis=0)) % p
    return out


def dense_rref_rows(R, rank: int, piv_cols, shift: int) -> ReducedRows:
    """The first ``rank`` rows of a dense RREF (ascending pivots) as the
    reference's answer rows: descending lead order, columns + ``shift``."""
    R = np.asarray(R)[:rank][::-1]
    nz = R != 0
    lens = nz.sum(axis=1)
    ptr = np.zeros(rank + 1, dtype=np.int64)
    np.cumsum(lens, out=ptr[1:])
    ri, ci = np.nonzero(nz)
    return ReducedRows(ptr, (ci + shift).astype(np.int32), R[ri, ci].astype(np.int32))
