"""Host-side containers for Macaulay matrices and their reduced rows.

A Macaulay matrix is kept in the flat CSR form the C ABI takes
(``include/gbgpu.h``): ``nr`` rows over ``nc = ncl + ncr`` columns, row ``i``
holding ``cols[row_ptr[i]:row_ptr[i+1]]`` with residues ``vals[...]`` in
``[1, p)``.  It restates the ``mat_t`` contract of the reference
(``src/data.h:137-155``, ``src/convert.c:30-135``, ``src/order.c:98-131``):

* the first entry of a row is its lead column; the other entries may come in
  any order (``src/convert.c:111-120``);
* every lead lies in the left block (``< ncl``) and every left column is the
  lead of at least one row; the first row per lead is the known pivot (A|B),
  all later rows with that lead form C|D (``src/la_ff_16.c:762-772``);
* every row is monic (lead coefficient 1), as F4 builds them
  (``src/basis.c:252``, ``src/hash.c:903-925``).

The reduced answer (:class:`ReducedRows`) is CSR with ascending columns, lead
coefficient 1, rows in the reference's output order.
"""
from __future__ import annotations

import dataclasses
import io
import struct
from typing import Dict, Iterator, List, Tuple

import numpy as np


def ff_bits(p: int) -> int:
    """Coefficient width the reference selects for prime ``p`` (``src/io.c:815-828``)."""
    if p < 1 << 7:
        return 8
    if p < 1 << 15:
        return 16
    return 32


def kernel_family(p: int) -> str:
    """Row-kernel family of ``src/io.c:710-729``: '17_bit' below 2^17, else '31_bit'."""
    return "17_bit" if p < 1 << 17 else "31_bit"


@dataclasses.dataclass
class MacaulayMatrix:
    """One input of the linear-algebra step (CSR, 0-based columns)."""

    p: int
    ncl: int
    ncr: int
    row_ptr: np.ndarray  # int64 [nr + 1]
    cols: np.ndarray  # int32 [nnz]
    vals: np.ndarray  # int32 [nnz]
    laopt: int = 1

    def __post_init__(self) -> None:
        self.row_ptr = np.ascontiguousarray(self.row_ptr, dtype=np.int64)
        self.cols = np.ascontiguousarray(self.cols, dtype=np.int32)
        self.vals = np.ascontiguousarray(self.vals, dtype=np.int32)

    @property
    def nr(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def nc(self) -> int:
        return int(self.ncl + self.ncr)

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def leads(self) -> np.ndarray:
        return self.cols[self.row_ptr[:-1]]

    def split_counts(self) -> Tuple[int, int]:
        """(nru, nrl): number of known pivots and of rows to reduce."""
        nru = int(np.unique(self.leads()).shape[0]) if self.nr else 0
        return nru, self.nr - nru

    def validate(self) -> None:
        """Raise ValueError when the matrix breaks the ``mat_t`` contract."""
        if self.p < 2 or self.p >= 1 << 31:
            raise ValueError(f"prime {self.p} out of range [2, 2^31)")
        lens = np.diff(self.row_ptr)
        if self.nr and lens.min() <= 0:
            raise ValueError("empty row")
        if self.nnz:
            if self.cols.min() < 0 or self.cols.max() >= self.nc:
                raise ValueError("column index out of range")
            if self.vals.min() < 1 or self.vals.max() >= self.p:
                raise ValueError("coefficient outside [1, p)")
        leads = self.leads()
        if self.nr and leads.max() >= self.ncl:
            raise ValueError("a lead lies in the right block")
        if np.any(self.vals[self.row_ptr[:-1]] != 1):
            raise ValueError("row not monic")
        have = np.zeros(self.ncl, dtype=bool)
        have[leads] = True
        if not have.all():
            raise ValueError("left column without a known pivot")
        row_of = np.repeat(np.arange(self.nr), lens)
        if np.any(self.cols < leads[row_of]):
            raise ValueError("entry left of its row's lead")

    def rows(self) -> Iterator[Tuple[np.ndarray, np.ndarray]]:
        for i in range(self.nr):
            a, b = self.row_ptr[i], self.row_ptr[i + 1]
            yield self.cols[a:b], self.vals[a:b]

    def subset(self, keep_lower: np.ndarray) -> "MacaulayMatrix":
        """Same known pivots, only the C|D rows selected by ``keep_lower``
        (indices into the non-pivot rows in row order)."""
        leads = self.leads()
        first = np.zeros(self.nr, dtype=bool)
        _, idx = np.unique(leads, return_index=True)
        first[idx] = True
        lower = np.flatnonzero(~first)
        sel = np.sort(np.concatenate([np.flatnonzero(first), lower[keep_lower]]))
        return self.take_rows(sel)

    def take_rows(self, sel: np.ndarray) -> "MacaulayMatrix":
        lens = np.diff(self.row_ptr)[sel]
        ptr = np.zeros(sel.shape[0] + 1, dtype=np.int64)
        np.cumsum(lens, out=ptr[1:])
        idx = np.concatenate([np.arange(self.row_ptr[i], self.row_ptr[i + 1]) for i in sel]) \
            if sel.shape[0] else np.zeros(0, dtype=np.int64)
        return MacaulayMatrix(self.p, self.ncl, self.ncr, ptr, self.cols[idx], self.vals[idx], self.laopt)


@dataclasses.dataclass
class ReducedRows:
    """Answer of the linear-algebra step: ``np`` rows in CSR form."""

    row_ptr: np.ndarray
    cols: np.ndarray
    vals: np.ndarray

    def __post_init__(self) -> None:
        self.row_ptr = np.ascontiguousarray(self.row_ptr, dtype=np.int64)
        self.cols = np.ascontiguousarray(self.cols, dtype=np.int32)
        self.vals = np.ascontiguousarray(self.vals, dtype=np.int32)

    @property
    def np(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def equals(self, other: "ReducedRows") -> bool:
        return (
            self.np == other.np
            and np.array_equal(self.row_ptr, other.row_ptr)
            and np.array_equal(self.cols[: self.nnz], other.cols[: other.nnz])
            and np.array_equal(self.vals[: self.nnz], other.vals[: other.nnz])
        )

    def first_difference(self, other: "ReducedRows") -> str:
        if self.np != other.np:
            return f"row count {self.np} != {other.np}"
        for i in range(self.np):
            a0, a1 = self.row_ptr[i], self.row_ptr[i + 1]
            b0, b1 = other.row_ptr[i], other.row_ptr[i + 1]
            if a1 - a0 != b1 - b0:
                return f"row {i}: length {a1 - a0} != {b1 - b0}"
            if not np.array_equal(self.cols[a0:a1], other.cols[b0:b1]):
                return f"row {i}: columns differ"
            if not np.array_equal(self.vals[a0:a1], other.vals[b0:b1]):
                return f"row {i}: coefficients differ"
        return "equal"


# --------------------------------------------------------------------------
# .gbm capture files (written by the test-only reference build) and the
# compressed .npz bundles the golden fixtures are stored in.

_GBM_HDR = struct.Struct("<4s8i")


def _read_rows(buf: io.BytesIO, nr: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    (nnz,) = struct.unpack("<q", buf.read(8))
    ptr = np.frombuffer(buf.read(8 * (nr + 1)), dtype=np.int64).copy()
    cols = np.frombuffer(buf.read(4 * nnz), dtype=np.int32).copy()
    vals = np.frombuffer(buf.read(4 * nnz), dtype=np.int32).copy()
    return ptr, cols, vals


def read_gbm(data: bytes) -> Tuple[int, MacaulayMatrix, ReducedRows, Dict[str, int]]:
    """Parse one capture: (kind, input, reference answer, header fields)."""
    buf = io.BytesIO(data)
    magic, kind, p, laopt, nr, nru, nrl, ncl, ncr = _GBM_HDR.unpack(buf.read(_GBM_HDR.size))
    if magic != b"GBM1":
        raise ValueError("not a .gbm capture")
    ptr, cols, vals = _read_rows(buf, nr)
    mat = MacaulayMatrix(p, ncl, ncr, ptr, cols, vals, laopt)
    (npiv,) = struct.unpack("<i", buf.read(4))
    optr, ocols, ovals = _read_rows(buf, npiv)
    hdr = dict(kind=kind, p=p, laopt=laopt, nr=nr, nru=nru, nrl=nrl, ncl=ncl, ncr=ncr)
    return kind, mat, ReducedRows(optr, ocols, ovals), hdr


@dataclasses.dataclass
class Capture:
    kind: int  # 0: linear_algebra call, 1: interreduce_matrix_rows call
    mat: MacaulayMatrix
    answer: ReducedRows


def save_captures(path: str, caps: List[Capture]) -> None:
    arrays = {}
    for k, c in enumerate(caps):
        m, a = c.mat, c.answer
        arrays[f"c{k}_hdr"] = np.array([c.kind, m.p, m.laopt, m.ncl, m.ncr], dtype=np.int64)
        arrays[f"c{k}_ptr"] = m.row_ptr
        arrays[f"c{k}_cols"] = m.cols
        arrays[f"c{k}_vals"] = m.vals
        arrays[f"c{k}_optr"] = a.row_ptr
        arrays[f"c{k}_ocols"] = a.cols
        arrays[f"c{k}_ovals"] = a.vals
    np.savez_compressed(path, **arrays)


def load_captures(path: str) -> List[Capture]:
    z = np.load(path)
    n = sum(1 for k in z.files if k.endswith("_hdr"))
    caps = []
    for k in range(n):
        kind, p, laopt, ncl, ncr = (int(x) for x in z[f"c{k}_hdr"])
        mat = MacaulayMatrix(p, ncl, ncr, z[f"c{k}_ptr"], z[f"c{k}_cols"], z[f"c{k}_vals"], laopt)
        ans = ReducedRows(z[f"c{k}_optr"], z[f"c{k}_ocols"], z[f"c{k}_ovals"])
        caps.append(Capture(kind, mat, ans))
    return caps
