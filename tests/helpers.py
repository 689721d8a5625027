"""Shared fixtures data for the test-suite (golden files, small generators)."""
import glob
import json
import os

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
