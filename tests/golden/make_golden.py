"""Regenerate the golden fixtures under tests/golden/ from the reference.

Run in a container that has the reference tree (default /root/reference) and
the test-only reference build oracle/_ref/libgbref.so (``make -C oracle``):

    python tests/golden/make_golden.py [--reference /root/reference]

It writes
  f4/<name>.json   -- for every end-to-end F4 program in the reference's
                      test/ directory: its inputs and parameters, read from
                      the C source as text, and the expected basis.  The
                      expected arrays are the ones the program itself checks
                      (tlen/tcf/texp, bld/nterms) where it has them
                      ("golden": "test-source"); for programs without checks,
                      the basis the reference build returns here
                      ("golden": "reference-run").
  mats/<name>.npz  -- every matrix the reference's F4 hands to its linear
                      algebra on that program (linear_algebra, src/f4.c:306,
                      and interreduce_matrix_rows, src/f4.c:137), together with
                      the reference's own answer, captured through the hooks of
                      oracle/ref/gbref_hook.c.
  kat_normalize_row.json -- the known answer of test/normalize_row.c.

These fixtures are what pins the C oracle and the GPU library; the GPU box
never reads the reference tree.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from gb_b200.matrix import Capture, read_gbm, save_captures  # noqa: E402
import oracle  # noqa: E402

# end-to-end programs of the reference's test suite (test/Makefile.am:22-62)
# that finish in seconds; the large disabled ones (test/Makefile.am:63-72)
# are left out, and so are the rational ones (they need GMP)
F4_PROGRAMS = [
    "cyclic_4_drl_7_bit", "cyclic_4_drl_15_bit", "cyclic_4_drl_17_bit",
    "cyclic_4_h_drl_17_bit", "cyclic_4_drl_31_bit", "cyclic_4_lex_17_bit",
    "cyclic_5_drl_17_bit", "cyclic_5_lex_17_bit",
    "red_gb_7_bit", "red_gb_15_bit", "red_gb_17_bit", "red_gb_31_bit",
    "cyclic_6_drl_17_bit_la1_t1", "cyclic_6_drl_17_bit_la1_t2",
    "cyclic_6_drl_17_bit_la2_t1", "cyclic_6_drl_17_bit_la2_t2",
    "cyclic_6_drl_17_bit_la42_t1", "cyclic_6_drl_17_bit_la42_t2",
    "cyclic_6_drl_17_bit_la43_t1", "cyclic_6_drl_17_bit_la43_t2",
    "cyclic_6_drl_17_bit_la44_t1", "cyclic_6_drl_17_bit_la44_t2",
    "katsura_4_lex", "katsura_5_lex", "cyclic_7",
]
# matrices are stored for these programs only (a few MB in all)
CAPTURE_PROGRAMS = [
    "cyclic_4_drl_7_bit", "cyclic_4_drl_15_bit", "cyclic_4_drl_17_bit",
    "cyclic_4_drl_31_bit", "cyclic_4_lex_17_bit", "cyclic_5_drl_17_bit",
    "cyclic_5_lex_17_bit", "red_gb_7_bit", "red_gb_15_bit", "red_gb_17_bit",
    "red_gb_31_bit", "cyclic_6_drl_17_bit_la1_t1", "cyclic_6_drl_17_bit_la2_t1",
    "katsura_4_lex", "katsura_5_lex",
]

_SCALARS = ["nr_vars", "nr_gens", "ht_size", "field_char", "mon_order", "nr_threads",
            "la_option", "reduce_gb", "max_nr_pairs", "reset_hash_table"]


def _strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
    return re.sub(r"//[^\n]*", " ", src)


def _int_array(src: str, name: str):
    m = re.search(r"\b" + name + r"\s*\[[^\]]*\]\s*=\s*\{([^}]*)\}", src)
    if not m:
        return None
    return [int(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()]


def parse_program(path: str) -> dict:
    src = _strip_comments(open(path).read())
    case = {"name": os.path.splitext(os.path.basename(path))[0]}
    for key in _SCALARS:
        m = re.search(r"const\s+int32_t\s+" + key + r"\s*=\s*(-?\d+)\s*;", src)
        if not m:
            raise ValueError(f"{path}: no {key}")
        case[key] = int(m.group(1))
    for arr in ("lens", "cfs", "exps"):
        case[arr] = _int_array(src, arr)
    m = re.search(r"\(\*bld\)\s*!=\s*(\d+)\s*\|\|\s*nterms\s*!=\s*(\d+)", src)
    golden = {}
    if m:
        golden["bld"], golden["nterms"] = int(m.group(1)), int(m.group(2))
    for arr in ("tlen", "tcf", "texp"):
        v = _int_array(src, arr)
        if v is not None:
            golden[arr] = v
    case["expected"] = golden
    case["golden"] = "test-source" if golden else "reference-run"
    return case


def run_case(case: dict, capture_dir=None):
    lens, cfs, exps = oracle.ref_f4(case, capture_dir=capture_dir)
    return lens, cfs, exps


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    tdir = os.path.join(args.reference, "test")
    os.makedirs(os.path.join(HERE, "f4"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "mats"), exist_ok=True)

    for name in F4_PROGRAMS:
        case = parse_program(os.path.join(tdir, name + ".c"))
        with tempfile.TemporaryDirectory() as cap:
            lens, cfs, exps = run_case(case, capture_dir=cap)
            caps = []
            for f in sorted(glob.glob(os.path.join(cap, "*.gbm"))):
                kind, mat, ans, _ = read_gbm(open(f, "rb").read())
                caps.append(Capture(kind, mat, ans))
        got = {"bld": int(lens.shape[0]), "nterms": int(lens.sum()), "tlen": lens.tolist(),
               "tcf": cfs.tolist(), "texp": exps.tolist()}
        exp = case["expected"]
        if case["golden"] == "test-source":
            for k, v in exp.items():
                if got[k] != v:
                    raise SystemExit(f"{name}: reference build disagrees with its own test on {k}")
        else:
            case["expected"] = got
        case["n_la_calls"] = len(caps)
        case["max_matrix"] = max(([c.mat.nr, c.mat.nc] for c in caps), default=[0, 0],
                                 key=lambda x: x[0] * x[1])
        with open(os.path.join(HERE, "f4", name + ".json"), "w") as fh:
            json.dump(case, fh)
        if name in CAPTURE_PROGRAMS:
            save_captures(os.path.join(HERE, "mats", name + ".npz"), caps)
        print(f"{name}: {case['golden']}, {len(caps)} la calls, largest {case['max_matrix']}")

    # test/normalize_row.c: normalise [16, 299, 298, ..., 285] modulo 101
    src = _strip_comments(open(os.path.join(tdir, "normalize_row.c")).read())
    checks = [(int(a), int(b)) for a, b in re.findall(r"row\[(\d+)\]\s*!=\s*(\d+)", src)]
    kat = {"p": 101, "row": [16] + [300 - i for i in range(1, 16)], "checks": checks}
    with open(os.path.join(HERE, "kat_normalize_row.json"), "w") as fh:
        json.dump(kat, fh)
    print("normalize_row:", checks)


if __name__ == "__main__":
    main()
