"""Random dense polynomial systems run through the reference's F4, with every
linear-algebra call captured (input matrix + the reference's answer).

    python tests/golden/make_f4_systems.py

Writes, for each system below, tests/golden/f4/<name>.json (inputs and the
basis the reference returns, "golden": "reference-run") and
tests/golden/mats/<name>.npz (the captured matrices).  Uses the test-only
reference build oracle/_ref/libgbref.so; the GPU box only reads the outputs.

Systems (seeded, all monomials of the given degree bound, coefficients uniform
in [1, p-1], terms in descending DRL order as gb's input expects):
  dense_quadratic_7  -- 7 polynomials in 7 variables, degree <= 2,
                        p = 32003 (16-bit path), la option 2, 1 thread.  The
                        configuration the reference's CPU-runnable case names.
  dense_cubic_5_p31  -- 5 polynomials in 5 variables, degree <= 3,
                        p = 2^31 - 1 (31-bit path), la option 1: a small
                        stand-in for the 10-variable dense cubic over 2^31 - 1,
                        whose full F4 run does not finish on a CPU.
"""
from __future__ import annotations

import glob
import itertools
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from gb_b200.matrix import Capture, read_gbm, save_captures  # noqa: E402


def monomials_drl_desc(nvars: int, maxdeg: int):
    """All exponent vectors of total degree <= maxdeg, in descending DRL order
    (degree first, then the smaller exponent of the last differing variable
    is larger, src/order.c:239-267)."""
    mons = [e for d in range(maxdeg + 1)
            for e in itertools.product(range(d + 1), repeat=nvars) if sum(e) == d]
    return sorted(mons, key=lambda e: (sum(e), tuple(-x for x in reversed(e))), reverse=True)


def dense_system(nvars: int, ngens: int, maxdeg: int, p: int, seed: int):
    rng = np.random.default_rng(seed)
    mons = monomials_drl_desc(nvars, maxdeg)
    lens, cfs, exps = [], [], []
    for _ in range(ngens):
        lens.append(len(mons))
        cfs += rng.integers(1, p, size=len(mons)).tolist()
        for e in mons:
            exps += list(e)
    return lens, cfs, exps


SYSTEMS = [
    dict(name="dense_quadratic_7", nvars=7, ngens=7, maxdeg=2, p=32003, la_option=2, seed=7),
    dict(name="dense_cubic_5_p31", nvars=5, ngens=5, maxdeg=3, p=2147483647, la_option=1,
         seed=5),
]


def main() -> None:
    os.makedirs(os.path.join(HERE, "f4"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "mats"), exist_ok=True)
    for sysdef in SYSTEMS:
        lens, cfs, exps = dense_system(sysdef["nvars"], sysdef["ngens"], sysdef["maxdeg"],
                                       sysdef["p"], sysdef["seed"])
        case = {"name": sysdef["name"], "nr_vars": sysdef["nvars"], "nr_gens": sysdef["ngens"],
                "ht_size": 12, "field_char": sysdef["p"], "mon_order": 0, "nr_threads": 1,
                "la_option": sysdef["la_option"], "reduce_gb": 0, "max_nr_pairs": 0,
                "reset_hash_table": 0, "lens": lens, "cfs": cfs, "exps": exps}
        with tempfile.TemporaryDirectory() as cap:
            blen, bcf, bexp = oracle.ref_f4(case, capture_dir=cap)
            caps = []
            for f in sorted(glob.glob(os.path.join(cap, "*.gbm"))):
                kind, mat, ans, _ = read_gbm(open(f, "rb").read())
                caps.append(Capture(kind, mat, ans))
        case["expected"] = {"bld": int(blen.shape[0]), "nterms": int(blen.sum()),
                            "tlen": blen.tolist(), "tcf": bcf.tolist(), "texp": bexp.tolist()}
        case["golden"] = "reference-run"
        case["n_la_calls"] = len(caps)
        case["max_matrix"] = max(([c.mat.nr, c.mat.nc] for c in caps), default=[0, 0],
                                 key=lambda x: x[0] * x[1])
        with open(os.path.join(HERE, "f4", sysdef["name"] + ".json"), "w") as fh:
            json.dump(case, fh)
        save_captures(os.path.join(HERE, "mats", sysdef["name"] + ".npz"), caps)
        print(f"{sysdef['name']}: basis {case['expected']['bld']} elements, "
              f"{len(caps)} la calls, largest {case['max_matrix']}")


if __name__ == "__main__":
    main()
