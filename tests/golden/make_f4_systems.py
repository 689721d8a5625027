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
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from gb_b200.matrix import Capture, read_gbm, save_captures  # noqa: E402
from gb_b200.synth import f4_case  # noqa: E402


SYSTEMS = [
    dict(name="dense_quadratic_7", nvars=7, ngens=7, maxdeg=2, p=32003, la_option=2, seed=7),
    dict(name="dense_cubic_5_p31", nvars=5, ngens=5, maxdeg=3, p=2147483647, la_option=1,
         seed=5),
]


def main() -> None:
    os.makedirs(os.path.join(HERE, "f4"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "mats"), exist_ok=True)
    for sysdef in SYSTEMS:
        case = f4_case(sysdef["name"], sysdef["nvars"], sysdef["ngens"], sysdef["maxdeg"],
                       sysdef["p"], sysdef["la_option"], sysdef["seed"])
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
