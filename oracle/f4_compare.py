"""TEST INFRASTRUCTURE ONLY: gb's F4 on a dense system with every la call
compared against the reference's own la, run as a child process.

    python -m oracle.f4_compare --nvars 10 --ngens 10 --maxdeg 3 \\
        --p 2147483647 --la-option 1 --seed 10 --budget 60 --log calls.log [--impl gpu]

The reference build (oracle/_ref/libgbref.so, src/f4.c:190 f4_julia) runs F4;
its hook (gbref_set_compare in ref/gbref_hook.c) sends each call at
src/f4.c:306 to the implementation under test (--impl gpu: libgbgpu.so's
gbgpu_linear_algebra; --impl reference: the reference's la again, a
self-check of the harness) and, on a deep copy of the matrix, to the
reference's own la, and logs one line per call.  Once the reference calls
have used --budget seconds the process ends, so a large F4 run is compared
round by round up to a fixed CPU budget.  The last line is "done" when F4
finished within the budget, "stop budget ..." otherwise.
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from gb_b200 import synth  # noqa: E402


def parse_log(path: str) -> dict:
    """Calls (dicts of the logged fields) and how the run ended."""
    calls, end = [], None
    with open(path) as fh:
        for line in fh:
            w = line.split()
            if not w:
                continue
            if w[0] == "call":
                d = {}
                for k, v in zip(w[0::2], w[1::2]):
                    d[k] = float(v) if k.endswith("_s") else int(v)
                calls.append(d)
            else:
                end = line.strip()
    return {"calls": calls, "end": end}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nvars", type=int, required=True)
    ap.add_argument("--ngens", type=int, required=True)
    ap.add_argument("--maxdeg", type=int, required=True)
    ap.add_argument("--p", type=int, required=True)
    ap.add_argument("--la-option", type=int, default=1)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--budget", type=float, required=True)
    ap.add_argument("--log", required=True)
    ap.add_argument("--impl", choices=["gpu", "reference"], default="gpu")
    a = ap.parse_args()
    case = synth.f4_case("f4_compare", a.nvars, a.ngens, a.maxdeg, a.p, a.la_option, a.seed,
                         nr_threads=a.threads)
    lib = oracle._load_ref()
    fn = None
    if a.impl == "gpu":
        from gb_b200 import la
        fn = la.function_address("gbgpu_linear_algebra")
    lib.gbref_set_compare.argtypes = [C.c_void_p, C.c_double, C.c_char_p]
    if lib.gbref_set_compare(fn, a.budget, a.log.encode()) != 0:
        raise SystemExit(f"cannot open {a.log}")
    oracle._run_f4(lib, case)
    lib.gbref_set_compare(None, 0.0, None)  # closes the log
    with open(a.log, "a") as fh:
        fh.write("done\n")


if __name__ == "__main__":
    main()
