"""Fingerprints of the reference's own results at the benchmark sizes, for bit-exact parity
tests that cannot carry the states themselves (68 MB / 1.2 GB).

Runs the reference build (oracle/_ref, compiled from the reference's sources by
oracle/Makefile) on:
  * ot2d_1024_t0.5: Orszag-Tang 1024^2 (HLLD, WCNS4, CUCT, RK3) through its exec_ loop to t = 0.5;
  * kh3d_256_20steps: Kelvin-Helmholtz 3D 256^3 (MLAU, WCNS4, CUCT, RK3), 20 exec_ steps;
  * kh3d_64_1000steps: the same problem at 64^3 for the configuration's full 1000 steps;
  * c4_<q>: instances q of the 512-member batched ensemble (problems.ensemble(512), log-uniform
    sides 64..512; Orszag-Tang/HLLD and Kelvin-Helmholtz/MLAU with drawn Mach and beta), each
    200 exec_ steps with its own CFL dt -- the smallest and largest of each half and the Mach /
    beta extremes (C4_SAMPLE);
and writes tests/golden/fullsize.json: SHA-256 of the final state (8 fields incl. ghosts,
little-endian float64), step count, time and dt.  The first two take ~15 minutes on 8 cores,
the others ~10 minutes.  Named keys recompute only those entries:

    python tests/golden/make_fullsize.py [--threads N] [key ...]
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refcase as R  # noqa: E402
from qasmhd_b200 import problems as P  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fullsize.json")

# ensemble members: OT smallest / largest, KH smallest / largest, KH lowest / highest Mach,
# lowest / highest beta, and two small KH instances at high Mach and at low beta
C4_SAMPLE = (192, 238, 325, 235, 471, 469, 263, 71, 173, 367)
C4_STEPS = 200


def fingerprint(state) -> str:
    return hashlib.sha256(np.ascontiguousarray(state, dtype="<f8").tobytes()).hexdigest()


def entries():
    out = {
        "ot2d_1024_t0.5": (lambda: P.orszag_tang(1024), R.MODE_EXEC, 0),
        "kh3d_256_20steps": (lambda: P.kelvin_helmholtz(3, 256), R.MODE_RUN, 20),
        "kh3d_64_1000steps": (lambda: P.kelvin_helmholtz(3, 64), R.MODE_RUN, 1000),
    }
    for q in C4_SAMPLE:
        out[f"c4_{q}"] = ((lambda q=q: P.ensemble(512)[q]), R.MODE_RUN, C4_STEPS)
    return out


def main():
    args = sys.argv[1:]
    threads = os.cpu_count()
    if args[:1] == ["--threads"]:
        threads, args = int(args[1]), args[2:]
    todo = entries()
    keys = args or list(todo)
    old = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for key in keys:
        build, mode, nsteps = todo[key]
        p = build()
        r = R.run_reference(p, mode, nsteps=nsteps, nthreads=threads, timeout=7200)
        old[key] = {"sha256": fingerprint(r["state"]), "steps": int(r["steps"]), "tim": float(r["tim"]),
                    "dt": float(r["dt"])}
        print(key, old[key], flush=True)
        with open(OUT, "w") as f:
            json.dump(old, f, indent=1)


if __name__ == "__main__":
    main()
