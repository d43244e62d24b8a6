"""Fingerprints of the reference's own results at the benchmark sizes, for bit-exact parity
tests that cannot carry the states themselves (68 MB / 1.2 GB).

Runs the reference build (oracle/_ref, compiled from the reference's sources by
oracle/Makefile) on:
  * Orszag-Tang 1024^2 (HLLD, WCNS4, CUCT, RK3) through its exec_ loop to t = 0.5;
  * Kelvin-Helmholtz 3D 256^3 (MLAU, WCNS4, CUCT, RK3), 20 exec_ steps;
and writes tests/golden/fullsize.json: SHA-256 of the final state (8 fields incl. ghosts,
little-endian float64), step count, time and dt.  Takes ~15 minutes on 8 cores.

    python tests/golden/make_fullsize.py [threads]
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


def fingerprint(state) -> str:
    return hashlib.sha256(np.ascontiguousarray(state, dtype="<f8").tobytes()).hexdigest()


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else os.cpu_count()
    out = {}
    p = P.orszag_tang(1024)
    r = R.run_reference(p, R.MODE_EXEC, nsteps=0, nthreads=threads, timeout=7200)
    out["ot2d_1024_t0.5"] = {"sha256": fingerprint(r["state"]), "steps": int(r["steps"]), "tim": float(r["tim"]),
                             "dt": float(r["dt"])}
    print("ot2d", out["ot2d_1024_t0.5"], flush=True)
    p = P.kelvin_helmholtz(3, 256)
    r = R.run_reference(p, R.MODE_RUN, nsteps=20, nthreads=threads, timeout=7200)
    out["kh3d_256_20steps"] = {"sha256": fingerprint(r["state"]), "steps": 20, "dt": float(r["dt"])}
    print("kh3d", out["kh3d_256_20steps"], flush=True)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "fullsize.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
