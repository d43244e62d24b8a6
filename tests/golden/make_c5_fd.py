"""Finite-difference reference for the adjoint's gradient on the C5 configuration, in extended
precision.

C5: 2D Kelvin-Helmholtz 256^2, M = 0.1, beta = 100, Roe + WCNS4 + CT + RK3, 400 steps with the
frozen dt sequence of the unperturbed run, uniform eta; loss = L2 misfit of the final
(vx, vy, bx, by) to the target run (seeded perturbation, eta* = 1e-4) -- the inversion of
qasmhd_b200.adjoint.KHInverse.  Central differences of that loss are taken on the reference's
own 2D stepping code compiled in long double (oracle/_ref/ref2d_ld_ctw1, built from
2D/SERIAL/MRX and common/*.c by oracle/Makefile): 32 seeded directions of the vy perturbation
(eps = 1e-6, the directions of adjoint.directional_check) and eta (step 1e-9).  In double
precision the same differences are quantised by the pressure recovery (a 1e-6 change of vy
moves `en` by tens of ulps); the 64-bit significand removes that floor.

Inputs made here on the CPU from the reference's double build: the dt sequence (exec_ rule,
setdt every second step, eta*) and the target observation (the reference's 400-step run from the
target perturbation).  Beside the differences the file holds the same directional derivatives
from the reference's dual-number build (oracle/_ref/ref2d_dual_ctw1: the exact derivative of
the double-precision program along each direction, `dual_dirs`, `dual_eta`).  Writes
tests/golden/c5_fd_longdouble.json (other sizes: c5_fd_longdouble_<n>_<nsteps>_<ndir>.json).
~2 hours on 8 cores at full size:

    python tests/golden/make_c5_fd.py [n nsteps ndir]     # defaults 256 400 32
    python tests/golden/make_c5_fd.py --dual FILE         # (re)compute the dual fields of FILE
"""
import json
import os
import struct
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refcase as R  # noqa: E402
from qasmhd_b200.problems import RMN_ROE, XOFF, kelvin_helmholtz  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c5_fd_longdouble.json")
MACH, BETA, ETA_TARGET, TARGET_SEED = 0.1, 100.0, 1e-4, 2025
DVY_SEED, DIR_SEED, ETA, EPS, EPS_ETA = 7, 11, 0.5e-4, 1e-6, 1e-9


def setup(n):
    base = kelvin_helmholtz(dim=2, n=n, mach=MACH, beta=BETA, rmn=RMN_ROE, odr=4, rk=3, ctw=1,
                            dvy_field=np.zeros((n, n)))
    x, y, _ = base.coords()
    Y, _X = np.meshgrid(y, x, indexing="ij")
    amp = (1e-3 * MACH * np.exp(-(Y / 0.1) ** 2))[XOFF:XOFF + n, XOFF:XOFF + n]
    return base, amp


def state(base, amp, dvy):
    """KHInverse.state in numpy: vy = amp * dvy on the interior, my = ro vy, en += ro vy^2 / 2."""
    n = amp.shape[0]
    u = base.state.reshape(8, base.ny, base.nx).copy()
    vy = np.zeros_like(u[0])
    vy[XOFF:XOFF + n, XOFF:XOFF + n] = amp * dvy
    ro = u[0]
    u[2] = ro * vy
    u[7] = u[7] + 0.5 * ro * vy * vy
    return u


def observe(u, n):
    s = (slice(XOFF, XOFF + n), slice(XOFF, XOFF + n))
    ro = u[0][s]
    return np.stack([u[1][s] / ro, u[2][s] / ro, u[4][s], u[5][s]])


def dual_derivatives(gold, ndir=None):
    """Directional derivatives of the loss along the golden's directions (the first ndir) and
    eta from the reference's dual-number build, with the golden's dt sequence:
    dL = 2 sum (obs - target) d(obs), d(vx) = d(mx)/ro - mx d(ro)/ro^2."""
    n = gold["n"]
    ndir = len(gold["fd_dirs"]) if ndir is None else ndir
    threads = os.cpu_count()
    base, amp = setup(n)
    dts = np.array(gold["dts"])
    ut = state(base, amp, np.random.default_rng(gold["target_seed"]).standard_normal((n, n)))
    fin_t, _ = R.run_reference_dual(base, ut.reshape(8, -1), np.zeros((8, base.nd)), dts,
                                    eta0=gold["eta_target"], nthreads=threads)
    target = observe(fin_t.reshape(8, base.ny, base.nx), n)
    u0 = state(base, amp, np.random.default_rng(gold["dvy_seed"]).standard_normal((n, n)))
    ro = u0[0]
    vy = u0[2] / ro
    s = (slice(XOFF, XOFF + n), slice(XOFF, XOFF + n))
    ampf = np.zeros_like(ro)
    ampf[s] = amp
    rng = np.random.default_rng(gold["dir_seed"])
    tangents = []
    for _ in range(ndir):
        dd = np.zeros_like(ro)
        dd[s] = rng.standard_normal((n, n))
        t = np.zeros_like(u0)
        t[2] = ro * ampf * dd  # d(my) for vy = amp * dvy
        t[7] = ro * vy * ampf * dd  # d(en) = ro vy d(vy)
        tangents.append((t, 0.0))
    tangents.append((np.zeros_like(u0), 1.0))  # eta
    out = []
    for t, deta in tangents:
        v, dv = R.run_reference_dual(base, u0.reshape(8, -1), t.reshape(8, -1), dts, eta0=gold["eta"],
                                     deta=deta, nthreads=threads)
        v = v.reshape(8, base.ny, base.nx)
        dv = dv.reshape(8, base.ny, base.nx)
        d = observe(v, n) - target
        r, dr = v[0][s], dv[0][s]
        dobs = np.stack([dv[1][s] / r - v[1][s] * dr / (r * r), dv[2][s] / r - v[2][s] * dr / (r * r),
                         dv[4][s], dv[5][s]])
        out.append(2.0 * float(np.sum(d * dobs)))
    return out[:-1], out[-1]


def add_dual(path):
    gold = json.load(open(path))
    t0 = time.time()
    gold["dual_dirs"], gold["dual_eta"] = dual_derivatives(gold)
    gold["dual_seconds"] = time.time() - t0
    with open(path, "w") as f:
        json.dump(gold, f, indent=1)
    fd, du = np.array(gold["fd_dirs"]), np.array(gold["dual_dirs"])
    print(path, "max |fd - dual| / max |fd| =", float(np.max(np.abs(fd - du)) / np.max(np.abs(fd))),
          "eta", abs(gold["fd_eta"] - gold["dual_eta"]) / abs(gold["dual_eta"]))


def main():
    if len(sys.argv) > 2 and sys.argv[1] == "--dual":
        add_dual(sys.argv[2])
        return
    n, nsteps, ndir = (int(a) for a in (sys.argv[1:4] if len(sys.argv) > 3 else (256, 400, 32)))
    threads = os.cpu_count()
    base, amp = setup(n)
    # dt sequence of the unperturbed run with eta* (the exec_ rule), from the reference's double build
    p = base.copy()
    p.eta0, p.nu0 = ETA_TARGET, 0.0
    dts = R.run_reference(p, R.MODE_DRUN, nsteps=nsteps, nthreads=threads)["dts"]
    assert len(dts) == nsteps
    # target observation: the reference's run from the target perturbation (value part of the dual build)
    ut = state(base, amp, np.random.default_rng(TARGET_SEED).standard_normal((n, n)))
    fin, _ = R.run_reference_dual(base, ut.reshape(8, -1), np.zeros((8, base.nd)), dts, eta0=ETA_TARGET,
                                  nthreads=threads)
    target = observe(fin.reshape(8, base.ny, base.nx), n)
    dvy = np.random.default_rng(DVY_SEED).standard_normal((n, n))
    rng = np.random.default_rng(DIR_SEED)
    dirs = np.stack([rng.standard_normal((n, n)) for _ in range(ndir)])
    hdr = struct.pack("<10i8d16i", 0x4C534151, n, n, RMN_ROE, 4, 3, 1, nsteps, threads, ndir,
                      base.gam, base.xmin, base.xmax, base.ymin, base.ymax, ETA, EPS, EPS_ETA,
                      *[int(v) for v in base.dnx], *[int(v) for v in base.dny])
    t0 = time.time()
    with tempfile.TemporaryDirectory(prefix="qasld_") as td:
        cin, cout = os.path.join(td, "case.bin"), os.path.join(td, "result.bin")
        with open(cin, "wb") as f:
            f.write(hdr)
            for a in (dts, base.state.reshape(-1), amp, dvy, dirs, target):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        subprocess.run([os.path.join(R.REF_DIR, "ref2d_ld_ctw1"), cin, cout], check=True)
        out = np.fromfile(cout, dtype="<f8")
    res = {"n": n, "nsteps": nsteps, "mach": MACH, "beta": BETA, "eta_target": ETA_TARGET,
           "target_seed": TARGET_SEED, "dvy_seed": DVY_SEED, "dir_seed": DIR_SEED, "eta": ETA, "eps": EPS,
           "eps_eta": EPS_ETA, "dts": [float(d) for d in dts], "fd_dirs": [float(v) for v in out[:ndir]],
           "fd_eta": float(out[ndir]), "loss": float(out[ndir + 1]), "seconds": time.time() - t0,
           "precision": "long double (x87, 64-bit significand)"}
    path = OUT if (n, nsteps, ndir) == (256, 400, 32) else OUT.replace(".json", f"_{n}_{nsteps}_{ndir}.json")
    with open(path, "w") as f:
        json.dump(res, f, indent=1)
    print(path, res["fd_dirs"][:3], res["fd_eta"], res["loss"], f"{res['seconds']:.0f} s")
    add_dual(path)


if __name__ == "__main__":
    main()
