"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference ships no golden vectors or known-answer tests, so every fixture
here is produced by running the reference's own code, compiled from its
sources by oracle/Makefile (oracle/_ref/ref1d, ref2d_ctw*, ref3d_ctw*,
ref_kat).  Inputs are regenerated deterministically by qasmhd_b200.problems
and numpy seeds; the fixtures store the outputs plus a SHA-256 of each input
so a drift of the generators is caught.

Run from the repository root:  python tests/golden/make_golden.py
(``--kat <name>`` or ``--steps <case> ...`` regenerate only those fixtures).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refcase as R  # noqa: E402
from qasmhd_b200 import problems as P  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


# ---------------------------------------------------------------------------
# point-function inputs (also used by the tests to rebuild the same inputs)
# ---------------------------------------------------------------------------

def kat_inputs(kind: str, n: int = 200, seed: int = 2024) -> np.ndarray:
    rng = np.random.default_rng(seed)

    def states(m):
        ro = rng.uniform(0.1, 2.0, m)
        v = rng.normal(0.0, 1.0, (m, 3))
        b = rng.normal(0.0, 1.0, (m, 2))
        pr = rng.uniform(0.05, 2.0, m)
        return np.column_stack([ro, v, b, pr])

    if kind == "flux":
        a = np.column_stack([states(n), states(n), rng.normal(0, 1, n), np.full(n, 5.0 / 3.0),
                             rng.normal(0, 0.5, (n, 2))])
        a[::9, 14] = 0.0          # Bn = 0
        a[1::9, 7:14] = a[1::9, 0:7]  # identical left/right states
        return a
    if kind == "interp":
        a = rng.normal(0, 1, (n, 5))
        a[::7] = a[::7, :1]       # constant stencils
        return a
    if kind in ("lrstate", "lrstate_prim", "lrstate_char"):
        ro = np.abs(rng.normal(1, 0.3, (n, 5))) + 0.1
        rest = rng.normal(0, 1, (n, 25))
        pr = np.abs(rng.normal(1, 0.3, (n, 5))) + 0.05
        a = np.concatenate([ro, rest, pr, rng.normal(0, 1, (n, 1)), np.full((n, 1), 5.0 / 3.0)], axis=1)
        a[::7, 5:10] = 0.0        # exactly-zero normal velocity stencils
        a[3::7, 25:30] = 0.0      # exactly-zero bu stencils
        a[5::11, 5:10] *= 8.0     # supersonic centres (fast-mode eigenvectors)
        return a
    if kind == "lrstate_vac":
        # near-vacuum stencils: density and / or pressure falling to 1e-16..1e-10 across the
        # stencil, so that reconstructed face values reach the positivity fallback of
        # mhd_lrstate (common/mhd_func.c:150-160: first order when rho or p <= 1e-12)
        ro = np.repeat(rng.uniform(0.5, 2.0, (n, 1)), 5, axis=1)
        pr = np.repeat(rng.uniform(0.5, 2.0, (n, 1)), 5, axis=1)
        tiny = 10.0 ** rng.uniform(-16, -10, n)
        for r in range(n):
            k = r % 4
            if k == 0:
                ro[r, 3:] = tiny[r]
            elif k == 1:
                pr[r, 3:] = tiny[r]
            elif k == 2:
                ro[r, :2] = tiny[r]
            else:
                pr[r, :2] = tiny[r]
                ro[r, 3:] = tiny[r]
        rest = rng.normal(0, 1, (n, 25))
        return np.concatenate([ro, rest, pr, rng.normal(0, 1, (n, 1)), np.full((n, 1), 5.0 / 3.0)], axis=1)
    if kind == "cuct":
        return np.concatenate([np.abs(rng.normal(1, 0.2, (n, 4))) + 0.1, rng.normal(0, 1, (n, 16))], axis=1)
    if kind == "energy":
        # ro, vx, vy, vz, bx, by, bz, pr-or-en, gamma: low-Mach rows (kinetic energy ~1e-8 of the
        # pressure's), exact zeros and the benchmark gammas
        a = np.column_stack([np.abs(rng.normal(1, 0.3, n)) + 0.05, rng.normal(0, 1, (n, 6)),
                             np.abs(rng.normal(1, 0.5, n)) + 0.05,
                             rng.choice([5.0 / 3.0, 2.0, 1.4], n)])
        a[::5, 1:4] *= 1e-4
        a[2::9, 2:4] = 0.0
        a[4::11, 5:7] = 0.0
        return a
    raise ValueError(kind)


KAT_FUNCS = {"flux": ([0, 1, 2, 3], 7), "interp": (list(range(10, 20)), 2), "lrstate": ([20, 21, 22, 23], 14),
             "lrstate_prim": ([24, 25, 26, 27], 14), "lrstate_char": ([40, 41, 42, 43], 14), "cuct": ([30], 1),
             "lrstate_vac": ([20, 21, 22, 23], 14),
             "energy": ([31, 32], 1)}


# ---------------------------------------------------------------------------
# step cases: (name, builder, mode, nsteps)
# ---------------------------------------------------------------------------

def _kh2_eta():
    p = P.kelvin_helmholtz(2, 16, mach=0.3, rmn=P.RMN_ROE)
    p.eta0 = 1e-3
    p.nu0 = 5e-4
    return p


def _wave3_eta(ctw, nu0, eta0, rmn=P.RMN_HLLD):
    """3D visco-resistive case (DMHD3D::dsptv); eta0=0.3 gives two sub-cycles per step."""
    p = P.smooth_wave(3, 8, ctw=ctw, rmn=rmn)
    p.nu0, p.eta0 = nu0, eta0
    return p


def _prim(p):
    """The primitive-variable reconstruction (mhd_reconst) instead of the characteristic one."""
    p.char_mode = 1
    return p


def _char(p):
    """The Athena-type characteristic reconstruction (mhd_c_reconst)."""
    p.char_mode = 2
    return p


def _wave_bc(dim, seed):
    rng = np.random.default_rng(seed)

    def flags():
        f = [int(rng.choice([-2, -1, 1, 2])) for _ in range(8)]
        f[0] = int(rng.choice([1, 2]))
        f[7] = int(rng.choice([1, 2]))
        return tuple(f)

    dn = tuple(flags() if a < dim and rng.random() < 0.7 else (0,) * 8 for a in range(3))
    return P.smooth_wave(dim, 12 if dim < 3 else 6, dn=dn, rmn=seed % 4)


STEP_CASES = [
    *[(f"bw1d_rmn{r}", (lambda r=r: P.brio_wu(64, rmn=r)), R.MODE_RUN, 5) for r in range(4)],
    *[(f"bw1d_odr{o}", (lambda o=o: P.brio_wu(64, odr=o, rk=min(o, 3))), R.MODE_RUN, 5) for o in (1, 2, 3)],
    ("bw1d_exec", lambda: P.brio_wu(64, tmax=0.02), R.MODE_EXEC, 0),
    ("hall1d_run", lambda: P.hall_shock(64, di=0.02), R.MODE_RUN, 6),
    ("bw1d_prim", lambda: _prim(P.brio_wu(64)), R.MODE_RUN, 5),
    ("ot2d_prim", lambda: _prim(P.orszag_tang(16)), R.MODE_RUN, 3),
    ("kh3d_prim", lambda: _prim(P.kelvin_helmholtz(3, 6, mach=0.3, rmn=P.RMN_MLAU)), R.MODE_RUN, 2),
    ("bw1d_char", lambda: _char(P.brio_wu(64)), R.MODE_RUN, 5),
    ("ot2d_char", lambda: _char(P.orszag_tang(16)), R.MODE_RUN, 3),
    ("kh2d_char_roe", lambda: _char(P.kelvin_helmholtz(2, 16, mach=0.3, rmn=P.RMN_ROE)), R.MODE_RUN, 3),
    ("kh3d_char", lambda: _char(P.kelvin_helmholtz(3, 6, mach=0.3, rmn=P.RMN_MLAU)), R.MODE_RUN, 2),
    ("hall1d_exec", lambda: P.hall_shock(64, di=1e-3, tmax=0.02), R.MODE_EXEC, 0),
    ("hall1d_de_run", lambda: P.hall_shock(64, di=0.01, d_ele=2.0), R.MODE_RUN, 4),
    *[(f"ot2d_rmn{r}", (lambda r=r: P.orszag_tang(16, rmn=r)), R.MODE_RUN, 3) for r in range(4)],
    ("ot2d_ctw0", lambda: P.orszag_tang(16, ctw=0), R.MODE_RUN, 3),
    *[(f"ot2d_odr{o}", (lambda o=o: P.orszag_tang(16, odr=o, rk=min(o, 3))), R.MODE_RUN, 3) for o in (1, 2, 3)],
    ("ot2d_exec", lambda: P.orszag_tang(16, tmax=0.05), R.MODE_EXEC, 0),
    ("kh2d_mlau", lambda: P.kelvin_helmholtz(2, 16, mach=0.3, rmn=P.RMN_MLAU), R.MODE_RUN, 3),
    ("kh2d_roe_eta", _kh2_eta, R.MODE_DRUN, 3),
    ("wave3d_eta_ctw1", lambda: _wave3_eta(1, 0.02, 0.05), R.MODE_DRUN, 2),
    ("ot2d_profile_eta", lambda: P.localized_dissipation(P.orszag_tang(16), 0.01, 0.05, 0.5), R.MODE_DRUN, 3),
    ("kh3d_profile_eta", lambda: P.localized_dissipation(P.kelvin_helmholtz(3, 8, mach=0.3, rmn=P.RMN_HLLD),
                                                        0.01, 0.08, 0.3), R.MODE_DRUN, 2),
    ("wave3d_eta_ctw0_sub2", lambda: _wave3_eta(0, 0.05, 0.3, rmn=P.RMN_ROE), R.MODE_DRUN, 2),
    ("rt2d_lhlld", lambda: P.rayleigh_taylor(2, 16, 32), R.MODE_RUN, 3),
    ("rt2d_mlau_exec", lambda: P.rayleigh_taylor(2, 16, 32, rmn=P.RMN_MLAU, tmax=0.03), R.MODE_EXEC, 0),
    ("rt3d_hlld_ctw0", lambda: P.rayleigh_taylor(3, 8, 16, rmn=P.RMN_HLLD, ctw=0), R.MODE_RUN, 2),
    *[(f"kh3d_rmn{r}", (lambda r=r: P.kelvin_helmholtz(3, 6, mach=0.3, rmn=r)), R.MODE_RUN, 2) for r in range(4)],
    *[(f"wave{d}d_bc{s}", (lambda d=d, s=s: _wave_bc(d, s)), R.MODE_RUN, 2) for d in (1, 2, 3) for s in (1, 2)],
]


def make_kat_prim() -> None:
    """mhd_lrstate with the primitive reconstruction: the harness's ids 20..23 built against
    mhd_reconst (oracle/_ref/ref_kat_prim), stored as 24..27 (the oracle's ids for that form)."""
    inp = kat_inputs("lrstate_prim")
    exe = os.path.join(R.REF_DIR, "ref_kat_prim")
    outs = {f"f{f + 4}": R.run_kat(f, inp, 14, exe=exe) for f in (20, 21, 22, 23)}
    np.savez_compressed(os.path.join(OUT, "kat_lrstate_prim.npz"), input_sha=sha(inp), **outs)
    print("kat lrstate_prim", inp.shape)


def make_kat_char() -> None:
    """mhd_lrstate with the Athena-type reconstruction: the harness's ids 20..23 built against
    mhd_c_reconst (oracle/_ref/ref_kat_char), stored as 40..43 (the oracle's ids for that form)."""
    inp = kat_inputs("lrstate_char")
    exe = os.path.join(R.REF_DIR, "ref_kat_char")
    outs = {f"f{f + 20}": R.run_kat(f, inp, 14, exe=exe) for f in (20, 21, 22, 23)}
    np.savez_compressed(os.path.join(OUT, "kat_lrstate_char.npz"), input_sha=sha(inp), **outs)
    print("kat lrstate_char", inp.shape)


def make_kat(name: str) -> None:
    """One point-function fixture, kat_<name>.npz."""
    if name in ("lrstate_prim", "lrstate_char"):
        return make_kat_prim() if name == "lrstate_prim" else make_kat_char()
    funcs, nout = KAT_FUNCS[name]
    inp = kat_inputs(name)
    outs = {f"f{f}": R.run_kat(f, inp, nout) for f in funcs}
    np.savez_compressed(os.path.join(OUT, f"kat_{name}.npz"), input_sha=sha(inp), **outs)
    print("kat", name, inp.shape)


def add_steps(names) -> None:
    """Recompute the named step cases only, keeping the others of steps.npz."""
    path = os.path.join(OUT, "steps.npz")
    data = dict(np.load(path)) if os.path.exists(path) else {}
    for name, build, mode, nsteps in STEP_CASES:
        if name not in names:
            continue
        p = build()
        r = R.run_reference(p, mode, nsteps=nsteps, nthreads=4)
        data[f"{name}__state"] = r["state"]
        data[f"{name}__dts"] = r["dts"]
        data[f"{name}__meta"] = np.array([r["steps"], r["tim"], r["dt"]])
        data[f"{name}__insha"] = np.array(sha(p.state))
        print("step", name, p.nd, r["steps"])
    np.savez_compressed(path, **data)


def main() -> None:
    if len(sys.argv) > 2 and sys.argv[1] == "--kat":  # one fixture only
        make_kat(sys.argv[2])
        return
    if len(sys.argv) > 2 and sys.argv[1] == "--steps":  # some step cases only
        add_steps(sys.argv[2:])
        return
    for name, (funcs, nout) in KAT_FUNCS.items():
        if name in ("lrstate_prim", "lrstate_char"):
            continue
        inp = kat_inputs(name)
        outs = {f"f{f}": R.run_kat(f, inp, nout) for f in funcs}
        np.savez_compressed(os.path.join(OUT, f"kat_{name}.npz"), input_sha=sha(inp), **outs)
        print("kat", name, inp.shape)
    make_kat_prim()
    make_kat_char()
    data = {}
    for name, build, mode, nsteps in STEP_CASES:
        p = build()
        r = R.run_reference(p, mode, nsteps=nsteps, nthreads=4)
        data[f"{name}__state"] = r["state"]
        data[f"{name}__dts"] = r["dts"]
        data[f"{name}__meta"] = np.array([r["steps"], r["tim"], r["dt"]])
        data[f"{name}__insha"] = np.array(sha(p.state))
        print("step", name, p.nd, r["steps"])
    np.savez_compressed(os.path.join(OUT, "steps.npz"), **data)


if __name__ == "__main__":
    main()
