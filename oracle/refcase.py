"""Drivers for the CPU oracles (test infrastructure; never used by the product).

* ``run_reference``: writes a case file, runs the reference's own stepping code
  compiled from its sources (``oracle/_ref/ref{1,2,3}d*``, built by
  ``oracle/Makefile`` with the reference flags -O2 -fopenmp) and reads back
  the state and the dt sequence.
* ``run_kat``: point-function known answers from ``oracle/_ref/ref_kat``.
* ``run_reference_dual``: the reference's 2D stepping code built with a
  forward-mode dual number for double (``oracle/_ref/ref2d_dual_ctw*``): final
  state and its directional derivative for a given tangent, dt held fixed.
* ``Restatement``: ctypes binding of ``oracle/liboracle_qas.so``, our plain-C
  restatement of the same algorithm (``oracle/qas_oracle.c``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(HERE, "liboracle_qas.so")

MODE_STEP, MODE_RUN, MODE_EXEC, MODE_DRUN, MODE_DSTEP, MODE_IO, MODE_IOLOAD = 0, 1, 2, 3, 4, 5, 6

_HDR = struct.Struct("<15i12d24i")
_RES = struct.Struct("<4i4d")
MAGIC_IN = 0x31534151
MAGIC_OUT = 0x32534151


def ref_binary(dim: int, ctw: int, gravity=False) -> str:
    """The reference build for a case: ref1d, ref{2,3}d_ctw*, the gravity drivers
    (2D/SERIAL/RTI, 3D/MPI/RTI) ref{2,3}d_g_ctw* (gravity=True), the Hall driver ref1d_hall
    (gravity="hall"), the primitive-reconstruction builds ref1d_prim / ref{2,3}d_prim_ctw1
    (gravity="prim") or the Athena-type reconstruction builds ref1d_char / ref{2,3}d_char_ctw1
    (gravity="char")."""
    if gravity in ("prim", "char"):
        name = f"ref1d_{gravity}" if dim == 1 else f"ref{dim}d_{gravity}_ctw{int(bool(ctw))}"
    elif dim == 1:
        name = "ref1d_hall" if gravity == "hall" else "ref1d"
    else:
        name = f"ref{dim}d_{'g_' if gravity else ''}ctw{int(bool(ctw))}"
    return os.path.join(REF_DIR, name)


def reference_available(dim: int = 2, ctw: int = 1, gravity: bool = False) -> bool:
    return os.access(ref_binary(dim, ctw, gravity), os.X_OK)


def host_isa_level() -> str:
    """x86-64 ISA level of this host for the -O3 timing builds: "v4" with AVX-512 (F, BW, CD,
    DQ, VL), else "v3" with AVX2 + FMA + BMI2, else "" (no such build runs here)."""
    try:
        flags = set()
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        return ""
    if {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags:
        return "v4"
    if {"avx2", "fma", "bmi2", "movbe"} <= flags:
        return "v3"
    return ""


def o3_binary(dim: int) -> Optional[str]:
    """The reference built with -O3 -march=<this host's ISA level> -fopenmp (CTW=1; timing
    only), or None when there is none for this host."""
    lvl = host_isa_level()
    if not lvl or dim not in (2, 3):
        return None
    exe = os.path.join(REF_DIR, f"ref{dim}d_o3{lvl}_ctw1")
    return exe if os.access(exe, os.X_OK) else None


def _nu_eta(prob):
    nu, eta = getattr(prob, "nu_arr", None), getattr(prob, "eta_arr", None)
    if nu is None and eta is None:
        return None
    z = np.zeros(prob.nd)
    return (np.ascontiguousarray(z if nu is None else nu, dtype=np.float64).reshape(-1),
            np.ascontiguousarray(z if eta is None else eta, dtype=np.float64).reshape(-1))


def _phi(prob) -> Optional[np.ndarray]:
    phi = getattr(prob, "phi", None)
    return None if phi is None else np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)


def write_case(path: str, prob, mode: int, nsteps: int = 0, dt: float = 0.0, nthreads: int = 0,
               state: Optional[np.ndarray] = None) -> None:
    st = prob.state if state is None else state
    st = np.ascontiguousarray(st, dtype=np.float64).reshape(8, -1)
    assert st.shape[1] == prob.nd, (st.shape, prob.nd)
    phi = _phi(prob)
    nue = _nu_eta(prob)
    flags = (0 if phi is None else 1) | (0 if nue is None else 2)
    hdr = _HDR.pack(MAGIC_IN, prob.dim, prob.nxm, prob.nym, prob.nzm,
                    prob.rmn, prob.odr, prob.rk, prob.ctw,
                    mode, nsteps, prob.flg, nthreads, prob.nout, flags,
                    prob.gam, prob.cfl, prob.dtrec, dt,
                    prob.xmin, prob.xmax, prob.ymin, prob.ymax, prob.zmin, prob.zmax,
                    # the Hall build reads (di, de) from the (nu0, eta0) fields
                    *((prob.di, prob.de) if getattr(prob, "hall", False) else (prob.nu0, prob.eta0)),
                    *[int(v) for v in prob.dnx], *[int(v) for v in prob.dny], *[int(v) for v in prob.dnz])
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(st.tobytes())
        if phi is not None:
            assert phi.size == prob.nd
            f.write(phi.tobytes())
        if nue is not None:
            f.write(nue[0].tobytes())
            f.write(nue[1].tobytes())


def read_result(path: str, prob):
    with open(path, "rb") as f:
        raw = f.read()
    magic, steps, ndt, nd, tim, dt, elapsed, _ = _RES.unpack_from(raw, 0)
    assert magic == MAGIC_OUT
    off = _RES.size
    dts = np.frombuffer(raw, dtype=np.float64, count=ndt, offset=off).copy()
    off += 8 * ndt
    st = np.frombuffer(raw, dtype=np.float64, count=8 * nd, offset=off).copy()
    st = st.reshape(8, prob.nz, prob.ny, prob.nx)
    off += 8 * 8 * nd
    step_times = np.zeros(0)
    if off + 4 <= len(raw):
        (nt,) = struct.unpack_from("<i", raw, off)
        step_times = np.frombuffer(raw, dtype=np.float64, count=nt, offset=off + 4).copy()
    return {"state": st, "dts": dts, "steps": steps, "tim": tim, "dt": dt, "elapsed": elapsed,
            "step_times": step_times}


def run_reference(prob, mode: int = MODE_RUN, nsteps: int = 1, dt: float = 0.0, nthreads: int = 0,
                  state: Optional[np.ndarray] = None, timeout: float = 3600.0, exe: Optional[str] = None,
                  bind: bool = False):
    """Run the reference's own code on ``prob`` and return its result dict (``exe``: another
    build of the same driver, e.g. o3_binary(), for timing; ``bind``: pin the OpenMP threads
    to consecutive cores, OMP_PROC_BIND=close OMP_PLACES=cores)."""
    if getattr(prob, "char_mode", 0):
        variant = "prim" if prob.char_mode == 1 else "char"
    elif getattr(prob, "hall", False):
        variant = "hall"
    else:
        variant = _phi(prob) is not None
    exe = exe or ref_binary(prob.dim, prob.ctw, variant)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"reference oracle binary missing: {exe} (build with `make -C oracle ref`)")
    with tempfile.TemporaryDirectory(prefix="qasref_") as td:
        cin = os.path.join(td, "case.bin")
        cout = os.path.join(td, "result.bin")
        write_case(cin, prob, mode, nsteps=nsteps, dt=dt, nthreads=nthreads, state=state)
        env = dict(os.environ)
        if nthreads > 0:
            env["OMP_NUM_THREADS"] = str(nthreads)
        if bind:
            env["OMP_PROC_BIND"] = "close"
            env["OMP_PLACES"] = "cores"
        subprocess.run([exe, cin, cout], check=True, env=env, timeout=timeout,
                       stdout=subprocess.DEVNULL)
        return read_result(cout, prob)


def reference_io(prob, directory: str, state: Optional[np.ndarray] = None, load: bool = False, n: int = 0,
                 cnt: int = 0, tim: float = 0.0, dt: float = 0.0, trec: float = 0.0):
    """The reference's own dout_ + bkup_save of `state` into `directory` (load=False), or its
    bkup_load from there (load=True: returns (state, (n, cnt, tim, dt, trec)))."""
    exe = ref_binary(prob.dim, prob.ctw)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"reference oracle binary missing: {exe}")
    import copy
    p = copy.copy(prob)
    p.cfl, p.dtrec = float(dt), float(trec)
    with tempfile.TemporaryDirectory(prefix="qasrefio_") as td:
        cin = os.path.join(td, "case.bin")
        cout = os.path.join(td, "result.bin")
        write_case(cin, p, MODE_IOLOAD if load else MODE_IO, nsteps=int(n), dt=float(tim), state=state)
        # cnt travels in the flg field
        raw = bytearray(open(cin, "rb").read())
        struct.pack_into("<i", raw, 4 * 11, int(cnt))
        open(cin, "wb").write(bytes(raw))
        subprocess.run([exe, cin, cout, directory], check=True, stdout=subprocess.DEVNULL)
        res = read_result(cout, prob)
    if not load:
        return None
    with open(os.path.join(directory, "loaded.txt")) as f:
        t = f.read().split()
    return res["state"], (int(t[0]), int(t[1]), float(t[2]), float(t[3]), float(t[4]))


def dual_binary(ctw: int) -> str:
    return os.path.join(REF_DIR, f"ref2d_dual_ctw{int(bool(ctw))}")


def run_reference_dual(prob, state: np.ndarray, tangent: np.ndarray, dts, eta0: float = 0.0, deta: float = 0.0,
                       nthreads: int = 0, timeout: float = 3600.0):
    """Tangent-linear run of the reference's 2D code (bound, ideal, sub-cycled dsptv with
    uniform eta0 and nu = 0 when eta0 > 0) with the given dt per step.  Returns
    (final state, d(final state)) for the initial tangent (state direction, deta)."""
    exe = dual_binary(prob.ctw)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"reference dual binary missing: {exe} (build with `make -C oracle ref`)")
    if prob.dim != 2:
        raise ValueError("the dual build covers the 2D driver")
    st = np.ascontiguousarray(state, dtype=np.float64).reshape(8, -1)
    tg = np.ascontiguousarray(tangent, dtype=np.float64).reshape(8, -1)
    d = np.ascontiguousarray(dts, dtype=np.float64)
    hdr = struct.pack("<10i7d16i", 0x44534151, prob.nxm, prob.nym, prob.rmn, prob.odr, prob.rk, int(bool(prob.ctw)),
                      d.size, nthreads, 0, prob.gam, prob.xmin, prob.xmax, prob.ymin, prob.ymax, float(eta0),
                      float(deta), *[int(x) for x in prob.dnx], *[int(x) for x in prob.dny])
    with tempfile.TemporaryDirectory(prefix="qasdual_") as td:
        cin = os.path.join(td, "case.bin")
        cout = os.path.join(td, "result.bin")
        with open(cin, "wb") as f:
            f.write(hdr)
            f.write(d.tobytes())
            f.write(st.tobytes())
            f.write(tg.tobytes())
        env = dict(os.environ)
        if nthreads > 0:
            env["OMP_NUM_THREADS"] = str(nthreads)
        subprocess.run([exe, cin, cout], check=True, env=env, timeout=timeout, stdout=subprocess.DEVNULL)
        out = np.fromfile(cout, dtype=np.float64).reshape(2, 8, -1)
    return out[0], out[1]


def run_kat(func: int, inputs: np.ndarray, nout: int, exe: Optional[str] = None) -> np.ndarray:
    """Known answers of the reference's point function `func` (``ref_kat``; ``exe``: another
    build of the same harness, e.g. ``ref_kat_prim`` with mhd_lrstate's primitive reconstruction)."""
    exe = exe or os.path.join(REF_DIR, "ref_kat")
    inputs = np.ascontiguousarray(inputs, dtype=np.float64)
    ncase, nin = inputs.shape
    with tempfile.TemporaryDirectory(prefix="qaskat_") as td:
        cin = os.path.join(td, "in.bin")
        cout = os.path.join(td, "out.bin")
        with open(cin, "wb") as f:
            f.write(struct.pack("<4i", func, ncase, nin, nout))
            f.write(inputs.tobytes())
        subprocess.run([exe, cin, cout], check=True, stdout=subprocess.DEVNULL)
        return np.fromfile(cout, dtype=np.float64).reshape(ncase, nout)


# ---------------------------------------------------------------------------
# ctypes binding of the plain-C restatement
# ---------------------------------------------------------------------------

class _OGrid(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("nxm", ctypes.c_int), ("nym", ctypes.c_int),
                ("nzm", ctypes.c_int), ("rmn", ctypes.c_int), ("odr", ctypes.c_int),
                ("rk", ctypes.c_int), ("ctw", ctypes.c_int),
                ("gam", ctypes.c_double), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("dz", ctypes.c_double),
                ("dnx", ctypes.c_int * 8), ("dny", ctypes.c_int * 8), ("dnz", ctypes.c_int * 8),
                ("phi", ctypes.POINTER(ctypes.c_double)), ("hall_de", ctypes.c_double),
                ("nu", ctypes.POINTER(ctypes.c_double)), ("eta", ctypes.POINTER(ctypes.c_double)),
                ("char_mode", ctypes.c_int)]


class Restatement:
    """The plain-C oracle (oracle/qas_oracle.c) driven through ctypes."""

    def __init__(self, path: str = LIB_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing (build with `make -C oracle oracle`)")
        self.lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        self.lib.qo_step.argtypes = [ctypes.POINTER(_OGrid), dp, ctypes.c_double]
        self.lib.qo_step.restype = ctypes.c_int
        self.lib.qo_bound.argtypes = [ctypes.POINTER(_OGrid), dp]
        self.lib.qo_bound.restype = None
        self.lib.qo_cfl_dt.argtypes = [ctypes.POINTER(_OGrid), dp, ctypes.c_double]
        self.lib.qo_cfl_dt.restype = ctypes.c_double
        self.lib.qo_dissipate.argtypes = [ctypes.POINTER(_OGrid), dp, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double]
        self.lib.qo_dissipate.restype = ctypes.c_int
        self.lib.qo_dsptv.argtypes = [ctypes.POINTER(_OGrid), dp, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double]
        self.lib.qo_dsptv.restype = ctypes.c_int
        self.lib.qo_kat.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
        self.lib.qo_hall.argtypes = [ctypes.POINTER(_OGrid), dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        self.lib.qo_hall.restype = ctypes.c_int
        self.lib.qo_haldt.argtypes = [ctypes.POINTER(_OGrid), dp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        self.lib.qo_haldt.restype = ctypes.c_double
        self.lib.qo_kat.restype = ctypes.c_int

    @staticmethod
    def grid(prob) -> _OGrid:
        g = _OGrid()
        g.dim, g.nxm, g.nym, g.nzm = prob.dim, prob.nxm, prob.nym, prob.nzm
        g.rmn, g.odr, g.rk, g.ctw = prob.rmn, prob.odr, prob.rk, prob.ctw
        g.gam, g.dx = prob.gam, prob.dx
        g.dy = prob.dy if prob.dim >= 2 else 0.0
        g.dz = prob.dz if prob.dim >= 3 else 0.0
        for m in range(8):
            g.dnx[m], g.dny[m], g.dnz[m] = int(prob.dnx[m]), int(prob.dny[m]), int(prob.dnz[m])
        g.char_mode = int(getattr(prob, "char_mode", 0))
        if getattr(prob, "hall", False):
            g.hall_de = float(prob.de)
        nue = _nu_eta(prob)
        if nue is not None:
            g._nue_keep = nue
            g.nu = nue[0].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            g.eta = nue[1].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        phi = _phi(prob)
        if phi is not None:
            g._phi_keep = phi  # the pointer below must outlive the call
            g.phi = phi.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        return g

    @staticmethod
    def _ptr(a: np.ndarray):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def dr(self, prob) -> float:
        d = [prob.dx]
        if prob.dim >= 2:
            d.append(prob.dy)
        if prob.dim >= 3:
            d.append(prob.dz)
        r = d[0]
        for v in d[1:]:
            r = v if r >= v else r   # min() of common/common_func.h:11-15
        return r

    def run(self, prob, nsteps: int, state: Optional[np.ndarray] = None, mode: int = MODE_RUN,
            dt: float = 0.0):
        """Same semantics as :func:`run_reference` for MODE_STEP/RUN/EXEC/DRUN/DSTEP."""
        g = self.grid(prob)
        st = np.ascontiguousarray((prob.state if state is None else state), dtype=np.float64).copy()
        p = self._ptr(st)
        dts = []
        dr = self.dr(prob)
        if mode == MODE_STEP:
            self.lib.qo_bound(ctypes.byref(g), p)
            rc = self.lib.qo_step(ctypes.byref(g), p, dt)
            assert rc == 0
            return {"state": st, "dts": np.array([dt]), "steps": 1, "tim": dt, "dt": dt}
        hall = getattr(prob, "hall", False)
        if hall:
            from qasmhd_b200.problems import hall_vphix
            vphix = hall_vphix(prob)
        if mode == MODE_DSTEP and hall:  # the Hall build's DSTEP: bound; one hall_(dt)
            self.lib.qo_bound(ctypes.byref(g), p)
            rc = self.lib.qo_hall(ctypes.byref(g), p, dt, prob.di, vphix)
            assert rc == 0
            return {"state": st, "dts": np.array([dt]), "steps": 1, "tim": dt, "dt": dt}
        if mode == MODE_DSTEP:
            self.lib.qo_bound(ctypes.byref(g), p)
            rc = self.lib.qo_dsptv(ctypes.byref(g), p, dt, prob.nu0, prob.eta0)
            assert rc == 0
            return {"state": st, "dts": np.array([dt]), "steps": 1, "tim": dt, "dt": dt}
        # setdt(1): CFL dt and nmax from the first dt (mhd2d_class.cpp:11-33)
        vmax = self.lib.qo_cfl_dt(ctypes.byref(g), p, 1.0)
        dt = prob.cfl * (dr if prob.dim > 1 else prob.dx) / vmax
        if prob.dim == 1:
            nrec = int(prob.dtrec / dt + 0.5)
            nmax = nrec * prob.nout
        else:
            nmax = int(prob.tmax / dt + 0.5)
        tim = 0.0
        n = 0
        steps = 0

        def one(n_now):
            nonlocal tim, dt
            tim += dt
            dts.append(dt)
            self.lib.qo_bound(ctypes.byref(g), p)
            if hall and prob.di != 0:  # Hall sub-cycles of HMHD1D::exec_ (hmhd1d_class.cpp:26-33)
                hmax = 1 + int(dt / self.lib.qo_haldt(ctypes.byref(g), p, prob.cfl, prob.di, vphix))
                for _ in range(hmax):
                    assert self.lib.qo_hall(ctypes.byref(g), p, dt / hmax, prob.di, vphix) == 0
                    self.lib.qo_bound(ctypes.byref(g), p)
            rc = self.lib.qo_step(ctypes.byref(g), p, dt)
            assert rc == 0
            if mode == MODE_DRUN:
                rc = self.lib.qo_dissipate(ctypes.byref(g), p, dt, prob.nu0, prob.eta0)
                assert rc == 0
            if prob.flg * (n_now % 2 == 0):
                vm = self.lib.qo_cfl_dt(ctypes.byref(g), p, 1.0)
                dt = prob.cfl * (dr if prob.dim > 1 else prob.dx) / vm

        if mode in (MODE_RUN, MODE_DRUN):
            for _ in range(nsteps):
                n += 1
                one(n)
                steps += 1
        elif mode == MODE_EXEC:
            while True:
                cond = (n < nmax and tim < prob.tmax) if (prob.flg or prob.dim > 1) else (n < nmax)
                n += 1
                if not cond:
                    break
                one(n)
                steps += 1
        else:
            raise ValueError(mode)
        return {"state": st, "dts": np.array(dts), "steps": steps, "tim": tim, "dt": dt}

    def kat(self, func: int, inputs: np.ndarray, nout: int) -> np.ndarray:
        inputs = np.ascontiguousarray(inputs, dtype=np.float64)
        ncase, nin = inputs.shape
        out = np.zeros((ncase, nout), dtype=np.float64)
        rc = self.lib.qo_kat(func, ncase, nin, nout, self._ptr(inputs), self._ptr(out))
        assert rc == 0, f"qo_kat({func}) failed"
        return out
