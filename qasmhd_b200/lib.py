"""ctypes binding of libqas.so (include/qas.h).

The shared library is built in-tree (``qasmhd_b200/libqas.so``) by
:func:`qasmhd_b200.build.build_library`.  Loading fails loudly when it is
missing: there is no CPU fallback for the product path.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# QASMHD_LIB: path of another build of the library (e.g. one compiled with other tuning macros)
LIB_PATH = os.environ.get("QASMHD_LIB") or os.path.join(HERE, "libqas.so")

# qas_status values
QAS_OK = 0
QAS_ERR_INVALID = 1
QAS_ERR_CUDA = 2
QAS_ERR_NOMEM = 3
QAS_ERR_NONFINITE = 4
QAS_ERR_TIMEOUT = 5
QAS_ERR_UNSUPPORTED = 6
QAS_ERR_NO_DEVICE = 7
QAS_ERR_IO = 8
QAS_ERR_HOST = 9

# every exported entry point of include/qas.h (checked by the CPU tests)
EXPORTS = (
    "qas_status_str", "qas_abi_version", "qas_last_cuda_error", "qas_create", "qas_destroy",
    "qas_cells", "qas_upload", "qas_download", "qas_upload_block", "qas_download_block",
    "qas_upload_block_async", "qas_download_block_async",
    "qas_device_state", "qas_stream", "qas_bound", "qas_step", "qas_cfl_vmax", "qas_cfl_dt",
    "qas_run", "qas_run_reset", "qas_step_host", "qas_pipe_plan", "qas_dissipate", "qas_dsptv", "qas_max_divb", "qas_sync",
    "qas_kernel_launches", "qas_bc_map", "qas_profile_run", "qas_set_option", "qas_set_tile",
    "qas_get_tile", "qas_autotune", "qas_batch_create", "qas_batch_destroy", "qas_batch_cells",
    "qas_batch_upload", "qas_batch_download", "qas_batch_run", "qas_batch_set_tile", "qas_batch_autotune",
    "qas_batch_stream", "qas_batch_kernel_launches", "qas_fp64_peak", "qas_adjoint_forward", "qas_adjoint_run",
    "qas_adjoint_backward", "qas_max_divb_noalloc", "qas_dout", "qas_dout_wait", "qas_bkup_save",
    "qas_bkup_load", "qas_dd_plan", "qas_dd_create", "qas_dd_destroy", "qas_dd_upload_block",
    "qas_dd_download_block", "qas_dd_run", "qas_dd_parts", "qas_dd_kernel_launches", "qas_set_gravity",
    "qas_set_hall", "qas_hall", "qas_set_dissipation", "qas_primitives",
)
QAS_OPT_FUSED_SWEEP = 1
QAS_OPT_LR_STAGING = 2
QAS_OPT_PIPE_ITEMS = 3
QAS_OPT_PIPE_LANES = 4
QAS_OPT_TEST_TMA_STALL = 5


class QasError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = status
        msg = f"{what}: qas status {status}"
        if _lib is not None:
            msg += f" ({_lib.qas_status_str(status).decode()})"
        if detail:
            msg += f" [{detail}]"
        super().__init__(msg)


class Grid(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("nxm", ctypes.c_int), ("nym", ctypes.c_int), ("nzm", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("gam", ctypes.c_double)]


ABI_VERSION = 2  # the layout of the structs below; qas_abi_version() of a matching libqas.so


class Scheme(ctypes.Structure):
    _fields_ = [("rmn", ctypes.c_int), ("odr", ctypes.c_int), ("rk", ctypes.c_int), ("ctw", ctypes.c_int),
                ("char_mode", ctypes.c_int)]


class BC(ctypes.Structure):
    _fields_ = [("dnx", ctypes.c_int * 8), ("dny", ctypes.c_int * 8), ("dnz", ctypes.c_int * 8)]


class RunOpts(ctypes.Structure):
    _fields_ = [("max_steps", ctypes.c_int), ("flg", ctypes.c_int), ("stop_rule", ctypes.c_int),
                ("cfl", ctypes.c_double), ("dtrec", ctypes.c_double), ("nout", ctypes.c_int),
                ("use_graph", ctypes.c_int), ("nu0", ctypes.c_double), ("eta0", ctypes.c_double)]


class KernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_longlong), ("total_ms", ctypes.c_double)]


class DdCopy(ctypes.Structure):
    _fields_ = [("part", ctypes.c_int), ("src_part", ctypes.c_int), ("src_plane", ctypes.c_int),
                ("dst_plane", ctypes.c_int), ("nplanes", ctypes.c_int)]


class RunInfo(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int), ("n", ctypes.c_int), ("nmax", ctypes.c_int),
                ("tim", ctypes.c_double), ("dt", ctypes.c_double)]


_lib: Optional[ctypes.CDLL] = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libqas.so (once) and declare the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m qasmhd_b200.build` "
                                "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    st = ctypes.c_int
    lib.qas_status_str.argtypes = [st]
    lib.qas_status_str.restype = ctypes.c_char_p
    lib.qas_abi_version.restype = ctypes.c_int
    lib.qas_last_cuda_error.restype = ctypes.c_char_p
    lib.qas_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(Grid), ctypes.POINTER(Scheme),
                               ctypes.POINTER(BC), ctypes.c_int]
    lib.qas_destroy.argtypes = [vp]
    lib.qas_cells.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.qas_upload.argtypes = [vp, ctypes.POINTER(dp)]
    lib.qas_download.argtypes = [vp, ctypes.POINTER(dp)]
    lib.qas_upload_block.argtypes = [vp, dp]
    lib.qas_download_block.argtypes = [vp, dp]
    lib.qas_upload_block_async.argtypes = [vp, dp]
    lib.qas_download_block_async.argtypes = [vp, dp]
    lib.qas_device_state.argtypes = [vp, ctypes.POINTER(dp)]
    lib.qas_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.qas_bound.argtypes = [vp]
    lib.qas_step.argtypes = [vp, ctypes.c_double]
    lib.qas_cfl_vmax.argtypes = [vp, dp]
    lib.qas_cfl_dt.argtypes = [vp, ctypes.c_double, dp]
    lib.qas_run.argtypes = [vp, ctypes.POINTER(RunOpts), ctypes.POINTER(RunInfo)]
    lib.qas_run_reset.argtypes = [vp]
    lib.qas_step_host.argtypes = [vp, dp, dp, ctypes.POINTER(RunOpts), ctypes.POINTER(RunInfo)]
    ipp = ctypes.POINTER(ctypes.c_int)
    lib.qas_pipe_plan.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ipp, ctypes.c_int, ipp, ipp]
    lib.qas_dissipate.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.qas_dsptv.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.qas_max_divb.argtypes = [vp, dp]
    lib.qas_sync.argtypes = [vp]
    lib.qas_kernel_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.qas_profile_run.argtypes = [vp, ctypes.POINTER(RunOpts), ctypes.c_int, ctypes.POINTER(KernelTime),
                                    ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.qas_set_option.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.qas_set_tile.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.qas_get_tile.argtypes = [vp, ctypes.c_char_p] + [ctypes.POINTER(ctypes.c_int)] * 3
    lib.qas_autotune.argtypes = [vp, ctypes.c_int]
    lib.qas_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(Grid), ctypes.POINTER(Scheme),
                                     ctypes.POINTER(BC), ctypes.c_int]
    lib.qas_batch_destroy.argtypes = [vp]
    lib.qas_batch_cells.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    lib.qas_batch_upload.argtypes = [vp, ctypes.c_int, dp]
    lib.qas_batch_download.argtypes = [vp, ctypes.c_int, dp]
    lib.qas_batch_run.argtypes = [vp, ctypes.POINTER(RunOpts), ctypes.POINTER(RunInfo)]
    lib.qas_batch_set_tile.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.qas_batch_autotune.argtypes = [vp, ctypes.c_int]
    lib.qas_batch_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.qas_batch_kernel_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.qas_fp64_peak.argtypes = [dp]
    lib.qas_adjoint_forward.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_double]
    lib.qas_adjoint_backward.argtypes = [vp, dp, dp, dp]
    lib.qas_adjoint_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_double, dp, dp, dp]
    lib.qas_dout.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                             ctypes.POINTER(dp)]
    lib.qas_dout_wait.argtypes = [vp]
    lib.qas_bkup_save.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int]
    ip = ctypes.POINTER(ctypes.c_int)
    lib.qas_bkup_load.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ip, ip, ip, dp, dp, dp]
    lib.qas_max_divb_noalloc.argtypes = [ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                                         ctypes.c_void_p, dp]
    lib.qas_bc_map.argtypes = [ctypes.POINTER(Grid), ctypes.POINTER(BC), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.POINTER(ctypes.c_int), dp, ctypes.c_int]
    ip = ctypes.POINTER(ctypes.c_int)
    lib.qas_dd_plan.argtypes = [ctypes.POINTER(Grid), ctypes.POINTER(BC), ctypes.c_int, ip, ctypes.POINTER(DdCopy),
                                ctypes.c_int, ip]
    lib.qas_dd_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(Grid), ctypes.POINTER(Scheme),
                                  ctypes.POINTER(BC), ctypes.c_int, ip]
    lib.qas_dd_destroy.argtypes = [vp]
    lib.qas_set_gravity.argtypes = [vp, dp]
    lib.qas_set_hall.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    lib.qas_set_dissipation.argtypes = [vp, dp, dp]
    lib.qas_primitives.argtypes = [vp, ctypes.POINTER(dp), ctypes.POINTER(dp)]
    lib.qas_hall.argtypes = [vp, ctypes.c_double]
    lib.qas_dd_upload_block.argtypes = [vp, dp]
    lib.qas_dd_download_block.argtypes = [vp, dp]
    lib.qas_dd_run.argtypes = [vp, ctypes.POINTER(RunOpts), ctypes.POINTER(RunInfo)]
    lib.qas_dd_parts.argtypes = [vp, ip]
    lib.qas_dd_kernel_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    for name in EXPORTS:
        if name not in ("qas_status_str", "qas_abi_version", "qas_last_cuda_error"):
            getattr(lib, name).restype = ctypes.c_int
    if lib.qas_abi_version() != ABI_VERSION:
        raise ImportError(f"{path} has ABI version {lib.qas_abi_version()}, the binding expects "
                          f"{ABI_VERSION}: rebuild it with `python -m qasmhd_b200.build`")
    _lib = lib
    return lib


def _check(status: int, what: str) -> None:
    if status != QAS_OK:
        detail = ""
        if status in (QAS_ERR_CUDA, QAS_ERR_NOMEM, QAS_ERR_IO, QAS_ERR_HOST) and _lib is not None:
            detail = _lib.qas_last_cuda_error().decode()
        raise QasError(status, what, detail)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Context:
    """One device simulation: a qas_ctx handle with numpy-friendly calls."""

    def __init__(self, dim: int, nxm: int, nym: int, nzm: int, dx: float, dy: float, dz: float, gam: float,
                 rmn: int, odr: int, rk: int, ctw: int, dnx: Sequence[int], dny: Sequence[int],
                 dnz: Sequence[int], device: int = -1, char_mode: int = 0):
        self.lib = load()
        g = Grid(dim, nxm, nym if dim >= 2 else 1, nzm if dim >= 3 else 1, dx, dy if dim >= 2 else 0.0,
                 dz if dim >= 3 else 0.0, gam)
        s = Scheme(rmn, odr, rk, ctw, char_mode)
        b = BC()
        for m in range(8):
            b.dnx[m], b.dny[m], b.dnz[m] = int(dnx[m]), int(dny[m]), int(dnz[m])
        h = ctypes.c_void_p()
        _check(self.lib.qas_create(ctypes.byref(h), ctypes.byref(g), ctypes.byref(s), ctypes.byref(b), device),
               "qas_create")
        self.h = h
        nd = ctypes.c_longlong()
        _check(self.lib.qas_cells(self.h, ctypes.byref(nd)), "qas_cells")
        self.nd = int(nd.value)
        self.dim = dim

    @classmethod
    def from_problem(cls, prob, device: int = -1) -> "Context":
        """A context for the problem; with gravity (prob.phi) the gravity form is switched on."""
        ctx = cls(prob.dim, prob.nxm, prob.nym, prob.nzm, prob.dx, prob.dy if prob.dim >= 2 else 0.0,
                  prob.dz if prob.dim >= 3 else 0.0, prob.gam, prob.rmn, prob.odr, prob.rk, prob.ctw,
                  prob.dnx, prob.dny, prob.dnz, device, getattr(prob, "char_mode", 0))
        if getattr(prob, "phi", None) is not None:
            ctx.set_gravity(prob.phi)
        if getattr(prob, "hall", False):
            ctx.set_hall(prob.di, prob.de)
        if getattr(prob, "nu_arr", None) is not None or getattr(prob, "eta_arr", None) is not None:
            ctx.set_dissipation(prob.nu_arr, prob.eta_arr)
        return ctx

    def primitives(self, shape) -> dict:
        """qas_primitives: vx, vy, vz, pr, cx, cy, cz of the current state (arrays of `shape`)."""
        dp = ctypes.POINTER(ctypes.c_double)
        out = {k: np.empty(shape, dtype=np.float64) for k in ("vx", "vy", "vz", "pr", "cx", "cy", "cz")}
        prim = (dp * 4)(*[_dptr(out[k]) for k in ("vx", "vy", "vz", "pr")])
        cc = (dp * 3)(*[_dptr(out[k]) for k in ("cx", "cy", "cz")])
        _check(self.lib.qas_primitives(self.h, prim, cc), "qas_primitives")
        return out

    def set_dissipation(self, nu: Optional[np.ndarray], eta: Optional[np.ndarray]) -> None:
        """qas_set_dissipation: per-cell viscosity / resistivity profiles (None = zero; both None
        removes them)."""
        def arr(a):
            if a is None:
                return None, None
            b = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
            if b.size != self.nd:
                raise ValueError(f"profile has {b.size} values, the grid {self.nd}")
            return b, _dptr(b)
        kn, pn = arr(nu)
        ke, pe = arr(eta)
        _check(self.lib.qas_set_dissipation(self.h, pn, pe), "qas_set_dissipation")

    def set_hall(self, di: float, de: float = 0.0) -> None:
        """qas_set_hall: the Hall form of the 1D driver (ion / electron inertia lengths)."""
        _check(self.lib.qas_set_hall(self.h, float(di), float(de)), "qas_set_hall")

    def hall(self, dt: float) -> None:
        """qas_hall: one hall_(dt) call."""
        _check(self.lib.qas_hall(self.h, float(dt)), "qas_hall")

    def set_gravity(self, phi: Optional[np.ndarray]) -> None:
        """qas_set_gravity: the gravitational potential of every padded cell, or None (off)."""
        if phi is None:
            _check(self.lib.qas_set_gravity(self.h, None), "qas_set_gravity")
            return
        a = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
        if a.size != self.nd:
            raise ValueError(f"phi has {a.size} values, the grid {self.nd}")
        _check(self.lib.qas_set_gravity(self.h, _dptr(a)), "qas_set_gravity")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.qas_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # state transfer -------------------------------------------------------
    def upload(self, state: np.ndarray) -> None:
        st = np.ascontiguousarray(state, dtype=np.float64).reshape(8, -1)
        assert st.shape[1] == self.nd, (st.shape, self.nd)
        _check(self.lib.qas_upload_block(self.h, _dptr(st)), "qas_upload_block")

    def download(self, shape=None) -> np.ndarray:
        out = np.empty((8, self.nd), dtype=np.float64)
        _check(self.lib.qas_download_block(self.h, _dptr(out)), "qas_download_block")
        return out if shape is None else out.reshape(shape)

    def download_into(self, out: np.ndarray) -> None:
        """Download into a caller-owned C-contiguous float64 buffer of 8*nd values (e.g. pinned)."""
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and out.size == 8 * self.nd
        _check(self.lib.qas_download_block(self.h, _dptr(out)), "qas_download_block")

    def upload_async(self, state: np.ndarray) -> None:
        """Queue the upload of a C-contiguous float64 block of 8*nd values (best pinned) on the
        context's stream; `state` must stay alive and unchanged until sync()."""
        assert state.dtype == np.float64 and state.flags["C_CONTIGUOUS"] and state.size == 8 * self.nd
        _check(self.lib.qas_upload_block_async(self.h, _dptr(state)), "qas_upload_block_async")

    def download_async(self, out: np.ndarray) -> None:
        """Queue the download of the state into `out` (8*nd float64 values, best pinned); the
        values are there after sync()."""
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and out.size == 8 * self.nd
        _check(self.lib.qas_download_block_async(self.h, _dptr(out)), "qas_download_block_async")

    def upload_fields(self, fields: Sequence[np.ndarray]) -> None:
        """Upload 8 separate host arrays (the reference's val[8] pointers)."""
        arrs = [np.ascontiguousarray(f, dtype=np.float64).reshape(-1) for f in fields]
        ptrs = (ctypes.POINTER(ctypes.c_double) * 8)(*[_dptr(a) for a in arrs])
        _check(self.lib.qas_upload(self.h, ptrs), "qas_upload")

    def download_fields(self, fields: Sequence[np.ndarray]) -> None:
        for f in fields:
            assert f.flags["C_CONTIGUOUS"] and f.dtype == np.float64 and f.size == self.nd
        ptrs = (ctypes.POINTER(ctypes.c_double) * 8)(*[_dptr(f) for f in fields])
        _check(self.lib.qas_download(self.h, ptrs), "qas_download")

    # stepping --------------------------------------------------------------
    def bound(self) -> None:
        _check(self.lib.qas_bound(self.h), "qas_bound")

    def step(self, dt: float) -> None:
        _check(self.lib.qas_step(self.h, float(dt)), "qas_step")

    def cfl_vmax(self) -> float:
        v = ctypes.c_double()
        _check(self.lib.qas_cfl_vmax(self.h, ctypes.byref(v)), "qas_cfl_vmax")
        return v.value

    def cfl_dt(self, cfl: float) -> float:
        v = ctypes.c_double()
        _check(self.lib.qas_cfl_dt(self.h, float(cfl), ctypes.byref(v)), "qas_cfl_dt")
        return v.value

    def run(self, max_steps: int = 0, flg: int = 1, stop_rule: int = 0, cfl: float = 0.4, dtrec: float = 1.0,
            nout: int = 1, use_graph: bool = True, nu0: float = 0.0, eta0: float = 0.0) -> RunInfo:
        o = RunOpts(int(max_steps), int(flg), int(stop_rule), float(cfl), float(dtrec), int(nout),
                    1 if use_graph else 0, float(nu0), float(eta0))
        info = RunInfo()
        _check(self.lib.qas_run(self.h, ctypes.byref(o), ctypes.byref(info)), "qas_run")
        return info

    def step_host(self, inp: np.ndarray, out: np.ndarray, flg: int = 1, stop_rule: int = 0, cfl: float = 0.4,
                  dtrec: float = 1.0, nout: int = 1) -> RunInfo:
        """One exec_ step on host blocks of 8*nd float64 (qas_step_host): upload, step and
        download with the copies overlapped; out may be inp (pinned memory for the overlap)."""
        for a in (inp, out):
            assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] and a.size == 8 * self.nd
        o = RunOpts(1, int(flg), int(stop_rule), float(cfl), float(dtrec), int(nout), 0, 0.0, 0.0)
        info = RunInfo()
        _check(self.lib.qas_step_host(self.h, _dptr(inp), _dptr(out), ctypes.byref(o), ctypes.byref(info)),
               "qas_step_host")
        return info

    def profile(self, nsteps: int, flg: int = 1, cfl: float = 0.4, nu0: float = 0.0, eta0: float = 0.0) -> dict:
        """Per-kernel {name: (launches, total_ms)} over nsteps eager exec_ steps (CUDA events)."""
        o = RunOpts(1, int(flg), 0, float(cfl), 1.0, 1, 0, float(nu0), float(eta0))
        out = (KernelTime * 32)()
        cnt = ctypes.c_int()
        _check(self.lib.qas_profile_run(self.h, ctypes.byref(o), int(nsteps), out, 32, ctypes.byref(cnt)),
               "qas_profile_run")
        return {out[i].name.decode(): (int(out[i].launches), float(out[i].total_ms)) for i in range(cnt.value)}

    def set_option(self, option: int, value: int) -> None:
        _check(self.lib.qas_set_option(self.h, int(option), int(value)), "qas_set_option")

    def set_tile(self, kernel: str, tx: int, ty: int = 1, tz: int = 1) -> None:
        _check(self.lib.qas_set_tile(self.h, kernel.encode(), tx, ty, tz), "qas_set_tile")

    def get_tile(self, kernel: str):
        t = [ctypes.c_int(), ctypes.c_int(), ctypes.c_int()]
        _check(self.lib.qas_get_tile(self.h, kernel.encode(), *[ctypes.byref(x) for x in t]), "qas_get_tile")
        return tuple(x.value for x in t)

    def autotune(self, trial_steps: int = 2) -> dict:
        _check(self.lib.qas_autotune(self.h, int(trial_steps)), "qas_autotune")
        return {k: self.get_tile(k) for k in ("k_prim", "k_dv", "k_lr", "k_flux", "k_emf", "k_update")}

    def run_reset(self) -> None:
        _check(self.lib.qas_run_reset(self.h), "qas_run_reset")

    def dissipate(self, dt: float, nu0: float, eta0: float) -> None:
        _check(self.lib.qas_dissipate(self.h, float(dt), float(nu0), float(eta0)), "qas_dissipate")

    def dsptv(self, dt: float, nu0: float, eta0: float) -> None:
        _check(self.lib.qas_dsptv(self.h, float(dt), float(nu0), float(eta0)), "qas_dsptv")

    # the reference's files ----------------------------------------------------
    def dout(self, directory: str, n: int, cnt: int, tim: float, coords=None) -> None:
        """dout_(): header files when n == 0 (`coords` = the x[, y[, z]] cell-centre coordinate
        arrays over the padded extents), t.dat appended otherwise, then outdat_<cnt>;
        asynchronous (dout_wait joins the writer)."""
        dp = ctypes.POINTER(ctypes.c_double)
        arr = None
        keep = []
        if coords is not None:  # copied by the call itself
            keep = [np.ascontiguousarray(c, dtype=np.float64) for c in coords]
            arr = (dp * 3)(*([k.ctypes.data_as(dp) for k in keep] + [None] * (3 - len(keep))))
        _check(self.lib.qas_dout(self.h, directory.encode(), int(n), int(cnt), float(tim), arr), "qas_dout")

    def dout_wait(self) -> None:
        _check(self.lib.qas_dout_wait(self.h), "qas_dout_wait")

    def bkup_save(self, directory: str, n: int, cnt: int, tim: float, dt: float, trec: float, rank: int = 0) -> None:
        _check(self.lib.qas_bkup_save(self.h, directory.encode(), int(n), int(cnt), float(tim), float(dt),
                                      float(trec), int(rank)), "qas_bkup_save")

    def bkup_load(self, directory: str, rank: int = 0):
        """Returns None when there is no stamp file, else (n, cnt, tim, dt, trec) with the state uploaded."""
        ld, n, cnt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        tim, dt, trec = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(self.lib.qas_bkup_load(self.h, directory.encode(), int(rank), ctypes.byref(ld), ctypes.byref(n),
                                      ctypes.byref(cnt), ctypes.byref(tim), ctypes.byref(dt), ctypes.byref(trec)),
               "qas_bkup_load")
        if not ld.value:
            return None
        return n.value, cnt.value, tim.value, dt.value, trec.value

    # discrete adjoint ---------------------------------------------------------
    def adjoint_forward(self, dts: Sequence[float], eta0: float = 0.0, ckpt_every: int = 20) -> None:
        """Run len(dts) exec_ steps (bound, ideal, dissipate) from the device state with the
        given dt per step, keeping checkpoints for adjoint_backward."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        _check(self.lib.qas_adjoint_forward(self.h, int(d.size), int(ckpt_every), _dptr(d), float(eta0)),
               "qas_adjoint_forward")

    def adjoint_backward(self, dldu: np.ndarray):
        """dL/d(final state) (8*nd values) -> (dL/d(initial state) as (8, nd), dL/deta0)."""
        g = np.ascontiguousarray(dldu, dtype=np.float64).reshape(8, -1)
        assert g.shape[1] == self.nd
        out = np.empty((8, self.nd), dtype=np.float64)
        eb = ctypes.c_double()
        _check(self.lib.qas_adjoint_backward(self.h, _dptr(g), _dptr(out), ctypes.byref(eb)), "qas_adjoint_backward")
        return out, eb.value

    def adjoint_run(self, dts: Sequence[float], dldu: np.ndarray, eta0: float = 0.0, ckpt_every: int = 20):
        """adjoint_forward then adjoint_backward in one call (qas_adjoint_run), for a known
        dL/d(final state): returns (dL/d(initial state) as (8, nd), dL/deta0)."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        g = np.ascontiguousarray(dldu, dtype=np.float64).reshape(8, -1)
        assert g.shape[1] == self.nd
        out = np.empty((8, self.nd), dtype=np.float64)
        eb = ctypes.c_double()
        _check(self.lib.qas_adjoint_run(self.h, int(d.size), int(ckpt_every), _dptr(d), float(eta0), _dptr(g),
                                        _dptr(out), ctypes.byref(eb)), "qas_adjoint_run")
        return out, eb.value

    def max_divb(self) -> float:
        v = ctypes.c_double()
        _check(self.lib.qas_max_divb(self.h, ctypes.byref(v)), "qas_max_divb")
        return v.value

    def sync(self) -> None:
        _check(self.lib.qas_sync(self.h), "qas_sync")

    def kernel_launches(self) -> int:
        v = ctypes.c_longlong()
        _check(self.lib.qas_kernel_launches(self.h, ctypes.byref(v)), "qas_kernel_launches")
        return int(v.value)

    def stream(self) -> int:
        v = ctypes.c_void_p()
        _check(self.lib.qas_stream(self.h, ctypes.byref(v)), "qas_stream")
        return int(v.value or 0)


def bc_map(prob, group: int, field: int, axis: int):
    """Host-only: the (source, factor) ghost-fill map of one group/field/axis (qas_bc_map)."""
    lib = load()
    g = Grid(prob.dim, prob.nxm, prob.nym if prob.dim >= 2 else 1, prob.nzm if prob.dim >= 3 else 1,
             prob.dx, prob.dy if prob.dim >= 2 else 0.0, prob.dz if prob.dim >= 3 else 0.0, prob.gam)
    b = BC()
    for m in range(8):
        b.dnx[m], b.dny[m], b.dnz[m] = int(prob.dnx[m]), int(prob.dny[m]), int(prob.dnz[m])
    n = (prob.nx, prob.ny, prob.nz)[axis]
    src = np.zeros(n, dtype=np.int32)
    fac = np.zeros(n, dtype=np.float64)
    _check(lib.qas_bc_map(ctypes.byref(g), ctypes.byref(b), group, field, axis,
                          src.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dptr(fac), n), "qas_bc_map")
    return src, fac


PIPE_ITEM_INTS = 38
PIPE_RANGE_NAMES = ("seg", "upd", "bnd", "prim", "dv", "fin", "lax", "fax", "emf")


def pipe_plan(planes: int, windows: int = 0, own_lanes: bool = True):
    """qas_step_host's wave along a last axis of `planes` padded planes (host only): the items,
    each {"nseg", "ends", name: [(lo, hi), (lo, hi)]} for the ranges of PIPE_RANGE_NAMES, and the
    issue lag."""
    lib = load()
    n, lag = ctypes.c_int(), ctypes.c_int()
    _check(lib.qas_pipe_plan(int(planes), int(windows), int(bool(own_lanes)), None, 0, ctypes.byref(n),
                             ctypes.byref(lag)), "qas_pipe_plan")
    buf = (ctypes.c_int * (PIPE_ITEM_INTS * n.value))()
    _check(lib.qas_pipe_plan(int(planes), int(windows), int(bool(own_lanes)), buf, n.value, ctypes.byref(n),
                             ctypes.byref(lag)), "qas_pipe_plan")
    items = []
    for q in range(n.value):
        rec = buf[q * PIPE_ITEM_INTS:(q + 1) * PIPE_ITEM_INTS]
        it = {"nseg": rec[0], "ends": bool(rec[1])}
        for k, name in enumerate(PIPE_RANGE_NAMES):
            it[name] = [(rec[2 + 18 * sg + 2 * k], rec[3 + 18 * sg + 2 * k]) for sg in range(2)]
        items.append(it)
    return items, lag.value


def dd_plan(prob, nparts: int):
    """Host-only: the slab split (global interior plane offsets, nparts+1 entries) and the
    ghost-plane copies [(part, src_part, src_plane, dst_plane, nplanes)] of a decomposition
    (qas_dd_plan)."""
    lib = load()
    g, _, b = _grid_scheme_bc(prob)
    lo = (ctypes.c_int * (nparts + 1))()
    cnt = ctypes.c_int()
    _check(lib.qas_dd_plan(ctypes.byref(g), ctypes.byref(b), int(nparts), lo, None, 0, ctypes.byref(cnt)),
           "qas_dd_plan")
    cps = (DdCopy * max(cnt.value, 1))()
    _check(lib.qas_dd_plan(ctypes.byref(g), ctypes.byref(b), int(nparts), lo, cps, cnt.value, ctypes.byref(cnt)),
           "qas_dd_plan")
    return list(lo), [(c.part, c.src_part, c.src_plane, c.dst_plane, c.nplanes) for c in cps[:cnt.value]]


class Decomposition:
    """One domain split into slabs along its last axis, each slab a context on its own device
    (or several on one): qas_dd_* (the reference's MPI rank decomposition in one process)."""

    def __init__(self, prob, nparts: int, devices: Optional[Sequence[int]] = None):
        self.lib = load()
        g, sc, b = _grid_scheme_bc(prob)
        devs = None
        if devices is not None:
            devs = (ctypes.c_int * nparts)(*[int(d) for d in devices])
        h = ctypes.c_void_p()
        _check(self.lib.qas_dd_create(ctypes.byref(h), ctypes.byref(g), ctypes.byref(sc), ctypes.byref(b),
                                      int(nparts), devs), "qas_dd_create")
        self.h = h
        self.shape = (8, prob.nz, prob.ny, prob.nx)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.qas_dd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, state: np.ndarray) -> None:
        a = np.ascontiguousarray(state, dtype=np.float64).reshape(self.shape)
        _check(self.lib.qas_dd_upload_block(self.h, _dptr(a)), "qas_dd_upload_block")

    def download(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        _check(self.lib.qas_dd_download_block(self.h, _dptr(out)), "qas_dd_download_block")
        return out

    def run(self, max_steps: int = 0, flg: int = 1, stop_rule: int = 0, cfl: float = 0.4, dtrec: float = 1.0,
            nout: int = 1) -> RunInfo:
        o = RunOpts(int(max_steps), int(flg), int(stop_rule), float(cfl), float(dtrec), int(nout), 0, 0.0, 0.0)
        info = RunInfo()
        _check(self.lib.qas_dd_run(self.h, ctypes.byref(o), ctypes.byref(info)), "qas_dd_run")
        return info

    def kernel_launches(self):
        k, c = ctypes.c_longlong(), ctypes.c_longlong()
        _check(self.lib.qas_dd_kernel_launches(self.h, ctypes.byref(k), ctypes.byref(c)), "qas_dd_kernel_launches")
        return int(k.value), int(c.value)


def _grid_scheme_bc(prob):
    g = Grid(prob.dim, prob.nxm, prob.nym if prob.dim >= 2 else 1, prob.nzm if prob.dim >= 3 else 1, prob.dx,
             prob.dy if prob.dim >= 2 else 0.0, prob.dz if prob.dim >= 3 else 0.0, prob.gam)
    sc = Scheme(prob.rmn, prob.odr, prob.rk, prob.ctw, getattr(prob, "char_mode", 0))
    b = BC()
    for m in range(8):
        b.dnx[m], b.dny[m], b.dnz[m] = int(prob.dnx[m]), int(prob.dny[m]), int(prob.dnz[m])
    return g, sc, b


class Batch:
    """An ensemble of independent problems stepped together (qas_batch_*)."""

    def __init__(self, probs, device: int = -1):
        self.lib = load()
        n = len(probs)
        gs, ss, bs = (Grid * n)(), (Scheme * n)(), (BC * n)()
        for q, p in enumerate(probs):
            gs[q], ss[q], bs[q] = _grid_scheme_bc(p)
        h = ctypes.c_void_p()
        _check(self.lib.qas_batch_create(ctypes.byref(h), n, gs, ss, bs, device), "qas_batch_create")
        self.h = h
        self.n = n
        self.nd = []
        for q in range(n):
            v = ctypes.c_longlong()
            _check(self.lib.qas_batch_cells(self.h, q, ctypes.byref(v)), "qas_batch_cells")
            self.nd.append(int(v.value))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.qas_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, q: int, state: np.ndarray) -> None:
        st = np.ascontiguousarray(state, dtype=np.float64).reshape(-1)
        assert st.size == 8 * self.nd[q]
        _check(self.lib.qas_batch_upload(self.h, q, _dptr(st)), "qas_batch_upload")

    def download(self, q: int, shape=None) -> np.ndarray:
        out = np.empty(8 * self.nd[q], dtype=np.float64)
        _check(self.lib.qas_batch_download(self.h, q, _dptr(out)), "qas_batch_download")
        return out if shape is None else out.reshape(shape)

    def run(self, max_steps: int = 0, flg: int = 1, stop_rule: int = 0, cfl: float = 0.4, dtrec: float = 1.0,
            nout: int = 1, use_graph: bool = True):
        o = RunOpts(int(max_steps), int(flg), int(stop_rule), float(cfl), float(dtrec), int(nout),
                    1 if use_graph else 0, 0.0, 0.0)
        info = (RunInfo * self.n)()
        _check(self.lib.qas_batch_run(self.h, ctypes.byref(o), info), "qas_batch_run")
        return [(info[q].steps, info[q].tim, info[q].dt) for q in range(self.n)]

    def set_tile(self, kernel: str, tx: int, ty: int = 1, tz: int = 1) -> None:
        _check(self.lib.qas_batch_set_tile(self.h, kernel.encode(), tx, ty, tz), "qas_batch_set_tile")

    def autotune(self, trial_steps: int = 2) -> None:
        _check(self.lib.qas_batch_autotune(self.h, int(trial_steps)), "qas_batch_autotune")

    def stream(self) -> int:
        v = ctypes.c_void_p()
        _check(self.lib.qas_batch_stream(self.h, ctypes.byref(v)), "qas_batch_stream")
        return int(v.value or 0)

    def kernel_launches(self) -> int:
        v = ctypes.c_longlong()
        _check(self.lib.qas_batch_kernel_launches(self.h, ctypes.byref(v)), "qas_batch_kernel_launches")
        return int(v.value)


def fp64_peak_tflops() -> float:
    """Measured FP64 throughput of the current device (qas_fp64_peak)."""
    lib = load()
    v = ctypes.c_double()
    _check(lib.qas_fp64_peak(ctypes.byref(v)), "qas_fp64_peak")
    return v.value


def max_divb_noalloc(grid: "Grid", odr: int, d_state_ptr: int, field_stride: int, stream: int = 0) -> float:
    """qas_max_divb_noalloc: max |div B| of a caller-owned device state (device pointer
    `d_state_ptr`, 8 fields `field_stride` doubles apart) on `stream`, allocating nothing."""
    lib = load()
    out = ctypes.c_double()
    _check(lib.qas_max_divb_noalloc(ctypes.byref(grid), int(odr), ctypes.c_void_p(d_state_ptr),
                                    int(field_stride), ctypes.c_void_p(stream), ctypes.byref(out)),
           "qas_max_divb_noalloc")
    return out.value
