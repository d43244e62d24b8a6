"""Initial states and run settings for the qasMHD problems this library steps.

A :class:`Problem` carries everything the reference fixes per problem
directory: the compile-time settings of ``mymacros.hpp`` (grid size, Riemann
solver ``rmn``, spatial order ``odr``, Runge-Kutta order ``rk``, CUCT weighting
``ctw``, CFL, output cadence; e.g. 2D/SERIAL/OTvortex/mymacros.hpp:4-14), the
run-time settings of ``paras()`` (domain, boundary flags ``dnxs/dnys/dnzs``,
gamma; 2D/SERIAL/OTvortex/mhd2d_paras.cpp:3-39) and the conservative state that
``init_()`` leaves behind (ro,mx,my,mz,bx,by,bz,en with 4 ghost cells per side,
ss = nx*(ny*k+j)+i; common/mhd_class.hpp:32-42).

Boundary flags follow the reference (common/common_func.h:256-271):
0 periodic, +1 Neumann, -1 Dirichlet, +2 open, -2 zero-fixed.

Everything here is host-side numpy; the state goes to the device through the
C-ABI (``qasmhd_b200.lib``).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Sequence

import numpy as np

XOFF = 4  # ghost cells per side (2D/SERIAL/OTvortex/mhd2d_class.hpp:10-12)
NM = 8    # number of MHD variables (common/mhd_class.hpp:17)

RMN_ROE, RMN_HLLD, RMN_LHLLD, RMN_MLAU = 0, 1, 2, 3


@dataclasses.dataclass
class Problem:
    """One simulation: grid, scheme, boundaries and the initial state."""

    name: str
    dim: int
    nxm: int
    nym: int = 1
    nzm: int = 1
    rmn: int = RMN_HLLD
    odr: int = 4
    rk: int = 3
    ctw: int = 1
    # face values: characteristic (0, mhd_m/a_reconst), primitive (1, mhd_reconst) or Athena-type
    # characteristic (2, mhd_c_reconst) variables
    char_mode: int = 0
    gam: float = 5.0 / 3.0
    cfl: float = 0.4
    dtrec: float = 1.0
    nout: int = 1
    xmin: float = 0.0
    xmax: float = 1.0
    ymin: float = 0.0
    ymax: float = 1.0
    zmin: float = 0.0
    zmax: float = 1.0
    dnx: Sequence[int] = (0,) * NM
    dny: Sequence[int] = (0,) * NM
    dnz: Sequence[int] = (0,) * NM
    nu0: float = 0.0
    eta0: float = 0.0
    # exec_ flag: 1 = dt refreshed every 2nd step (2D/3D drivers), 0 = constant dt (1D driver)
    flg: int = 1
    state: Optional[np.ndarray] = None  # shape (8, nz, ny, nx) incl. ghosts
    # gravitational potential phi_g (nz, ny, nx) of the gravity drivers, None without gravity
    phi: Optional[np.ndarray] = None
    # per-cell viscosity / resistivity of the dissipative drivers (the API's nu/eta), None: uniform
    nu_arr: Optional[np.ndarray] = None
    eta_arr: Optional[np.ndarray] = None
    # Hall driver (1D/SERIAL/h-shock, HMHD1D): on/off, ion inertia length di, electron inertia
    # length de (absolute, = dx*D_ELE)
    hall: bool = False
    di: float = 0.0
    de: float = 0.0

    @property
    def nx(self) -> int:
        return self.nxm + 2 * XOFF

    @property
    def ny(self) -> int:
        return self.nym + 2 * XOFF if self.dim >= 2 else 1

    @property
    def nz(self) -> int:
        return self.nzm + 2 * XOFF if self.dim >= 3 else 1

    @property
    def nd(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def interior_cells(self) -> int:
        return self.nxm * (self.nym if self.dim >= 2 else 1) * (self.nzm if self.dim >= 3 else 1)

    @property
    def dx(self) -> float:
        return (self.xmax - self.xmin) / self.nxm

    @property
    def dy(self) -> float:
        return (self.ymax - self.ymin) / self.nym

    @property
    def dz(self) -> float:
        return (self.zmax - self.zmin) / self.nzm

    @property
    def tmax(self) -> float:
        return self.dtrec * self.nout

    def coords(self):
        """Cell-centre coordinates incl. ghosts, (i-xoff+0.5)*dx+xmin as in
        2D/SERIAL/KHI/mhd2d_paras.cpp:36-37."""
        x = (np.arange(self.nx) - XOFF + 0.5) * self.dx + self.xmin
        y = (np.arange(self.ny) - XOFF + 0.5) * self.dy + self.ymin if self.dim >= 2 else np.zeros(1)
        z = (np.arange(self.nz) - XOFF + 0.5) * self.dz + self.zmin if self.dim >= 3 else np.zeros(1)
        return x, y, z

    def copy(self) -> "Problem":
        p = dataclasses.replace(self)
        p.state = None if self.state is None else self.state.copy()
        p.phi = None if self.phi is None else self.phi.copy()
        p.nu_arr = None if self.nu_arr is None else self.nu_arr.copy()
        p.eta_arr = None if self.eta_arr is None else self.eta_arr.copy()
        return p


def _energy(ro, vx, vy, vz, bx, by, bz, pr, gam):
    """Total energy, same expression order as mhd_energy (common/mhd_func.c:18-28)."""
    v2 = vx * vx + vy * vy + vz * vz
    b2 = bx * bx + by * by + bz * bz
    return pr / (gam - 1) + 0.5 * (ro * v2 + b2)


def _pack(ro, vx, vy, vz, bx, by, bz, pr, cx, cy, cz, gam):
    """Primitive -> conservative (cnsvt, common/mhd_class.hpp:73-79); B energy
    uses the cell-centre field cx,cy,cz."""
    st = np.empty((NM,) + ro.shape, dtype=np.float64)
    st[0] = ro
    st[1] = ro * vx
    st[2] = ro * vy
    st[3] = ro * vz
    st[4] = bx
    st[5] = by
    st[6] = bz
    st[7] = _energy(ro, vx, vy, vz, cx, cy, cz, pr, gam)
    return st


def _df(f0m1, f0, f1, f2, odr):
    """df1[ODR-1] on four consecutive values (common/common_interp.h:17-24)."""
    if odr >= 3:
        return (27.0 * (f1 - f0) - (f2 - f0m1)) / 24.0
    return f1 - f0


# ----------------------------------------------------------------------------
# C1: Brio-Wu shock tube
# ----------------------------------------------------------------------------

def brio_wu(nxm: int = 1024, rmn: int = RMN_HLLD, odr: int = 4, rk: int = 3,
            tmax: float = 0.1) -> Problem:
    """Brio & Wu shock tube on x in [0,1], outflow boundaries, gamma=2.

    Left (ro,pr,vx,vy,vz,bx,by,bz)=(1,1,0,0,0,0.75,1,0), right
    (0.125,0.1,0,0,0,0.75,-1,0); discontinuity at x=0.5 (the reference puts the
    same states on [-0.5,0.5] split at x<=0, 1D/SERIAL/shock/mhd1d_init_.cpp:14-30).
    The 1D driver runs with a constant dt (exec_(0), 1D/SERIAL/shock/main.cpp).
    """
    p = Problem(name=f"briowu_{nxm}", dim=1, nxm=nxm, rmn=rmn, odr=odr, rk=rk, ctw=0,
                gam=2.0, cfl=0.4, dtrec=tmax, nout=1, xmin=0.0, xmax=1.0,
                dnx=(2,) * NM, flg=0)
    x, _, _ = p.coords()
    left = x <= 0.5
    ro = np.where(left, 1.0, 0.125)
    pr = np.where(left, 1.0, 0.1)
    z = np.zeros_like(x)
    bx = np.full_like(x, 0.75)
    by = np.where(left, 1.0, -1.0)
    st = _pack(ro, z, z, z, bx, by, z, pr, bx, by, z, p.gam)
    p.state = st.reshape(NM, 1, 1, p.nx)
    return p


def localized_dissipation(prob: Problem, nu0: float, eta0: float, lam: float = 1.0) -> Problem:
    """The localized profiles of the reconnection drivers' setdc, nu = nu0 exp(-r/lambda) and
    eta = eta0 exp(-r/lambda) with r = sqrt(x^2 + y^2) over every padded cell
    (2D/SERIAL/MRX/dmhd2d_init_.cpp:85-106, 3D/MPI/MRX/dmhd3d_init_.cpp:98-118); returns a copy
    of the problem carrying them."""
    p = prob.copy()
    x, y, z = p.coords()
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    p.nu_arr = nu0 * np.exp(-r / lam)
    p.eta_arr = eta0 * np.exp(-r / lam)
    return p


def hall_shock(nxm: int = 400, di: float = 1e-3, rmn: int = RMN_LHLLD, odr: int = 4, rk: int = 3,
               tmax: float = 1.0, nout: int = 1, d_ele: float = 0.0) -> Problem:
    """Brio-Wu states of the Hall driver (1D/SERIAL/h-shock/mhd1d_init_.cpp, NUM 2) on
    x in [-0.5, 0.5] split at x <= 0, gamma = 2, Neumann (+1) boundaries for every field
    (hmhd1d_paras.cpp:6-20), ion inertia length di, electron inertia length de = dx*d_ele (the
    reference's D_ELE; 0 in its configurations), and the driver's exec_(0) loop (constant dt,
    h-shock/main.cpp)."""
    p = Problem(name=f"hallshock_{nxm}", dim=1, nxm=nxm, rmn=rmn, odr=odr, rk=rk, ctw=0, gam=2.0, cfl=0.4,
                dtrec=tmax, nout=nout, xmin=-0.5, xmax=0.5, dnx=(1,) * NM, flg=0, hall=True, di=di, de=0.0)
    p.de = p.dx * d_ele
    x, _, _ = p.coords()
    left = x <= 0
    ro = np.where(left, 1.0, 0.125)
    pr = np.where(left, 1.0, 0.1)
    z = np.zeros_like(x)
    bx = np.full_like(x, 0.75)
    by = np.where(left, 1.0, -1.0)
    st = _pack(ro, z, z, z, bx, by, z, pr, bx, by, z, p.gam)
    p.state = st.reshape(NM, 1, 1, p.nx)
    return p


def hall_vphix(prob) -> float:
    """Whistler speed factor of HMHD1D::paras (1D/SERIAL/h-shock/hmhd1d_paras.cpp:29-34)."""
    idx = 1.0 / prob.dx
    kpeak = math.pi * idx
    if prob.de != 0:
        k_e = 1.0 / prob.de
        kpeak = k_e if kpeak >= k_e else kpeak  # min() of common/common_func.h
    return prob.di * kpeak


# ----------------------------------------------------------------------------
# C2: Orszag-Tang vortex
# ----------------------------------------------------------------------------

def orszag_tang(n: int = 1024, rmn: int = RMN_HLLD, odr: int = 4, rk: int = 3, ctw: int = 1,
                tmax: float = 0.5, nym: Optional[int] = None) -> Problem:
    """Orszag-Tang vortex on [0,2pi]^2, periodic, gamma=5/3.

    ro=25/(36pi), pr=5/(12pi), v=(-sin y, sin x, 0),
    B=(-sin y, sin 2x, 0)/sqrt(4pi) built on the faces from the corner vector
    potential A_z=(cos y + cos(2x)/2)/sqrt(4pi) with the same difference
    operator df1[ODR-1] the CT update uses (the idiom of
    2D/SERIAL/loop/mhd2d_init_.cpp:22-55), so the ODR-consistent div B is zero.
    """
    nym = n if nym is None else nym
    p = Problem(name=f"ot_{n}x{nym}", dim=2, nxm=n, nym=nym, rmn=rmn, odr=odr, rk=rk, ctw=ctw,
                gam=5.0 / 3.0, cfl=0.4, dtrec=tmax, nout=1,
                xmin=0.0, xmax=2.0 * math.pi, ymin=0.0, ymax=2.0 * math.pi, flg=1)
    x, y, _ = p.coords()
    dx, dy = p.dx, p.dy
    s4 = math.sqrt(4.0 * math.pi)
    X, Y = np.meshgrid(x, y)  # (ny, nx)
    # corner potential at (x-dx/2, y-dy/2), one extra ring for the 4-point stencils
    xc = (np.arange(-1, p.nx + 2) - XOFF) * dx + p.xmin
    yc = (np.arange(-1, p.ny + 2) - XOFF) * dy + p.ymin
    XC, YC = np.meshgrid(xc, yc)
    az = (np.cos(YC) + 0.5 * np.cos(2.0 * XC)) / s4        # index [j+1, i+1] <-> corner (i-1/2, j-1/2)
    # bx at face (i-1/2, j) = +D_y A over corners j-3/2..j+3/2 (rows j..j+3 of az)
    bx = _df(az[0:-3, 1:-2], az[1:-2, 1:-2], az[2:-1, 1:-2], az[3:, 1:-2], odr) / dy
    by = -_df(az[1:-2, 0:-3], az[1:-2, 1:-2], az[1:-2, 2:-1], az[1:-2, 3:], odr) / dx
    ro = np.full_like(X, 25.0 / (36.0 * math.pi))
    pr = np.full_like(X, 5.0 / (12.0 * math.pi))
    vx = -np.sin(Y)
    vy = np.sin(X)
    z = np.zeros_like(X)
    cx = -np.sin(Y) / s4
    cy = np.sin(2.0 * X) / s4
    st = _pack(ro, vx, vy, z, bx, by, z, pr, cx, cy, z, p.gam)
    p.state = st.reshape(NM, 1, p.ny, p.nx)
    return p


# ----------------------------------------------------------------------------
# C3/C4/C5: Kelvin-Helmholtz
# ----------------------------------------------------------------------------

def kelvin_helmholtz(dim: int = 3, n: int = 256, mach: float = 0.01, beta: float = 100.0,
                     rmn: int = RMN_MLAU, odr: int = 4, rk: int = 3, ctw: int = 1,
                     gam: float = 5.0 / 3.0, seed: int = 12345, nym: Optional[int] = None,
                     nzm: Optional[int] = None, noise: float = 1e-3, tmax: float = 1e30,
                     nout: int = 1, dvy_field: Optional[np.ndarray] = None) -> Problem:
    """Low-Mach Kelvin-Helmholtz layer on [-0.5,0.5]^dim.

    Periodic in x (and z), open (+2) in y.  vx=(M/2) tanh(y/0.05) with sonic Mach
    M (sound speed 1: ro=1, pr=1/gam), uniform guide field bz giving plasma
    beta=2pr/B^2, weak bx=0.01.  Gaussian velocity perturbations of amplitude
    noise*M localised by exp(-(y/0.1)^2) come from numpy's default_rng(seed),
    so both codes receive the identical state.  ``dvy_field`` (interior-shaped)
    replaces the random vy perturbation (used by the gradient tests).
    """
    nym = n if nym is None else nym
    nzm = (n if nzm is None else nzm) if dim >= 3 else 1
    dn_y = (2,) * NM
    p = Problem(name=f"kh{dim}d_{n}", dim=dim, nxm=n, nym=nym, nzm=nzm, rmn=rmn, odr=odr, rk=rk,
                ctw=ctw, gam=gam, cfl=0.4, dtrec=tmax, nout=nout,
                xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5,
                zmin=-0.5, zmax=0.5, dnx=(0,) * NM, dny=dn_y, dnz=(0,) * NM, flg=1)
    x, y, z = p.coords()
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")  # (nz, ny, nx)
    rng = np.random.default_rng(seed)
    amp = noise * mach * np.exp(-(Y / 0.1) ** 2)
    shape = X.shape
    ro = np.ones(shape)
    pr = np.full(shape, 1.0 / gam)
    vx = 0.5 * mach * np.tanh(Y / 0.05) + amp * rng.standard_normal(shape)
    if dvy_field is not None:
        full = np.zeros(shape)
        sl = (slice(XOFF, XOFF + nzm) if dim >= 3 else slice(0, 1),
              slice(XOFF, XOFF + nym), slice(XOFF, XOFF + p.nxm))
        full[sl] = np.asarray(dvy_field, dtype=np.float64).reshape(full[sl].shape)
        vy = amp * full
        rng.standard_normal(shape)
    else:
        vy = amp * rng.standard_normal(shape)
    vz = amp * rng.standard_normal(shape) if dim >= 3 else np.zeros(shape)
    bx = np.full(shape, 0.01)
    by = np.zeros(shape)
    bz = np.full(shape, math.sqrt(2.0 * (1.0 / gam) / beta))
    st = _pack(ro, vx, vy, vz, bx, by, bz, pr, bx, by, bz, gam)
    p.state = st
    return p


def smooth_wave(dim: int, n: int, rmn: int = RMN_HLLD, odr: int = 4, rk: int = 3, ctw: int = 1,
                seed: int = 7, amp: float = 1e-2, dn=None) -> Problem:
    """Small random smooth perturbation of a uniform magnetised plasma; periodic
    unless ``dn`` gives per-axis flag tuples.  Used by parity tests to exercise
    every solver/BC combination on small grids."""
    rng = np.random.default_rng(seed)
    nyz = n if dim >= 2 else 1
    p = Problem(name=f"wave{dim}d_{n}", dim=dim, nxm=n, nym=nyz, nzm=n if dim >= 3 else 1,
                rmn=rmn, odr=odr, rk=rk, ctw=ctw, gam=5.0 / 3.0, cfl=0.4,
                xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0, flg=1)
    if dn is not None:
        p.dnx, p.dny, p.dnz = dn
    shape = (p.nz, p.ny, p.nx)
    x, y, z = p.coords()
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    ph = rng.uniform(0, 2 * np.pi, size=8)

    def wave(k):
        return np.sin(2 * np.pi * X + ph[k]) * np.cos(2 * np.pi * (Y + Z) + ph[k])

    ro = 1.0 + amp * wave(0)
    vx = 0.3 + amp * wave(1)
    vy = -0.2 + amp * wave(2)
    vz = 0.1 + amp * wave(3)
    bx = 0.7 + amp * wave(4)
    by = 0.4 + amp * wave(5)
    bz = -0.3 + amp * wave(6)
    pr = 0.8 + amp * wave(7)
    st = _pack(ro, vx, vy, vz, bx, by, bz, pr, bx, by, bz, p.gam)
    p.state = st
    return p


# ----------------------------------------------------------------------------
# C4: batched ensemble
# ----------------------------------------------------------------------------

def rayleigh_taylor(dim: int = 2, nxm: int = 128, ngm: int = 1024, nym3: Optional[int] = None,
                    rmn: int = RMN_LHLLD, odr: int = 4, rk: int = 3, ctw: int = 1, gam: float = 5.0 / 3.0,
                    tmax: float = 1e30, nout: int = 1) -> Problem:
    """Rayleigh-Taylor instability of the gravity drivers (2D/SERIAL/RTI, 3D/MPI/RTI).

    Gravity along the last axis h (y in 2D, z in 3D) from phi_g = g0*lg*log(cosh(h/lg)), g0 = 1,
    lg = 8 cells; a heavy layer (ro 1) above |h| = 0.35 L_h over a light one (ro 0.1 in 2D,
    0.2 in 3D), tanh-smoothed over width 1; pressure from the hydrostatic balance
    dP/dh = -ro dphi/dh integrated from h = 0 (base 500 in 2D, 50 in 3D) by the midpoint rule
    with 1 + round(|h|/dh) intervals, floored at 1e-4; a uniform field transverse to gravity
    (bz in 2D, by in 3D) at plasma beta 1e3 (2D) / 1e2 (3D); a single-mode velocity kick of
    amplitude 0.01 along h localised at the two interfaces.  Box: x (and y in 3D) in [0, 20],
    h in [-10 ngm/nxm, +10 ngm/nxm]; periodic across, open (+2) along h.  The total energy
    carries ro*phi_g, as the drivers' init_ does (2D/SERIAL/RTI/mhd2d_init_.cpp:8-88).
    """
    if dim not in (2, 3):
        raise ValueError("the gravity drivers are 2D and 3D")
    nym = (nxm if nym3 is None else nym3) if dim == 3 else ngm
    nzm = ngm if dim == 3 else 1
    hext = 0.5 * 20.0 * ngm / nxm
    kw = dict(xmin=0.0, xmax=20.0)
    if dim == 2:
        kw.update(ymin=-hext, ymax=hext)
        dn = dict(dnx=(0,) * NM, dny=(2,) * NM, dnz=(0,) * NM)
    else:
        kw.update(ymin=0.0, ymax=20.0, zmin=-hext, zmax=hext)
        dn = dict(dnx=(0,) * NM, dny=(0,) * NM, dnz=(2,) * NM)
    p = Problem(name=f"rt{dim}d_{nxm}x{ngm}", dim=dim, nxm=nxm, nym=nym, nzm=nzm, rmn=rmn, odr=odr, rk=rk,
                ctw=ctw, gam=gam, cfl=0.4, dtrec=tmax, nout=nout, flg=1, **kw, **dn)
    x, y, z = p.coords()
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    H = Y if dim == 2 else Z
    dh = p.dy if dim == 2 else p.dz
    lh = p.ymax - p.ymin if dim == 2 else p.zmax - p.zmin
    g0, lg, width, s0 = 1.0, 8.0 * dh, 1.0, 0.35 * lh
    ro_u, ro_l = 1.0, (0.1 if dim == 2 else 0.2)
    pr0, beta = (500.0, 1e3) if dim == 2 else (50.0, 1e2)
    b0 = math.sqrt(2.0 * pr0 / beta)

    def layer(vu, vl, h):
        return 0.5 * (2.0 + np.tanh((h - s0) / width) - np.tanh((h + s0) / width)) * (vu - vl) + vl

    def pressure(h):
        n = 1 + int(abs(h) / dh + 0.5)
        d = h / n
        acc = pr0
        for q in range(n):
            hc = (q + 0.5) * d
            acc += -layer(ro_u, ro_l, hc) * (g0 * math.tanh(hc / lg)) * d
        return acc

    hs = y if dim == 2 else z
    pr_h = np.array([max(pressure(h), 1e-4) for h in hs])
    pr = pr_h[None, :, None] if dim == 2 else pr_h[:, None, None]
    pr = np.broadcast_to(pr, X.shape).astype(np.float64)
    ro = layer(ro_u, ro_l, H)
    kick = 0.01 * np.cos(2 * math.pi * X / 20.0) * (1.0 if dim == 2 else np.cos(2 * math.pi * Y / 20.0))
    vh = kick * (np.exp(-((H - s0) ** 2) / (4 * width ** 2)) - np.exp(-((H + s0) ** 2) / (4 * width ** 2)))
    zero = np.zeros_like(X)
    vx, vy, vz = (zero, vh, zero) if dim == 2 else (zero, zero, vh)
    bx = zero
    by = zero if dim == 2 else np.full_like(X, b0)
    bz = np.full_like(X, b0) if dim == 2 else zero
    phi = g0 * lg * np.log(np.cosh(H / lg))
    st = _pack(ro, vx, vy, vz, bx, by, bz, pr, bx, by, bz, gam)
    st[7] = st[7] + ro * phi
    p.state = st
    p.phi = phi
    return p


def ensemble(n: int = 512, lo: int = 64, hi: int = 512, seed: int = 2025, odr: int = 4) -> list:
    """Seeded ensemble of 2D instances with log-uniform sides in [lo, hi]
    (non-square allowed): even members are Orszag-Tang (HLLD), odd members
    Kelvin-Helmholtz (MLAU) with Mach number log-uniform in [1e-3, 1] and
    plasma beta log-uniform in [0.1, 1e3]."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        nx = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        ny = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        if q % 2 == 0:
            p = orszag_tang(nx, nym=ny, rmn=RMN_HLLD, odr=odr)
        else:
            mach = math.exp(rng.uniform(math.log(1e-3), math.log(1.0)))
            beta = math.exp(rng.uniform(math.log(0.1), math.log(1e3)))
            p = kelvin_helmholtz(2, nx, nym=ny, mach=mach, beta=beta, rmn=RMN_MLAU, odr=odr,
                                 seed=int(rng.integers(1 << 30)))
        p.name = f"ens{q}_{p.name}"
        out.append(p)
    return out
