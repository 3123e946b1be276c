"""Synthetic cases: decks and initial fields of the named workloads.

There is no public dataset behind the reference's benchmarks; the fields are
analytic (Taylor-Green vortex) or seeded (isotropic turbulence), and the
cylinder grid is generated analytically.  Arrays are numpy float64 in C order
[k][j][i], i.e. the reference's Fortran order (i fastest).
"""
from __future__ import annotations

import math

import numpy as np

from .params import (BC_USER_DEF, GRID2D_PLANE, GRIDGEN, GRID1D, SCHEME_CD6, SCHEME_HYBRID, SCHEME_OMP6,
                     SCHEME_WENO7, SPLIT_LLF, SPLIT_SW, OcfdParams, default_params)

TWO_PI = 6.2831853071795864
PI = 3.1415926535897932


def periodic_box(p: OcfdParams, nx: int, ny: int, nz: int) -> OcfdParams:
    p.nx, p.ny, p.nz = nx, ny, nz
    p.iperiodic[0] = p.iperiodic[1] = p.iperiodic[2] = 1
    for d in range(3):
        for c in range(3):
            p.periodic_span[d][c] = TWO_PI if c == d else 0.0
    return p


def box_coords(nx: int, ny: int, nz: int):
    """mesh_gen('box') (OCFD_mesh.f90:335-347): x_i = 2*pi/N * i, i = 1..N."""
    x = 2.0 * PI / float(nx) * np.arange(1, nx + 1, dtype=np.float64)
    y = 2.0 * PI / float(ny) * np.arange(1, ny + 1, dtype=np.float64)
    z = 2.0 * PI / float(nz) * np.arange(1, nz + 1, dtype=np.float64)
    return x, y, z


def tgv_params(n: int, scheme=SCHEME_WENO7, character=0, ma=0.1, re=1600.0, dt=0.005, steps=100,
               split=SPLIT_SW, ny: int | None = None, nz: int | None = None) -> OcfdParams:
    """Taylor-Green vortex deck: periodic [0,2pi]^3 box grid, CD6 viscous terms."""
    p = default_params()
    periodic_box(p, n, ny or n, nz or n)
    p.iflag_gridtype = GRIDGEN
    p.scheme_invis = scheme
    p.scheme_vis = SCHEME_CD6
    p.if_scheme_character = character
    p.flux_splitting = split
    p.ma, p.re, p.pr, p.gamma = ma, re, 0.7, 1.4
    p.dt = dt
    p.end_time = dt * steps
    p.istep_show = max(steps, 1)
    p.istep_save = 10 ** 8
    p.hybrid_para[3] = 0.0  # no forced patches (the reference's patch loop has an undefined je)
    return p


def tgv_char_params(n: int, scheme: str, dt: float = 0.0005, steps: int = 500) -> OcfdParams:
    """Characteristic-flux Taylor-Green decks of the 256^3 runs (du_inviscous_Character,
    SW, CD6): "OMP6", or "HYBRID" with sensor 1, thresholds 0.004 / 0.01 and UD7L_Diss = 0
    (the linear faces are CD8 central).  dt = 0.0005: the stated 0.002 is above the
    stability limit of RK3 with these schemes at Ma 0.1 on 256^3."""
    from .params import SCHEME

    p = tgv_params(n, scheme=SCHEME[scheme], character=1, split=SPLIT_SW, dt=dt, steps=steps)
    if scheme == "HYBRID":
        p.hybrid_para[0] = 1
        p.hybrid_para[1] = 0.004
        p.hybrid_para[2] = 0.01
        p.ud7l_diss = 0.0
    return p


def tgv_prims(p: OcfdParams):
    """TGV initial primitives: rho=1, u=sin x cos y cos z, v=-cos x sin y cos z, w=0,
    p = p0 + (cos2x+cos2y)(cos2z+2)/16, T = p/(rho p0), p0 = 1/(gamma Ma^2)."""
    x, y, z = box_coords(p.nx, p.ny, p.nz)
    # the trigonometric factors are evaluated on the 1-D coordinates and
    # broadcast (the same values and products as on the full 3-D mesh)
    X, Y, Z = x[None, None, :], y[None, :, None], z[:, None, None]
    shape = (p.nz, p.ny, p.nx)
    p0 = 1.0 / (p.gamma * p.ma * p.ma)
    d = np.ones(shape)
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros(shape)
    pr = p0 + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    T = pr / (d * p0)
    return [np.ascontiguousarray(np.broadcast_to(a, shape)) for a in (d, u, v, w, T)]


def hit_params(n: int, re: float = 500.0, ma: float = 1.0, dt: float = 1e-3, steps: int = 300,
               mixed: bool = False) -> OcfdParams:
    """Decaying isotropic turbulence deck: HYBRID + LLF, non-characteristic, 1-D grid file."""
    p = default_params()
    periodic_box(p, n, n, n)
    p.iflag_gridtype = GRID1D
    p.scheme_invis = SCHEME_HYBRID
    p.scheme_vis = SCHEME_CD6
    p.if_scheme_character = 0
    p.flux_splitting = SPLIT_LLF
    p.ud7l_diss = 0.0  # linear part = CD8 central
    p.hybrid_para[0] = 1.0  # sensor 1
    p.hybrid_para[1] = 0.02
    p.hybrid_para[2] = 0.1
    p.hybrid_para[3] = 0.0
    p.ma, p.re, p.pr, p.gamma = ma, re, 0.7, 1.4
    p.dt = dt
    p.end_time = dt * steps
    p.istep_show = max(steps, 1)
    p.istep_save = 10 ** 8
    p.precision = 1 if mixed else 0
    return p


def hit_coords(n: int):
    """1-D grid file of examples/isotropic: x = (i-1) 2 pi / N."""
    x = (np.arange(n, dtype=np.float64)) * (TWO_PI / n)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    return X.copy(), Y.copy(), Z.copy()


def hit_prims(n: int, mt: float, ma: float, k0: float = 4.0, seed: int = 20261203):
    """Seeded solenoidal random-phase velocity with E(k) ~ k^4 exp(-2 (k/k0)^2),
    scaled to turbulent Mach number mt = sqrt(<u^2+v^2+w^2>)/<c> with c = sqrt(T)/Ma
    (the ana_box definitions, OCFD_ANA.f90:227,265); rho = T = 1.  Built on the
    real-to-complex half spectrum with broadcast wavenumbers, so the host memory
    peak stays near 8 GB at 512^3."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n, d=1.0 / n)
    kr = np.fft.rfftfreq(n, d=1.0 / n)
    KZ = k[:, None, None]
    KY = k[None, :, None]
    KX = kr[None, None, :]
    kk2 = KZ ** 2 + KY ** 2 + KX ** 2
    kk2[0, 0, 0] = 1.0
    kk = np.sqrt(kk2)
    amp = np.sqrt(kk ** 4 * np.exp(-2.0 * (kk / k0) ** 2) / (4.0 * np.pi * kk2))
    amp[0, 0, 0] = 0.0
    del kk
    comps = [amp * np.exp(1j * rng.uniform(0, 2 * np.pi, size=amp.shape)) for _ in range(3)]
    del amp
    # solenoidal projection: c -= (c.k) k / |k|^2
    dot = (comps[0] * KX + comps[1] * KY + comps[2] * KZ) / kk2
    comps[0] -= dot * KX
    comps[1] -= dot * KY
    comps[2] -= dot * KZ
    del dot, kk2
    vel = []
    while comps:
        vel.append(np.fft.irfftn(comps.pop(0), s=(n, n, n), axes=(0, 1, 2)))
    c_mean = 1.0 / ma
    rms = math.sqrt(float(np.mean(vel[0] ** 2) + np.mean(vel[1] ** 2) + np.mean(vel[2] ** 2)))
    s = mt * c_mean / rms
    u, v, w = [np.ascontiguousarray(a * s) for a in vel]
    d = np.ones_like(u)
    T = np.ones_like(u)
    return [d, u, v, w, T]


def cylinder_params(ni: int = 301, nj: int = 401, nk: int = 8, ma: float = 6.0, re: float = 1e5,
                    tw: float = 3.0, dt: float = 2e-5, steps: int = 2000, character: int = 1) -> OcfdParams:
    """Mach 6 blunt cylinder: i circumferential, j wall-normal (j=1 wall), k span periodic.
    Isothermal wall through the BC_User_Def slot, ghost-cell WENO5 closure at the wall."""
    p = default_params()
    p.nx, p.ny, p.nz = ni, nj, nk
    p.iperiodic[0] = 0
    p.iperiodic[1] = 0
    p.iperiodic[2] = 1
    p.periodic_span[2][2] = 0.1
    p.iflag_gridtype = GRID2D_PLANE
    p.scheme_invis = SCHEME_WENO7
    p.scheme_vis = SCHEME_CD6
    p.if_scheme_character = character
    p.flux_splitting = SPLIT_SW
    p.ibc = BC_USER_DEF
    p.bc_para[0] = tw
    p.ghost_cell[2] = 2
    p.scheme_boundary[2] = 1
    p.ma, p.re, p.pr, p.gamma = ma, re, 0.7, 1.4
    p.dt = dt
    p.end_time = dt * steps
    p.istep_show = max(steps, 1)
    p.istep_save = 10 ** 8
    p.hybrid_para[3] = 0.0
    return p


def cylinder_grid(ni: int, nj: int, nk: int, r: float = 1.0, ax: float = 4.0, ay: float = 6.0,
                  h1: float = 1e-4, span: float = 0.1):
    """Body-fitted grid: circle of radius r (j=1) to an ellipse with semi-axes ax (streamwise)
    and ay (transverse) (j=nj), over the windward half theta from 3pi/2 down to pi/2 (i, so
    that (i, j, k) is right-handed and the Jacobian positive), with tanh clustering of
    first-cell height h1*r at the wall; k is a periodic span."""
    th = np.linspace(1.5 * PI, 0.5 * PI, ni)
    # tanh stretching: s in [0,1] with ds(0) ~ h1 / length
    eta = np.linspace(0.0, 1.0, nj)
    L = 0.5 * ((ax - r) + (ay - r))
    target = h1 * r / L

    def dist(beta):
        return 1.0 + np.tanh(beta * (eta - 1.0)) / np.tanh(beta)

    lo, hi = 1e-3, 20.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if dist(mid)[1] > target:
            lo = mid
        else:
            hi = mid
    s = dist(0.5 * (lo + hi))
    X2 = np.empty((nj, ni))
    Y2 = np.empty((nj, ni))
    for j in range(nj):
        xi_in, yi_in = r * np.cos(th), r * np.sin(th)
        xo, yo = ax * np.cos(th), ay * np.sin(th)
        X2[j] = xi_in + s[j] * (xo - xi_in)
        Y2[j] = yi_in + s[j] * (yo - yi_in)
    z1 = span * np.arange(nk, dtype=np.float64) / nk
    X = np.broadcast_to(X2, (nk, nj, ni)).copy()
    Y = np.broadcast_to(Y2, (nk, nj, ni)).copy()
    Z = np.broadcast_to(z1[:, None, None], (nk, nj, ni)).copy()
    return X, Y, Z


def cylinder_prims(ni: int, nj: int, nk: int):
    """Impulsive start: uniform free stream (1,1,0,0,1) with the wall values applied by the BC."""
    d = np.ones((nk, nj, ni))
    return [d, np.ones_like(d), np.zeros_like(d), np.zeros_like(d), np.ones_like(d)]
