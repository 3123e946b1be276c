"""Shared set-up for the parity tests: the same case on the oracle and on the GPU."""
from __future__ import annotations

import numpy as np

from ocfd_b200 import cases
from ocfd_b200.params import (BC_BLUNT2D, BC_USER_DEF, SCHEME_HYBRID, SCHEME_OMP6, SCHEME_UD7L, SCHEME_WENO5,
                              SCHEME_WENO7, SPLIT_LLF, SPLIT_SW)

LAP = 4


def tgv_case(scheme=SCHEME_WENO7, character=0, split=SPLIT_SW, n=(24, 20, 16), dt=0.005, ma=0.1, re=1600.0,
             sensor=1, t1=0.004, t2=0.01, cd8=False, mixed=False):
    p = cases.tgv_params(n[0], scheme=scheme, character=character, split=split, ny=n[1], nz=n[2], dt=dt, ma=ma, re=re)
    if scheme == SCHEME_HYBRID:
        p.hybrid_para[0] = sensor
        p.hybrid_para[1] = t1
        p.hybrid_para[2] = t2
        p.hybrid_para[3] = 0
        p.ud7l_diss = 0.0
    if cd8:
        p.scheme_vis = 6
    p.precision = 1 if mixed else 0
    return p, None, cases.tgv_prims(p)


def curvilinear_case(bc=BC_USER_DEF, character=1, scheme=SCHEME_WENO7, n=(24, 20, 8), ghost=True, dt=2e-5,
                     ma=3.0, re=1e4, h1=2e-2):
    ni, nj, nk = n
    p = cases.cylinder_params(ni, nj, nk, ma=ma, re=re, dt=dt, steps=10, character=character)
    p.scheme_invis = scheme
    p.ibc = bc
    if not ghost:
        p.ghost_cell[2] = 0
        p.scheme_boundary[2] = 0
    X, Y, Z = cases.cylinder_grid(ni, nj, nk, h1=h1)
    prims = cases.cylinder_prims(ni, nj, nk)
    # a smooth perturbation so that every term is exercised
    kk, jj, ii = np.meshgrid(np.arange(nk), np.arange(nj), np.arange(ni), indexing="ij")
    prims[2] = prims[2] + 0.05 * np.sin(2 * np.pi * ii / ni) * np.cos(2 * np.pi * kk / nk)
    prims[4] = prims[4] * (1.0 + 0.02 * np.cos(np.pi * jj / nj))
    return p, (X, Y, Z), prims


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def interior(h):
    return h[LAP:-LAP, LAP:-LAP, LAP:-LAP]


def boundary_layer_case(kind="bl", n=(24, 20, 8), ghost=False, tw=-1.0, pert=True, nonref=0, outlet=2,
                        inlet_2d=False, ma=2.25, re=1.0e4, dt=5.0e-4, seed=11):
    """Flat-plate boundary layer (BC_BoundaryLayer, kind "bl", periodic span) or
    swept-corner style span (BC_SweptCorner, kind "sc": walls on part of the
    span, k- symmetry plane).  2-D plane grid: x uniform in [0.1, 1.1], y
    sinh-stretched in [0, 0.4]; span uniform.  Inlet and initial field: a
    synthetic compressible boundary-layer profile (u = tanh(3 y / 0.1), adiabatic
    Crocco temperature, constant pressure)."""
    from ocfd_b200 import bclayer
    from ocfd_b200.params import BC_BOUNDARYLAYER, BC_SWEPTCORNER, GRID2D_PLANE, SCHEME_WENO7, default_params

    ni, nj, nk = n
    p = default_params()
    p.nx, p.ny, p.nz = ni, nj, nk
    p.iperiodic[0] = p.iperiodic[1] = 0
    p.iperiodic[2] = 1 if kind == "bl" else 0
    lz = 0.2
    p.periodic_span[2][2] = lz
    p.iflag_gridtype = GRID2D_PLANE
    p.scheme_invis = SCHEME_WENO7
    p.if_scheme_character = 1
    p.ma, p.re, p.dt = ma, re, dt
    p.ibc = BC_BOUNDARYLAYER if kind == "bl" else BC_SWEPTCORNER
    x = 0.1 + np.arange(ni) / (ni - 1.0)
    b = 2.5
    y = 0.4 * np.sinh(b * np.arange(nj) / (nj - 1.0)) / np.sinh(b)
    dz = lz / nk
    z = (np.arange(nk) + 0.5) * dz if kind == "sc" else np.arange(nk) * dz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    u = np.tanh(3.0 * y / 0.1)
    T = 1.0 + 0.89 * 0.2 * ma * ma * (1.0 - u * u)
    prof = np.stack([1.0 / T, u, np.zeros_like(u), np.zeros_like(u), T], axis=1)  # (ny, 5)
    prims = [np.ascontiguousarray(np.broadcast_to(prof[:, q][None, :, None], (nk, nj, ni))) for q in range(5)]
    rng = np.random.default_rng(seed)
    inlet = bclayer.inlet_from_profile(prof, nk)
    if inlet_2d:
        inlet = inlet * (1.0 + 0.01 * np.cos(2 * np.pi * np.arange(nk) / nk))[None, :, None]
    if kind == "bl":
        bclayer.boundary_layer_bc_para(p, inlet=2 if inlet_2d else 1, upper=0, nonref=nonref, outlet=outlet, tw=tw,
                                       dis_type=1 if pert else 0, amp=0.02, xbegin=0.3, xend=0.8, mt=3, mz=2,
                                       zl=lz, freq=20.0)
        if ghost:
            p.ghost_cell[2] = -1
            p.scheme_boundary[2] = -1
        pertb = bclayer.wall_perturbation(1 if pert else 0, X[:, 0, :], Z[:, 0, :], 0.3, 0.8, 2, lz, rng)
    else:
        bclayer.swept_corner_bc_para(p, outlet=outlet, tw=tw, wall_zl=0.5 * lz, dis_type=1 if pert else 0,
                                     amp=0.02, xbegin=0.3, xend=0.8, mt=3, mz=-1, freq=20.0, z1=0, z2=1)
        p.ghost_cell[4] = -1
        p.scheme_boundary[4] = -1
        pertb = bclayer.wall_perturbation(1 if pert else 0, X[:, 0, :], Z[:, 0, :], 0.3, 0.8, -1, 0.5 * lz, rng)
    tm, fait = bclayer.time_factor(3, rng)
    data = bclayer.BcLayerData(inlet=inlet, pertb=pertb, beta=20.0 if pert else 0.0, tm=tm, fait=fait)
    return p, (X, Y, Z), prims, data


def annulus_case(nx=24, ny=16, nz=20):
    """Periodic annular duct in axisymmetric form: i axial (periodic, length 2),
    j radial (R from 0.5 to 1.5, slightly curved walls), k the full circle of
    angles (periodic, no span shift: the angle wraps).  Uniform axial flow with
    a smooth perturbation; no boundary condition on the radial faces."""
    from ocfd_b200.params import BC_NONE, GRID2D_AXIAL_SYMM, default_params

    p = default_params()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.iperiodic[0], p.iperiodic[1], p.iperiodic[2] = 1, 0, 1
    p.periodic_span[0][0] = 2.0
    p.iflag_gridtype = GRID2D_AXIAL_SYMM
    p.ibc = BC_NONE
    p.scheme_invis = SCHEME_WENO7
    p.if_scheme_character = 1
    p.flux_splitting = SPLIT_SW
    p.ma, p.re, p.pr, p.gamma = 0.5, 1000.0, 0.7, 1.4
    p.dt = 1e-3
    p.hybrid_para[3] = 0.0
    i = np.arange(1, nx + 1)[None, :]
    j = np.arange(ny)[:, None]
    x2 = 2.0 * i / nx + 0.0 * j
    r2 = 0.5 + j / (ny - 1.0) + 0.05 * np.sin(np.pi * i / nx) * (j / (ny - 1.0))
    seta = 2.0 * np.pi * np.arange(nz) / nz
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    d = 1.0 + 0.02 * np.cos(2 * np.pi * ii / nx)
    u = 1.0 + 0.05 * np.sin(2 * np.pi * ii / nx) * np.cos(2 * np.pi * kk / nz)
    v = 0.03 * np.sin(np.pi * jj / ny) * np.sin(2 * np.pi * kk / nz)
    w = 0.02 * np.cos(2 * np.pi * ii / nx)
    T = 1.0 + 0.01 * np.cos(np.pi * jj / ny)
    return p, (x2, r2, seta), [d, u, v, w, T]
