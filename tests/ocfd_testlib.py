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
