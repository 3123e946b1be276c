"""The C oracle against a second, independent transcription of the reference
(oracle/npref.py, NumPy, written from the Fortran rather than from the C).

Both keep the Fortran operand order without fused multiply-adds, so they must
agree bit for bit: on random pencils through every reconstruction scheme,
splitting and boundary closure, on the characteristic L / R matrices, on the
CD6 / CD8 derivatives with their closures, and on whole right-hand sides
(du_inviscous, du_inviscous_Character, du_viscous) of small periodic and
body-fitted grids.  A constant or operand misread the same way in both would
still pass; a misreading in one of them does not."""
import ctypes as C

import numpy as np
import pytest

import npref
from ocfd_testlib import curvilinear_case, tgv_case
from ocfd_b200.params import (BC_BLUNT2D, BC_USER_DEF, SCHEME_HYBRID, SCHEME_OMP6, SCHEME_UD7L, SCHEME_WENO5,
                              SCHEME_WENO7, SPLIT_LLF, default_params)
from pyoracle import Oracle, char_matrices, lib

SCHEMES = [SCHEME_WENO5, SCHEME_WENO7, SCHEME_OMP6, SCHEME_UD7L, SCHEME_HYBRID]


def _pencil_oracle(scheme, bi, sb, n=16):
    p = default_params()
    p.nx, p.ny, p.nz = n, 8, 8
    p.scheme_invis = scheme
    p.iperiodic[0] = 0 if bi == 1 else 1
    p.scheme_boundary[0], p.scheme_boundary[1] = sb
    p.ud7l_diss = 0.3
    o = Oracle(p)
    return o


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("bnd", [(0, 0), (1, 0), (1, 1), (1, -1)], ids=["periodic", "sb0", "sb1", "sbm1"])
def test_flux_pencils(scheme, bnd):
    """OCFD2d_flux1/2 (OCFD_inviscous.f90:210-361) on random pencils."""
    bi, sb = bnd
    n = 16
    o = _pencil_oracle(scheme, bi, (sb, sb))
    rng = np.random.default_rng(100 * scheme + 10 * bi + sb + 1)
    U = [o.p.ud7l[q] for q in range(8)]
    for trial in range(6):
        f1d = rng.normal(size=n + 8) * (1.0 + 5.0 * (trial % 2)) + (3.0 if trial > 2 else 0.0)
        scm = rng.integers(1, 4, size=n + 1).astype(np.int32)
        for sign in (+1, -1):
            want = o.flux1d(f1d, sign, 0, scm)
            got = npref.flux_pencils(f1d[None], sign, scheme, (o.p.bound_index[0], o.p.bound_index[1]),
                                     (sb, sb), U, scm[None])[0]
            np.testing.assert_array_equal(got, want, err_msg=f"sign {sign} trial {trial}")
    o.close()


def test_char_matrices():
    """The L (S) and R (S1) matrices of flux_charteric (OCFD_inviscous_character.f90:
    216-248), both branches of the basis choice."""
    rng = np.random.default_rng(7)
    for t in range(40):
        uvwc = np.array([rng.normal(), rng.normal(), rng.normal(), 1.0 + rng.random()])
        a = rng.normal(size=3)
        if t % 2:
            a[2] *= 0.01  # |n3| <= |n2| branch
        else:
            a[1] *= 0.01
        S, S1 = char_matrices(1.4, uvwc, a)
        gS, gS1 = npref.char_basis(1.4, *[np.array([x]) for x in uvwc[:3]], np.array([uvwc[3]]),
                                   *[np.array([x]) for x in a])
        np.testing.assert_array_equal(np.array([[x[0] for x in r] for r in gS]), S)
        np.testing.assert_array_equal(np.array([[x[0] for x in r] for r in gS1]), S1)


@pytest.mark.parametrize("cd", [5, 6], ids=["cd6", "cd8"])
@pytest.mark.parametrize("periodic", [1, 0], ids=["periodic", "closed"])
def test_central_derivatives(cd, periodic):
    """OCFD_dx0/dy0/dz0 (OCFD_dxyz_viscous.f90:3-239) with the boundary closures."""
    p = default_params()
    p.nx, p.ny, p.nz = 14, 12, 10
    p.scheme_vis = cd
    for d in range(3):
        p.iperiodic[d] = periodic
    o = Oracle(p)
    rng = np.random.default_rng(cd + 10 * periodic)
    f = rng.normal(size=o.shape_h)
    for d in range(3):
        np.testing.assert_array_equal(npref.d0(o.p, f, d), o.d0(d, f), err_msg=f"direction {d}")
    o.close()


TGV = {
    "weno7_sw": dict(scheme=SCHEME_WENO7, character=0),
    "weno7_sw_char": dict(scheme=SCHEME_WENO7, character=1),
    "omp6_sw_char": dict(scheme=SCHEME_OMP6, character=1),
    "omp6_sw": dict(scheme=SCHEME_OMP6, character=0),
    "weno5_llf": dict(scheme=SCHEME_WENO5, character=0, split=SPLIT_LLF),
    "weno5_llf_char": dict(scheme=SCHEME_WENO5, character=1, split=SPLIT_LLF),
    "ud7l_sw_cd8": dict(scheme=SCHEME_UD7L, character=0, cd8=True),
    "hybrid1_llf": dict(scheme=SCHEME_HYBRID, character=0, split=SPLIT_LLF, ma=0.5),
    "hybrid1_sw_char": dict(scheme=SCHEME_HYBRID, character=1, ma=0.5),
}


def _state(o):
    return npref.State(o.p, [o.prim(q).copy() for q in range(5)], [m.copy() for m in o.metrics()], o.rhybrid.copy())


def _rhs_check(o, mass=False):
    """du of one stage of the oracle against npref on the same state."""
    o.halo_prims()
    if o.p.scheme_invis == SCHEME_HYBRID:
        o.comput_rhybrid()
    st = _state(o)
    if o.p.if_scheme_character:
        o.du_inviscous_character()
        want = npref.du_inviscous_character(st)
    else:
        o.du_inviscous()
        want = npref.du_inviscous(st)
    np.testing.assert_array_equal(want, o.du, err_msg="inviscid")
    o.du_viscous()
    np.testing.assert_array_equal(npref.du_viscous(st, want), o.du, err_msg="viscous")


@pytest.mark.parametrize("name", list(TGV))
def test_rhs_periodic(name):
    p, _, prims = tgv_case(**TGV[name], n=(16, 12, 10))
    o = Oracle(p)
    o.init_mesh()
    o.init3d(prims)
    o.step(1)  # a state that is no longer symmetric
    _rhs_check(o)
    o.close()


@pytest.mark.parametrize("bc,ghost,scheme,character",
                         [(BC_USER_DEF, True, SCHEME_WENO7, 1), (BC_BLUNT2D, False, SCHEME_WENO5, 1),
                          (BC_USER_DEF, False, SCHEME_OMP6, 0), (BC_BLUNT2D, True, SCHEME_WENO7, 0)])
def test_rhs_curvilinear(bc, ghost, scheme, character):
    """Body-fitted grid with wall and free-stream boundaries: every closure of the
    flux-vector and characteristic sweeps and of the viscous derivatives."""
    p, mesh, prims = curvilinear_case(bc=bc, ghost=ghost, scheme=scheme, character=character)
    o = Oracle(p)
    o.init_mesh(*mesh)
    o.init3d(prims)
    _rhs_check(o)
    o.close()


def test_rhs_mass_force():
    p, _, prims = tgv_case(scheme=SCHEME_WENO7, character=1, n=(16, 12, 10))
    p.if_mass_force = 1
    p.mass_force[0], p.mass_force[1], p.mass_force[2] = 0.3, -0.2, 0.15
    o = Oracle(p)
    o.init_mesh()
    o.init3d(prims)
    _rhs_check(o)
    o.close()
