"""BC_BoundaryLayer / BC_SweptCorner without a GPU: the host data of
ocfd_b200.bclayer (file formats, wall perturbation, time factor) and the
oracle's boundary values against the formulas of OCFD_BC_Boundarylayers.f90."""
import math

import numpy as np
import pytest

from ocfd_b200 import _lib, bclayer
from ocfd_testlib import boundary_layer_case
from pyoracle import Oracle
import ctypes as C

LAP = 4


def test_profile_and_plane_files_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    prof = rng.normal(size=(7, 5))
    prof[:, 3] = 0.0  # w is not stored in the 1-D files
    bclayer.write_profile_1d(str(tmp_path / "flow1d-inlet.dat"), np.arange(7.0), prof)
    np.testing.assert_array_equal(bclayer.read_profile_1d(str(tmp_path / "flow1d-inlet.dat"), 7), prof)
    plane = rng.normal(size=(5, 4, 6))
    bclayer.write_plane_2d(str(tmp_path / "flow2d-upper.dat"), plane)
    np.testing.assert_array_equal(bclayer.read_plane_2d(str(tmp_path / "flow2d-upper.dat"), 6, 4), plane)


def test_wall_perturbation_and_time_factor():
    x = np.tile(np.linspace(0.0, 1.0, 11), (4, 1))
    z = np.tile(np.linspace(0.0, 0.3, 4)[:, None], (1, 11))
    rng = np.random.default_rng(2)
    w = bclayer.wall_perturbation(1, x, z, 0.2, 0.8, 0, 1.0, rng)
    # mz = 0: gz = 1, fx = 4/sqrt(27) sin(s)(1 - cos(s)), zero outside [xbegin, xend]
    s = 2.0 * bclayer.PI * (x[0] - 0.2) / 0.6
    fx = np.where((x[0] >= 0.2) & (x[0] <= 0.8), 4.0 / math.sqrt(27.0) * np.sin(s) * (1.0 - np.cos(s)), 0.0)
    np.testing.assert_allclose(w[0], fx, atol=1e-14)
    assert np.abs(w).max() <= 1.0 + 1e-12
    tm, fait = bclayer.time_factor(4, rng)
    assert abs(tm.sum() - 1.0) < 1e-15 and np.allclose(tm[1:] / tm[:-1], 1.0 / 1.25)
    assert ((fait >= 0.0) & (fait < 1.0)).all()


@pytest.mark.parametrize("tw", [-1.0, 2.0])
def test_oracle_boundary_layer_values(tw):
    p, X, prims, data = boundary_layer_case("bl", tw=tw, outlet=2)
    o = Oracle(p)
    o.init_mesh(*X)
    o.set_bc_layer(data)
    o.init3d(prims)
    d, u, v, T = o.prim(0), o.prim(1), o.prim(2), o.prim(4)
    L = LAP
    # inlet i = 1 from the data (the wall condition, applied later, owns j = 1)
    np.testing.assert_array_equal(d[L:-L, L + 1:-L, L], data.inlet[0][:, 1:])
    np.testing.assert_array_equal(T[L:-L, L + 1:-L, L], data.inlet[4][:, 1:])
    # wall j = 1: blowing/suction along the wall normal, ht at t = 0
    ht = sum(data.tm[m] * math.sin((m + 1) * data.beta * 0.0 + 2.0 * bclayer.PI * data.fait[m])
             for m in range(len(data.tm)))
    A = p.bc_para[7]
    aix, aiy = o.metric(6), o.metric(7)
    k, i = 1, 10
    h = (k + L, L, i + L)
    nrm = 1.0 / math.sqrt(aix[h] ** 2 + aiy[h] ** 2 + o.metric(8)[h] ** 2)
    assert v[h] == A * ht * data.pertb[k, i] * aiy[h] * nrm
    if tw > 0:
        assert T[h] == tw
    else:
        assert T[h] == (4.0 * T[k + L, L + 1, i + L] - T[k + L, L + 2, i + L]) / 3.0
    # outlet i = nx: second-order extrapolation
    nx = p.nx
    np.testing.assert_array_equal(u[L:-L, L:-L, nx - 1 + L],
                                  2.0 * u[L:-L, L:-L, nx - 2 + L] - u[L:-L, L:-L, nx - 3 + L])
    o.close()


def test_oracle_swept_corner_side_and_ghost():
    p, X, prims, data = boundary_layer_case("sc", n=(24, 20, 12))
    o = Oracle(p)
    o.init_mesh(*X)
    o.set_bc_layer(data)
    o.init3d(prims)
    w, d = o.prim(3), o.prim(0)
    L = LAP
    nz = p.nz
    # k = nz copies k = nz - 1 (BC_Para(12) = 1)
    np.testing.assert_array_equal(d[nz - 1 + L, L:-L, L:-L], d[nz - 2 + L, L:-L, L:-L])
    # k- ghost cells mirror the first planes, w changes sign
    for g in range(1, L + 1):
        np.testing.assert_array_equal(w[L - g, L:-L, L:-L], -w[L + g - 1, L:-L, L:-L])
        np.testing.assert_array_equal(d[L - g, L:-L, L:-L], d[L + g - 1, L:-L, L:-L])
    o.close()


def test_library_accepts_and_rejects_boundary_layer_decks():
    p, X, prims, data = boundary_layer_case("bl")
    q = p.copy()
    assert _lib.lib().ocfd_set_parameters(C.byref(q)) == 0
    q = p.copy()
    q.iperiodic[1] = 1  # the wall and the upper boundary need a non-periodic j
    assert _lib.lib().ocfd_set_parameters(C.byref(q)) == _lib.OCFD_E_PARAM
    q = p.copy()
    q.ghost_cell[2] = -2
    assert _lib.lib().ocfd_set_parameters(C.byref(q)) == _lib.OCFD_E_PARAM


def test_analysis_deck_and_statistics_format():
    from ocfd_b200 import analysis

    deck = """ $control_opencfd
 nx_global=16
 ANA_Number=2
 ANA_Para(1,1)=100, 10, 50
 ANA_Para(1,2)=103, 5, 1, 2, 1, 3, 7
 $end
"""
    e = analysis.read_analysis(deck, is_text=True)
    assert [(c, k) for c, k, _ in e] == [(100, 10), (103, 5)]
    assert list(e[1][2][:5]) == [1.0, 2.0, 1.0, 3.0, 7.0]
    # '(20(E20.13E2))' of the statistics.dat row (OCFD_ANA.f90:307)
    assert analysis.fortran_e(30.6443393820) == " 0.3064433938200E+02"
    assert analysis.fortran_e(-1.2345e-4) == "-0.1234500000000E-03"
