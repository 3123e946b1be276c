"""Grid types read from OCFD-grid.dat on the GPU against the oracle (through the
C ABI): the axisymmetric plane grid (Iflag_Gridtype 21, read_mesh2d_AxialSymm,
OCFD_mesh.f90:286-317) and the 3-D grid with its metrics and Jacobian in the
file (Iflag_Gridtype 31, read_mesh3d with comput_Jacobian3d skipped,
OCFD_mesh.f90:11,24-26,187-217).  Strict build: the 22 metric arrays and the
state after three time steps are bit-identical to the oracle; production
build: metrics within 1e-13 of the largest component of their row, state
within 1e-12 relative L2."""
import numpy as np
import pytest

from ocfd_testlib import annulus_case, curvilinear_case, interior, rel_l2
from ocfd_b200 import fileio
from ocfd_b200.params import GRID2D_AXIAL_SYMM, GRID_AND_JACOBIAN3D
from ocfd_b200.solver import Solver
from pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _run(p, mesh, prims, strict):
    o = Oracle(p)
    o.init_mesh(*mesh)
    o.init3d(prims)
    s = Solver(p, strict=strict)
    s.init_mesh(*mesh)
    s.init3d(prims)
    return o, s


# metric arrays compared on a common scale: the three components of a row
# (an analytically zero component holds rounding noise only)
GROUPS = [(0,), (1,), (2,), (3, 4, 5), (6, 7, 8), (9, 10, 11), (12,), (13, 14, 15), (16, 17, 18), (19, 20, 21)]


def _check_pair(o, s, strict):
    mg = s.download_metrics()
    for grp in GROUPS:
        scale = max(float(np.max(np.abs(interior(o.metric(m))))) for m in grp)
        for m in grp:
            a, b = interior(mg[m]), interior(o.metric(m))
            if strict:
                np.testing.assert_array_equal(a, b, err_msg=f"metric {m}")
            else:
                err = float(np.max(np.abs(a - b))) / scale
                assert err <= 1e-13, (m, err)
    o.step(3)
    s.step(3)
    f = s.download_f()
    if strict:
        np.testing.assert_array_equal(f, o.f)
    else:
        assert rel_l2(f, o.f) < 1e-12, rel_l2(f, o.f)


@pytest.mark.parametrize("strict", [True, False], ids=["strict", "fast"])
def test_axisymmetric_grid_file(tmp_path, strict):
    p, (x2, r2, seta), prims = annulus_case()
    path = str(tmp_path / "OCFD-grid.dat")
    fileio.write_grid(path, GRID2D_AXIAL_SYMM, x2, r2, seta)
    mesh = fileio.read_grid(path, GRID2D_AXIAL_SYMM, p.nx, p.ny, p.nz)
    o, s = _run(p, mesh, prims, strict)
    # positive Jacobian everywhere (x along i, R along j, the angle along k: right-handed)
    assert np.all(interior(o.metric(12)) > 0)
    _check_pair(o, s, strict)


@pytest.mark.parametrize("strict", [True, False], ids=["strict", "fast"])
def test_grid_and_jacobian_file(tmp_path, strict):
    """The metrics the oracle computes for the body-fitted cylinder grid, written
    with the coordinates as an Iflag_Gridtype 31 file: read back, they give the
    same 22 arrays as the computed ones, and the same steps."""
    p, mesh, prims = curvilinear_case()
    o0 = Oracle(p)
    o0.init_mesh(*mesh)
    jac = [np.ascontiguousarray(interior(o0.metric(m))) for m in range(3, 13)]
    ref = [o0.metric(m).copy() for m in range(22)]
    o0.close()
    path = str(tmp_path / "OCFD-grid.dat")
    fileio.write_grid(path, GRID_AND_JACOBIAN3D, *mesh, jac=jac)
    p.iflag_gridtype = GRID_AND_JACOBIAN3D
    x, y, z, jac_back = fileio.read_grid(path, GRID_AND_JACOBIAN3D, p.nx, p.ny, p.nz)
    o, s = _run(p, (x, y, z, jac_back), prims, strict)
    for m in range(22):
        np.testing.assert_array_equal(interior(o.metric(m)), interior(ref[m]), err_msg=f"metric {m}")
    _check_pair(o, s, strict)
