"""Grid types 21 and 31 on the oracle alone (no GPU): the axisymmetric file
gives a valid right-handed grid, and a GRID_AND_JACOBIAN3D file holding the
metrics the oracle computed reproduces all 22 metric arrays bit for bit
(init_mesh, OCFD_mesh.f90:1-58: only comput_Jacobian3d is skipped)."""
import numpy as np

from ocfd_testlib import annulus_case, curvilinear_case, interior
from ocfd_b200 import fileio
from ocfd_b200.params import GRID2D_AXIAL_SYMM, GRID_AND_JACOBIAN3D
from pyoracle import Oracle


def test_axisymmetric_grid_oracle(tmp_path):
    p, (x2, r2, seta), _ = annulus_case()
    path = str(tmp_path / "OCFD-grid.dat")
    fileio.write_grid(path, GRID2D_AXIAL_SYMM, x2, r2, seta)
    X, Y, Z = fileio.read_grid(path, GRID2D_AXIAL_SYMM, p.nx, p.ny, p.nz)
    np.testing.assert_array_equal(np.hypot(Y, Z)[0], np.hypot(r2 * np.cos(seta[0]), r2 * np.sin(seta[0])))
    o = Oracle(p)
    o.init_mesh(X, Y, Z)
    J = interior(o.metric(12))
    assert np.all(np.isfinite(J)) and np.all(J > 0)
    # the radial metric row points along R: Aiy, Aiz proportional to (cos, sin) of the angle
    aiy, aiz = interior(o.metric(7)), interior(o.metric(8))
    ang = np.arctan2(aiz, aiy)
    want = np.broadcast_to(seta[:, None, None], ang.shape)
    dang = np.angle(np.exp(1j * (ang - want)))
    assert np.max(np.abs(dang)) < 0.05


def test_grid_and_jacobian_oracle(tmp_path):
    p, mesh, _ = curvilinear_case()
    o0 = Oracle(p)
    o0.init_mesh(*mesh)
    jac = [np.ascontiguousarray(interior(o0.metric(m))) for m in range(3, 13)]
    path = str(tmp_path / "OCFD-grid.dat")
    fileio.write_grid(path, GRID_AND_JACOBIAN3D, *mesh, jac=jac)
    p.iflag_gridtype = GRID_AND_JACOBIAN3D
    o = Oracle(p)
    o.init_mesh(*fileio.read_grid(path, GRID_AND_JACOBIAN3D, p.nx, p.ny, p.nz))
    for m in range(22):
        np.testing.assert_array_equal(o.metric(m), o0.metric(m), err_msg=f"metric {m}")
