"""The C++ host driver (in place of the reference's Fortran main program) and
the reference's file formats, without a GPU: the driver reads a deck like the
Python reader does, and flow / grid files written by either host read back
bit-exactly in the other."""
import json
import os
import subprocess

import numpy as np
import pytest

from ocfd_b200 import fileio
from ocfd_b200.params import (GRID1D, GRID2D_AXIAL_SYMM, GRID2D_PLANE, GRID3D, GRID_AND_JACOBIAN3D, read_namelist,
                              set_parameters_py)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
PKG = os.path.join(ROOT, "opencfd-sc_b200")
DRIVER = os.path.join(PKG, "host", "ocfd_sc")


@pytest.fixture(scope="module")
def driver():
    subprocess.run(["make", "-s", "host/ocfd_sc"], cwd=PKG, check=True)
    return DRIVER


@pytest.mark.parametrize("deck", ["deck_tgv.in", "deck_blunt.in"])
def test_driver_reads_decks_like_python(driver, deck):
    out = subprocess.run([driver, "--print-params", "--deck", os.path.join(GOLDEN, deck)], check=True,
                         capture_output=True, text=True).stdout
    c = json.loads(out)
    p = set_parameters_py(read_namelist(os.path.join(GOLDEN, deck)))
    for k in ("nx", "ny", "nz", "iflag_gridtype", "scheme_invis", "scheme_vis", "if_scheme_character",
              "flux_splitting", "ibc", "if_viscous", "nfiltering", "istep_show", "istep_save"):
        assert c[k] == getattr(p, k), k
    for k in ("ma", "re", "gamma", "pr", "dt", "end_time", "hx", "cv", "cp"):
        assert c[k] == getattr(p, k), k
    assert c["iperiodic"] == list(p.iperiodic)
    assert c["scheme_boundary"] == list(p.scheme_boundary)
    assert c["ghost_cell"] == list(p.ghost_cell)
    assert c["hybrid_para"] == [p.hybrid_para[i] for i in range(3)]


def test_driver_rejects_unknown_scheme(driver, tmp_path):
    deck = tmp_path / "bad.in"
    deck.write_text(open(os.path.join(GOLDEN, "deck_tgv.in")).read().replace('"omp6"', '"WENO9"'))
    r = subprocess.run([driver, "--print-params", "--deck", str(deck)], capture_output=True, text=True)
    assert r.returncode != 0 and "not supported" in r.stderr


def test_driver_flow_file_reads_in_python(driver, tmp_path):
    subprocess.run([driver, "--io-selftest", str(tmp_path)], check=True, capture_output=True)
    istep, tt, q = fileio.read_flow(str(tmp_path / "OCFD00000007.dat"), 5, 4, 3)
    assert istep == 7 and tt == 0.035
    c = np.arange(60, dtype=np.float64).reshape(3, 4, 5)
    for v in range(5):
        np.testing.assert_array_equal(q[v], 0.25 * v + 1e-3 * c)


def test_flow_file_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    prims = [rng.normal(size=(6, 5, 7)) for _ in range(5)]
    path = str(tmp_path / "OCFD00000100.dat")
    fileio.write_flow(path, 100, 0.5, prims)
    # 1 header record + 5 * nz plane records, each framed by two 4-byte markers
    assert os.path.getsize(path) == (12 + 8) + 5 * 6 * (5 * 7 * 8 + 8)
    istep, tt, back = fileio.read_flow(path, 7, 5, 6)
    assert (istep, tt) == (100, 0.5)
    for a, b in zip(prims, back):
        np.testing.assert_array_equal(a, b)
    with pytest.raises(ValueError):
        fileio.read_flow(path, 6, 5, 6)


def _grid_case(gridtype, nx=6, ny=5, nz=4):
    """Grid-file contents (x, y, z[, jac]) of a type and the expanded (nz, ny, nx)
    arrays init_mesh receives."""
    rng = np.random.default_rng(gridtype)
    jac = None
    if gridtype == GRID1D:
        x, y, z = rng.normal(size=nx), rng.normal(size=ny), rng.normal(size=nz)
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    elif gridtype in (GRID2D_PLANE, GRID2D_AXIAL_SYMM):
        x, y, z = rng.normal(size=(ny, nx)), rng.normal(size=(ny, nx)), rng.normal(size=nz)
        X = np.broadcast_to(x, (nz, ny, nx))
        if gridtype == GRID2D_PLANE:
            Y = np.broadcast_to(y, (nz, ny, nx))
            Z = np.broadcast_to(z[:, None, None], (nz, ny, nx))
        else:  # y holds R, z the angle: y = R cos(seta), z = R sin(seta)
            Y = y[None] * np.cos(z)[:, None, None]
            Z = y[None] * np.sin(z)[:, None, None]
    else:
        X, Y, Z = (rng.normal(size=(nz, ny, nx)) for _ in range(3))
        x, y, z = X, Y, Z
        if gridtype == GRID_AND_JACOBIAN3D:
            jac = [rng.normal(size=(nz, ny, nx)) for _ in range(10)]
    return (x, y, z, jac), (X, Y, Z, jac)


@pytest.mark.parametrize("gridtype", [GRID1D, GRID2D_PLANE, GRID2D_AXIAL_SYMM, GRID3D, GRID_AND_JACOBIAN3D])
def test_grid_file_round_trip(tmp_path, gridtype):
    nx, ny, nz = 6, 5, 4
    (x, y, z, jac), (X, Y, Z, J) = _grid_case(gridtype, nx, ny, nz)
    path = str(tmp_path / "OCFD-grid.dat")
    fileio.write_grid(path, gridtype, x, y, z, jac=jac)
    got = fileio.read_grid(path, gridtype, nx, ny, nz)
    assert len(got) == (4 if gridtype == GRID_AND_JACOBIAN3D else 3)
    for a, b in zip(got[:3], (X, Y, Z)):
        np.testing.assert_array_equal(a, b)
    if J is not None:
        for a, b in zip(got[3], J):
            np.testing.assert_array_equal(a, b)
    if gridtype == GRID_AND_JACOBIAN3D:
        with pytest.raises(ValueError):
            fileio.write_grid(path, gridtype, x, y, z)


@pytest.mark.parametrize("gridtype", [GRID2D_AXIAL_SYMM, GRID_AND_JACOBIAN3D])
def test_driver_reads_grid_files_like_python(driver, tmp_path, gridtype):
    """The C++ host reads a grid file written by the Python host into the same
    coordinates (bit for bit; the axisymmetric y and z within an ulp, since the
    two evaluate cos and sin with different libraries) and metric arrays."""
    nx, ny, nz = 7, 6, 5
    (x, y, z, jac), _ = _grid_case(gridtype, nx, ny, nz)
    path = str(tmp_path / "OCFD-grid.dat")
    fileio.write_grid(path, gridtype, x, y, z, jac=jac)
    out = str(tmp_path / "dump.bin")
    subprocess.run([driver, "--grid-dump", str(gridtype), str(nx), str(ny), str(nz), path, out], check=True)
    got = np.fromfile(out, dtype="<f8").reshape(-1, nz, ny, nx)
    want = fileio.read_grid(path, gridtype, nx, ny, nz)
    arrays = list(want[:3]) + (list(want[3]) if gridtype == GRID_AND_JACOBIAN3D else [])
    assert got.shape[0] == len(arrays)
    np.testing.assert_array_equal(got[0], arrays[0])
    for a, b in zip(got[1:], arrays[1:]):
        if gridtype == GRID2D_AXIAL_SYMM:
            np.testing.assert_allclose(a, b, rtol=4.5e-16, atol=1e-300)
        else:
            np.testing.assert_array_equal(a, b)
