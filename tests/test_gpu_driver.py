"""The C++ host driver end to end on the GPU: a deck, a grid file and a restart
file in the working directory, as the reference's program reads them
(read_parameter, init_mesh with Iflag_Gridtype = 10, read_flow_data); the flow
files it saves match the oracle run from the same inputs (production build,
FP64 bar 1e-10 relative L2) and carry the reference's Istep/tt header."""
import os
import subprocess

import numpy as np
import pytest

from ocfd_b200 import cases, fileio
from ocfd_b200.params import GRID1D, read_namelist
from ocfd_testlib import interior, rel_l2
from pyoracle import Oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "opencfd-sc_b200")

DECK = """ $control_opencfd
 nx_global=24
 ny_global=20
 nz_global=16
 Iflag_Gridtype=10
 Scheme_Invis="WENO7"
 Scheme_Vis="CD6"
 IF_Scheme_Character=1
 Ma=0.3
 Re=1600.0
 BoundaryCondition="BC_NONE"
 Istep_show=2
 Istep_save=2
 dt=0.004
 End_time=1.0
 Iperiodic_X=1
 Iperiodic_Y=1
 Iperiodic_Z=1
 Periodic_ISpan= 6.2831853071795864, 0., 0.
 Periodic_JSpan= 0., 6.2831853071795864, 0.
 Periodic_KSpan= 0., 0., 6.2831853071795864
 $end
"""


def test_driver_restart_run_matches_oracle(tmp_path):
    subprocess.run(["make", "-s", "host/ocfd_sc"], cwd=PKG, check=True)
    (tmp_path / "opencfd2.in").write_text(DECK)
    p = read_namelist(str(tmp_path / "opencfd2.in"))
    x, y, z = cases.box_coords(p.nx, p.ny, p.nz)
    fileio.write_grid(str(tmp_path / "OCFD-grid.dat"), GRID1D, x, y, z)
    prims = cases.tgv_prims(cases.tgv_params(24, ny=20, nz=16, ma=0.3))
    rng = np.random.default_rng(5)
    prims = [q + 1e-3 * rng.normal(size=q.shape) for q in prims]
    fileio.write_flow(str(tmp_path / "opencfd.dat"), 10, 0.04, prims)

    r = subprocess.run([os.path.join(PKG, "host", "ocfd_sc"), "--steps", "4"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Kinetic-energy" in r.stdout and "The END" in r.stdout

    o = Oracle(p)
    o.init_mesh(*fileio.read_grid(str(tmp_path / "OCFD-grid.dat"), GRID1D, p.nx, p.ny, p.nz))
    o.init3d(prims)
    o.set_time(10, 0.04)
    for istep in (12, 14):
        o.step(2)
        got_step, tt, q = fileio.read_flow(str(tmp_path / f"OCFD{istep:08d}.dat"), p.nx, p.ny, p.nz)
        assert got_step == istep and abs(tt - (0.04 + (istep - 10) * 0.004)) < 1e-12
        for v in range(5):
            ref = interior(o.prim(v))
            assert rel_l2(q[v], ref) < 1e-10, (istep, v)
    o.close()


def test_driver_analysis_files_match_python_host(tmp_path):
    """ANA_Para in the deck: the C++ driver runs OCFD_analysis after each step
    (Q criterion, statistics.dat, time averages with restart-file output,
    plane and block savedata) and writes the same bytes as the Python host's
    analysis schedule over the same library."""
    from ocfd_b200 import analysis
    from ocfd_b200.solver import Solver

    subprocess.run(["make", "-s", "host/ocfd_sc"], cwd=PKG, check=True)
    deck = DECK.replace(" $end", """ ANA_Number=5
 ANA_Para(1,1)=101, 2
 ANA_Para(1,2)=102, 1
 ANA_Para(1,3)=100, 1, 2
 ANA_Para(1,4)=103, 2, 5, 3, 6, 2, 5, 1, 3, 7
 ANA_Para(1,5)=103, 2, 3, 2, 1, 4, 9
 $end""")
    run_dir, py_dir = tmp_path / "drv", tmp_path / "py"
    run_dir.mkdir()
    py_dir.mkdir()
    (run_dir / "opencfd2.in").write_text(deck)
    p = read_namelist(str(run_dir / "opencfd2.in"))
    x, y, z = cases.box_coords(p.nx, p.ny, p.nz)
    fileio.write_grid(str(run_dir / "OCFD-grid.dat"), GRID1D, x, y, z)
    prims = cases.tgv_prims(cases.tgv_params(24, ny=20, nz=16, ma=0.3))
    fileio.write_flow(str(run_dir / "opencfd.dat"), 10, 0.04, prims)
    r = subprocess.run([os.path.join(PKG, "host", "ocfd_sc"), "--steps", "4"], cwd=run_dir,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

    s = Solver(p)
    s.init_mesh(*fileio.read_grid(str(run_dir / "OCFD-grid.dat"), GRID1D, p.nx, p.ny, p.nz))
    s.init3d(prims, 10, 0.04)
    ana = analysis.Analysis(s, analysis.read_analysis(deck, is_text=True), outdir=str(py_dir))
    for _ in range(4):
        s.step(1)
        ana.run()
    s.close()
    names = sorted(f.name for f in py_dir.iterdir())
    assert "Q-0000012.dat" in names and "statistics.dat" in names and "OCFD00000012.dat.average" in names
    assert "savedata-block007.dat" in names and "savedata-XY001.dat" in names
    for name in names:
        assert (run_dir / name).read_bytes() == (py_dir / name).read_bytes(), name
