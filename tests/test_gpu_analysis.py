"""The analyses of OCFD_analysis on the device (GPU, through the C ABI) against
the oracle -- Q criterion, running time average, corner wall statistics, box
download -- strict build bit for bit; and the host dispatcher writing the
reference's files from a deck's ANA_Para."""
import os

import numpy as np
import pytest

from ocfd_b200 import analysis, fileio
from ocfd_b200.solver import Solver
from ocfd_testlib import boundary_layer_case, curvilinear_case, interior, tgv_case
from pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _pair(p, X, prims, strict=True, data=None):
    s = Solver(p, strict=strict)
    o = Oracle(p)
    for x in (s, o):
        if X is None:
            x.init_mesh()
        else:
            x.init_mesh(*X)
        if data is not None:
            x.set_bc_layer(data)
        x.init3d(prims)
    return s, o


@pytest.mark.parametrize("case", ["tgv", "curvilinear"])
def test_q_criterion_and_time_average(case):
    if case == "tgv":
        p, X, prims = tgv_case()
    else:
        p, X, prims = curvilinear_case()
    s, o = _pair(p, X, prims)
    mean = np.zeros((5, p.nz, p.ny, p.nx))
    for k in range(3):
        s.step(1)
        o.step(1)
        s.ana_time_average()
        o.ana_time_average(mean, k)
    np.testing.assert_array_equal(s.ana_q(), o.ana_q())
    got, kk, tt = s.download_average()
    assert kk == 3 and tt == 3 * p.dt
    for q in range(5):
        np.testing.assert_array_equal(got[q], mean[q])
    # the means restart from an uploaded state
    s.upload_average(got, kk, tt)
    s.ana_time_average()
    o.ana_time_average(mean, 3)
    np.testing.assert_array_equal(s.download_average()[0][4], mean[4])
    s.close()
    o.close()


def test_corner_statistics_and_block():
    p, X, prims, data = boundary_layer_case("bl", pert=False)
    s, o = _pair(p, X, prims, data=data)
    s.step(2)
    o.step(2)
    np.testing.assert_array_equal(s.ana_corner(), o.ana_corner())
    blk = s.download_block(3, 7, 2, 5, 1, 4)
    for q in range(5):
        np.testing.assert_array_equal(blk[q], interior(o.prim(q))[0:4, 1:5, 2:7])
    s.close()
    o.close()


def test_analysis_dispatcher_writes_reference_files(tmp_path):
    p, X, prims = tgv_case()
    deck = """ $control_opencfd
 ANA_Number=4
 ANA_Para(1,1)=101, 2
 ANA_Para(1,2)=102, 1
 ANA_Para(1,3)=100, 1, 2
 ANA_Para(1,4)=103, 2, 5, 3, 4, 1, 2, 2, 7, 2
 $end
"""
    entries = analysis.read_analysis(deck, is_text=True)
    s = Solver(p)
    s.init_mesh()
    s.init3d(prims)
    ana = analysis.Analysis(s, entries, outdir=str(tmp_path))
    for _ in range(2):
        s.step(1)
        ana.run()
    q = s.ana_q()
    with open(tmp_path / "Q-0000002.dat", "rb") as fh:
        for k in range(p.nz):
            np.testing.assert_array_equal(np.frombuffer(fileio._read_record(fh, p.nx * p.ny * 8)).reshape(p.ny, p.nx),
                                          q[k])
    rows = open(tmp_path / "statistics.dat").read().splitlines()
    assert len(rows) == 2 and len(rows[0]) == 400
    means, k_avg, t_avg = s.download_average()
    with open(tmp_path / "OCFD00000002.dat.average", "rb") as fh:
        r1 = fileio._read_record(fh, 12)
        assert np.frombuffer(r1[:4], "<i4")[0] == k_avg == 2
        a = np.frombuffer(fileio._read_record(fh, p.nx * p.ny * 8)).reshape(p.ny, p.nx)
        np.testing.assert_array_equal(a, means[0][0])
    blk = s.download_block(3, 4, 1, 2, 2, 7)
    with open(tmp_path / "savedata-block002.dat", "rb") as fh:
        fileio._read_record(fh, 12)
        d = np.frombuffer(fileio._read_record(fh, blk[0].size * 8)).reshape(blk[0].shape)
        np.testing.assert_array_equal(d, blk[0])
    assert os.path.exists(tmp_path / "savedata-block002.dat")
    s.close()
