"""Full-length parity on the named configurations (GPU, through the C ABI).

Config 1 -- TGV 64^3, flux-vector WENO7, SW, CD6, dt = 0.005, 100 steps: the
strict build is bit-identical to the oracle after all 100 steps and the
production build within 1e-10 relative L2 (the stated FP64 bar); the
kinetic-energy history (show_flow_msg every 10 steps) agrees to 1e-12.
Mixed precision on the characteristic OMP6 TGV: relative kinetic-energy error
below 1e-5 against the FP64 run (the stated mixed-precision bar).
"""
import os

import numpy as np
import pytest

from ocfd_b200 import cases
from ocfd_b200.params import SCHEME_OMP6, SCHEME_WENO7
from ocfd_b200.solver import Solver
from ocfd_testlib import rel_l2
from pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _config1():
    return cases.tgv_params(64, scheme=SCHEME_WENO7, character=0, dt=0.005, steps=100)


@pytest.fixture(scope="module")
def oracle_config1():
    p = _config1()
    o = Oracle(p)
    o.init_mesh()
    o.init3d(cases.tgv_prims(o.p))
    ke = []
    for _ in range(10):
        o.step(10)
        ke.append(o.show_flow_msg()[1])
    f = o.f.copy()
    o.close()
    return f, np.array(ke)


@pytest.mark.parametrize("strict", [True, False], ids=["strict", "fast"])
def test_config1_tgv64_weno7_100_steps(oracle_config1, strict):
    f_ref, ke_ref = oracle_config1
    p = _config1()
    s = Solver(p, strict=strict)
    s.init_mesh()
    s.init3d(cases.tgv_prims(s.p))
    ke = []
    for _ in range(10):
        s.step(10)
        ke.append(s.show_flow_msg()[1])
    f = s.download_f()
    s.close()
    if strict:
        np.testing.assert_array_equal(f, f_ref)
    err = rel_l2(f, f_ref)
    assert err < 1e-10, err
    assert np.max(np.abs(np.array(ke) - ke_ref) / ke_ref) < 1e-12


def test_mixed_precision_kinetic_energy_error():
    n, steps = 64, 100
    out = {}
    for mixed in (0, 1):
        p = cases.tgv_params(n, scheme=SCHEME_OMP6, character=1, dt=0.002, steps=steps)
        p.precision = mixed
        s = Solver(p)
        s.init_mesh()
        s.init3d(cases.tgv_prims(s.p))
        s.step(steps)
        out[mixed] = (s.show_flow_msg()[1], s.download_f())
        s.close()
    ke_err = abs(out[1][0] - out[0][0]) / out[0][0]
    assert ke_err < 1e-5, ke_err
    assert rel_l2(out[1][1], out[0][1]) < 1e-5
