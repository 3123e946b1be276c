"""Full-length parity on the named configurations (GPU, through the C ABI).

Config 1 -- TGV 64^3, flux-vector WENO7, SW, CD6, dt = 0.005, 100 steps: the
strict build is bit-identical to the oracle after all 100 steps and the
production build within 1e-10 relative L2 (the stated FP64 bar); the
kinetic-energy history (show_flow_msg every 10 steps) agrees to 1e-12.
Mixed precision on the characteristic OMP6 TGV: relative kinetic-energy error
below 1e-5 against the FP64 run (the stated mixed-precision bar).

Config 4 at its stated size -- the Mach 6 cylinder, 301 x 401 x 8 body-fitted
grid, characteristic WENO7, isothermal wall -- 10 steps against the oracle:
strict build bit-identical, production build within 1e-10 relative L2.
Config 3's set-up on 128^3 (isotropic turbulence, hybrid sensor 1, LLF,
flux-vector form, dt at CFL 0.5) -- 5 steps against the oracle, the same bars.
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


def _run_pair(p, mesh, prims, steps):
    """The oracle's state after `steps` steps, then the two builds'."""
    o = Oracle(p)
    o.init_mesh(*mesh)
    o.init3d(prims)
    o.step(steps)
    ref = o.f.copy()
    o.close()
    out = {}
    for strict in (True, False):
        s = Solver(p, strict=strict)
        s.init_mesh(*mesh)
        s.init3d(prims)
        s.step(steps)
        out[strict] = s.download_f()
        s.close()
    return ref, out


def test_config4_cylinder_full_size_10_steps():
    p = cases.cylinder_params()
    ref, out = _run_pair(p, cases.cylinder_grid(p.nx, p.ny, p.nz), cases.cylinder_prims(p.nx, p.ny, p.nz), 10)
    np.testing.assert_array_equal(out[True], ref)
    err = rel_l2(out[False], ref)
    assert err < 1e-10, err


def test_config3_isotropic_turbulence_128_5_steps():
    import math

    n, ma = 128, 1.0
    prims = cases.hit_prims(n, mt=0.6, ma=ma)
    vmax = float(np.max(np.abs(prims[1]) + np.abs(prims[2]) + np.abs(prims[3]) + np.sqrt(prims[4]) / ma))
    p = cases.hit_params(n, re=1000.0, ma=ma, dt=0.5 * (2.0 * math.pi / n) / vmax)
    ref, out = _run_pair(p, cases.hit_coords(n), prims, 5)
    np.testing.assert_array_equal(out[True], ref)
    err = rel_l2(out[False], ref)
    assert err < 1e-12, err
