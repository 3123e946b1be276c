"""BC_BoundaryLayer and BC_SweptCorner with their user-defined ghost cells
(GPU, through the C ABI) against the oracle: the strict build bit for bit, the
production build within 1e-10 relative L2, over several steps, for the inlet
data (1-D and 2-D), the wall perturbation varying in time, isothermal and
adiabatic walls, both outlet extrapolations and the upper-boundary modes."""
import numpy as np
import pytest

from ocfd_b200.solver import Solver
from ocfd_testlib import boundary_layer_case, rel_l2
from pyoracle import Oracle

pytestmark = pytest.mark.gpu

CASES = {
    "bl": dict(kind="bl"),
    "bl-ghost": dict(kind="bl", ghost=True),
    "bl-isothermal-2d-inlet": dict(kind="bl", tw=2.0, inlet_2d=True, outlet=1),
    "bl-dirichlet-upper-still": dict(kind="bl", nonref=2, pert=False),
    "sc": dict(kind="sc", n=(24, 20, 12)),
    "sc-isothermal": dict(kind="sc", tw=2.0, outlet=1, n=(24, 20, 12)),
}


def _run(cls, case, steps, strict=None):
    p, X, prims, data = boundary_layer_case(**case)
    s = cls(p) if strict is None else cls(p, strict=strict)
    s.init_mesh(*X)
    s.set_bc_layer(data)
    s.init3d(prims)
    s.step(steps)
    if cls is Oracle:
        out = s.f.copy(), [s.prim(q).copy() for q in range(5)]
    else:
        out = s.download_state()
    s.close()
    return out


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("strict", [True, False], ids=["strict", "fast"])
def test_boundary_layer_bc_matches_oracle(name, strict):
    f_ref, pr_ref = _run(Oracle, CASES[name], 4)
    f, pr = _run(Solver, CASES[name], 4, strict=strict)
    if strict:
        np.testing.assert_array_equal(f, f_ref)
        for a, b in zip(pr, pr_ref):
            inner = (slice(4, -4),) * 3
            np.testing.assert_array_equal(a[inner], b[inner])
    assert rel_l2(f, f_ref) < 1e-10


def test_boundary_layer_metric_ghost_mirror():
    """Jac_Ghost_flatplate: the j- ghost metrics mirror the interior about y = 0
    (strict build against the oracle, bit for bit, on the ghost rows)."""
    p, X, prims, data = boundary_layer_case("bl", ghost=True)
    s = Solver(p, strict=True)
    s.init_mesh(*X)
    m = s.download_metrics()
    s.close()
    o = Oracle(p)
    o.init_mesh(*X)
    ghost = (slice(4, -4), slice(0, 4), slice(4, -4))  # k, j = -3..0, i interior
    for q in range(22):
        np.testing.assert_array_equal(m[q][ghost], o.metric(q)[ghost])
    o.close()
    # Aky (4) flips sign, Akx (3) does not: j = 0 mirrors j = 2
    np.testing.assert_array_equal(m[4][4:-4, 3, 4:-4], -m[4][4:-4, 5, 4:-4])
    np.testing.assert_array_equal(m[3][4:-4, 3, 4:-4], m[3][4:-4, 5, 4:-4])
