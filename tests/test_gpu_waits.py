"""Bounded device waits (GPU, through the C ABI): the TMA-staged face sweeps
wait on an mbarrier for their tile copies with an iteration limit.  A host-side
test switch (OCFD_TEST_STALL_TMA=1, read when the sweep arguments are built)
makes every wait unreachable -- the staging expects 16 bytes more than its
copies deliver -- so the blocks must give up, record error 4 and leave.  The
step then reports OCFD_E_TIMEOUT instead of hanging or faulting, the instance
stages its tiles with plain loads from then on, and restarted from the initial
field it gives the same bits as a fresh instance (plain and TMA-staged sweeps
compute the same arithmetic)."""
import numpy as np
import pytest

from ocfd_b200 import cases
from ocfd_b200._lib import OCFD_E_TIMEOUT, OcfdError
from ocfd_b200.params import SCHEME_OMP6
from ocfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _solver(p, prims):
    s = Solver(p)
    s.init_mesh()
    s.init3d(prims)
    return s


def test_tma_wait_timeout_is_reported(monkeypatch):
    p = cases.tgv_params(32, scheme=SCHEME_OMP6, character=1, dt=0.002)  # FP64, periodic: TMA sweeps
    prims = cases.tgv_prims(p)
    ref = _solver(p, prims)
    ref.step(2)
    f_ref, pr_ref = ref.download_state()
    ref.close()

    s = _solver(p, prims)
    monkeypatch.setenv("OCFD_TEST_STALL_TMA", "1")
    with pytest.raises(OcfdError) as err:
        s.step(1)
    assert err.value.code == OCFD_E_TIMEOUT
    monkeypatch.delenv("OCFD_TEST_STALL_TMA")
    s.init3d(prims)
    s.step(2)
    f, pr = s.download_state()
    s.close()
    np.testing.assert_array_equal(f, f_ref)
    for a, b in zip(pr, pr_ref):
        np.testing.assert_array_equal(a, b)
