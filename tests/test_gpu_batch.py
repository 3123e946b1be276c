"""Batched ensemble (GPU, through the C ABI): ragged periodic instances with
different Re, Ma and dt advanced by one persistent launch per RK stage (the
flux-vector WENO7 and characteristic OMP6 forms) or one launch per kernel and
RK stage give the same bits as each instance stepped alone, for both tile
variants, with members used on their own between batch steps, with the
negative-temperature repair inside the persistent launch, and on the
concurrent fallback path for configurations the batched launch does not
cover."""
import numpy as np
import pytest

from ocfd_b200 import cases
from ocfd_b200.params import SCHEME_HYBRID, SCHEME_OMP6, SCHEME_WENO7, SPLIT_LLF
from ocfd_b200.solver import Batch, Solver
from ocfd_testlib import curvilinear_case

pytestmark = pytest.mark.gpu

SHAPES = [(24, 20, 16), (32, 32, 32), (16, 40, 24), (48, 16, 20)]


def _params(shape, q, scheme, character, mixed, split=1):
    nx, ny, nz = shape
    p = cases.tgv_params(nx, ny=ny, nz=nz, scheme=scheme, character=character, split=split,
                         ma=0.1 + 0.1 * q, re=400.0 + 700.0 * q, dt=0.004 - 0.0005 * q)
    if scheme == SCHEME_HYBRID:
        p.hybrid_para[0] = 2 if q % 2 else 1
        p.hybrid_para[1] = 0.004
        p.hybrid_para[2] = 0.01
        p.ud7l_diss = 0.0
    p.precision = 1 if mixed else 0
    return p


def _make(p):
    s = Solver(p)
    s.init_mesh()
    s.init3d(cases.tgv_prims(s.p))
    return s


def _alone(ps, steps):
    out = []
    for p in ps:
        s = _make(p)
        s.step(steps)
        out.append(s.download_state())
        s.close()
    return out


def _same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    for x, y in zip(a[1], b[1]):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("scheme,character,mixed,split", [
    (SCHEME_WENO7, 0, False, 1),
    (SCHEME_OMP6, 1, False, 1),
    (SCHEME_OMP6, 1, True, 1),
    (SCHEME_HYBRID, 0, True, SPLIT_LLF),
], ids=["weno7-fp64", "omp6char-fp64", "omp6char-mixed", "hybrid-llf-mixed"])
def test_batch_equals_alone(scheme, character, mixed, split):
    ps = [_params(sh, q, scheme, character, mixed, split) for q, sh in enumerate(SHAPES)]
    ref = _alone(ps, 5)
    members = [_make(p) for p in ps]
    b = Batch(members)
    b.step(5)
    fused, variants = b.info()
    assert fused
    if scheme == SCHEME_HYBRID:
        assert b.mode() == 1
    else:
        # five steps: the launch mode was chosen by timing two steps in each
        assert b.mode() in (1, 2)
        t = b.mode_times()
        assert t is not None and min(t) > 0
        assert b.mode() == (2 if t[1] < t[0] else 1)
    for s, r in zip(members, ref):
        _same(s.download_state(), r)
        assert s.time()[0] == 5
    b.close()
    for s in members:
        s.close()


@pytest.mark.parametrize("variants", [(0, 0, 0), (1, 1, 1), (1, 0, 1)])
def test_batch_tile_variants_agree(variants):
    ps = [_params(sh, q, SCHEME_WENO7, 1, False) for q, sh in enumerate(SHAPES[:3])]
    ref = _alone(ps, 3)
    members = [_make(p) for p in ps]
    b = Batch(members)
    b.set_tiles(variants)
    b.step(3)
    assert b.info() == (True, list(variants))
    for s, r in zip(members, ref):
        _same(s.download_state(), r)
    b.close()
    for s in members:
        s.close()


def test_batch_with_members_stepped_alone_between():
    ps = [_params(sh, q, SCHEME_OMP6, 1, False) for q, sh in enumerate(SHAPES[:3])]
    ref = _alone(ps, 6)
    members = [_make(p) for p in ps]
    b = Batch(members)
    b.step(2)
    members[1].step(1)  # member 1 now one step ahead: the batch rebuilds its tables
    e = members[0].show_flow_msg()
    assert np.isfinite(e).all()
    b.step(3)
    members[0].step(1)
    members[2].step(1)
    # member 1 has taken 2 + 1 + 3 = 6 steps, members 0 and 2 have 2 + 3 + 1 = 6
    for s, r in zip(members, ref):
        assert s.time()[0] == 6
        _same(s.download_state(), r)
    b.close()
    for s in members:
        s.close()


def test_batch_fallback_for_walls():
    p1, X, prims = curvilinear_case(n=(24, 20, 8))
    p2 = _params((24, 20, 16), 0, SCHEME_WENO7, 1, False)
    a = Solver(p1)
    a.init_mesh(*X)
    a.init3d(prims)
    a.step(4)
    ref1 = a.download_state()
    a.close()
    ref2 = _alone([p2], 4)[0]
    s1 = Solver(p1)
    s1.init_mesh(*X)
    s1.init3d(prims)
    s2 = _make(p2)
    b = Batch([s1, s2])
    b.step(4)
    assert b.info()[0] is False
    _same(s1.download_state(), ref1)
    _same(s2.download_state(), ref2)
    b.close()
    s1.close()
    s2.close()


def _ragged_weno7_mixed(count):
    sizes = [16, 24, 32, 40, 48]
    return [_params((sizes[q % 5], sizes[(q + 2) % 5], sizes[(q + 4) % 5]), q % 4, SCHEME_WENO7, 0, True)
            for q in range(count)]


def test_persistent_stage_many_members():
    """Twelve ragged members in the served configuration (flux-vector WENO7,
    mixed precision): the persistent launch per stage, the launch per kernel and
    each member alone give the same bits."""
    ps = _ragged_weno7_mixed(12)
    ref = _alone(ps, 4)
    for persistent in (True, False):
        members = [_make(p) for p in ps]
        b = Batch(members)
        b.set_persistent(persistent)
        assert b.mode() == (2 if persistent else 1)
        b.step(4)
        for s, r in zip(members, ref):
            _same(s.download_state(), r)
        b.close()
        for s in members:
            s.close()


def _planted(p):
    """A member whose state has negative internal energy at two points: every
    stage finds T <= 0 there and repairs it (handle_NegativeT)."""
    s = _make(p)
    f = s.download_f()
    for (k, j, i) in [(3, 4, 5), (7, 2, 9)]:
        f[4, k, j, i] = 0.3 * (f[1, k, j, i] ** 2 + f[2, k, j, i] ** 2 + f[3, k, j, i] ** 2) / f[0, k, j, i]
    s.upload_state(f=f)
    s.comput_duvwT()
    return s


@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "mixed"])
def test_persistent_stage_negative_temperature_repair(mixed):
    ps = [_params(sh, q, SCHEME_OMP6, 1, mixed) for q, sh in enumerate(SHAPES[:3])]
    ref = []
    for q, p in enumerate(ps):
        s = _planted(p) if q == 1 else _make(p)
        s.step(2)
        ref.append(s.download_state())
        if q == 1:
            assert s.comput_duvwT() > 0  # the planted points stay negative: the stages repaired them
        s.close()
    members = [_planted(p) if q == 1 else _make(p) for q, p in enumerate(ps)]
    b = Batch(members)
    b.set_persistent(True)
    assert b.mode() == 2
    b.step(2)
    for s, r in zip(members, ref):
        _same(s.download_state(), r)
    b.close()
    for s in members:
        s.close()


def test_persistent_stage_wait_timeout_is_reported(monkeypatch):
    """The dependency waits of the persistent launch are bounded: with a work
    list whose phase-A counts cannot be reached (a test switch read when the
    tables are built), the kernel gives up after about a second, finishes, and
    the step reports OCFD_E_TIMEOUT; the batch then continues with one launch
    per kernel, with no error left behind (restarted from the initial field,
    the members give the same bits as alone)."""
    from ocfd_b200._lib import OCFD_E_TIMEOUT, OcfdError

    ps = _ragged_weno7_mixed(2)
    members = [_make(p) for p in ps]
    b = Batch(members)
    b.set_persistent(True)
    monkeypatch.setenv("OCFD_TEST_STALL_BATCH_WAIT", "1")
    with pytest.raises(OcfdError) as err:
        b.step(1)
    assert err.value.code == OCFD_E_TIMEOUT
    monkeypatch.delenv("OCFD_TEST_STALL_BATCH_WAIT")
    assert b.mode() == 1
    # the timed-out step left invalid states: start again from the initial field
    ref = _alone(ps, 2)
    for s in members:
        s.init3d(cases.tgv_prims(s.p))
    b.step(2)
    for s, r in zip(members, ref):
        _same(s.download_state(), r)
    b.close()
    for s in members:
        s.close()
