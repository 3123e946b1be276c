"""Serving loop (GPU): requests of mixed sizes arriving over time are admitted
into free slots while others run, advanced together by the batched launches
(the larger ones on their own step graphs at the same time), and each result
equals the same request solved alone (bit for bit: the stated tolerance is
zero)."""
import numpy as np
import pytest

from ocfd_b200 import serving
from ocfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _alone(req, mixed):
    p, xyz, prims = serving.request_setup(req, mixed)
    s = serving._start(p, xyz, prims, 0)
    s.step(req.steps)
    out = s.download_state(), s.show_flow_msg().tolist()
    s.close()
    return out


@pytest.mark.parametrize("solo_min", [96, 48], ids=["all-batched", "48-on-own-graphs"])
def test_each_result_is_the_same_alone_and_in_the_mix(solo_min):
    reqs = serving.make_stream(7, rate=40.0, seed=7, sizes=(32, 48), steps=(12, 40))
    srv = serving.Server(mixed=True, max_slots=4, round_steps=5, keep=[r.rid for r in reqs], solo_min=solo_min)
    out = srv.run(reqs, realtime=True)
    assert len(out["results"]) == len(reqs)
    assert out["rounds"] > 1
    if solo_min > 48:
        assert out["batched_rounds"] == out["rounds"]
    assert out["max_active"] > 1
    assert out["p99_s"] >= out["p50_s"] > 0.0
    for r in reqs:
        res = out["results"][r.rid]
        (f_a, prims_a), e_a = _alone(r, True)
        f_m, prims_m = res.state
        np.testing.assert_array_equal(f_m, f_a)
        for x, y in zip(prims_m, prims_a):
            np.testing.assert_array_equal(x, y)
        assert res.E0 == e_a


def test_admission_respects_the_memory_budget():
    from ocfd_b200.solver import footprint, set_parameters

    reqs = serving.make_stream(5, rate=0.0, seed=3, sizes=(48,), steps=(10, 10))
    p, _, _ = serving.request_setup(reqs[0], True)
    one = footprint(set_parameters(p))
    srv = serving.Server(mixed=True, hbm_budget=int(2.5 * one), max_slots=8, round_steps=10)
    out = srv.run(reqs, realtime=False)
    assert out["max_active"] == 2
    assert len(out["results"]) == 5
