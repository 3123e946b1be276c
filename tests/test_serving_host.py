"""Serving loop bookkeeping on the CPU (no GPU): the instances and the batch
are stand-ins that count the steps they are given, so the test checks the
loop itself -- every request receives exactly its step count, no instance is
stepped after it finished or before it was admitted, instances of at least
solo_min^3 points never enter a batch while smaller ones do, the round in
flight is retired only after the next one was enqueued, admission respects the
memory budget and the slot count, and every request gets a result."""
import numpy as np
import pytest

from ocfd_b200 import serving

EVENTS = []


class FakeSolver:
    def __init__(self, p):
        self.n = p.nx
        self.done = 0
        self.closed = False

    def step(self, k, sync=True):
        assert not self.closed
        self.done += k
        EVENTS.append(("step", id(self), k))

    def sync(self):
        EVENTS.append(("retire", id(self)))

    def show_flow_msg(self):
        return np.array([float(self.done), 0.0, 0.0])

    def download_state(self):
        return None

    def close(self):
        assert not self.closed
        self.closed = True


class FakeBatch:
    def __init__(self, members):
        self.members = list(members)
        self.closed = False
        EVENTS.append(("batch", tuple(m.n for m in self.members)))

    def set_tiles(self, variants):
        pass

    def set_persistent(self, on):
        EVENTS.append(("persistent", on))

    def step(self, k, sync=True):
        assert not self.closed
        for m in self.members:
            m.step(k, sync)

    def info(self):
        return True, [0, 0, 0]

    def mode(self):
        return 1

    def mode_times(self):
        return (1.0, 2.0)

    def close(self):
        self.closed = True


@pytest.fixture
def fake_backend(monkeypatch):
    EVENTS.clear()
    monkeypatch.setattr(serving, "_start", lambda p, xyz, prims, device: FakeSolver(p))
    monkeypatch.setattr(serving, "Batch", FakeBatch)
    return EVENTS


@pytest.mark.parametrize("solo_min", [24, 1000])
def test_serving_loop_bookkeeping(fake_backend, solo_min):
    reqs = serving.make_stream(14, rate=0.0, seed=11, sizes=(8, 16, 24, 32), steps=(3, 40))
    srv = serving.Server(mixed=True, hbm_budget=1 << 40, max_slots=5, round_steps=7, solo_min=solo_min,
                         max_points=10 ** 9)
    out = srv.run(reqs, realtime=False)
    res = out["results"]
    assert sorted(res) == [r.rid for r in reqs]
    for r in reqs:
        assert res[r.rid].E0[0] == r.steps  # exactly its own step count
        assert res[r.rid].finished >= res[r.rid].admitted
    assert 1 < out["max_active"] <= 5
    batches = [e[1] for e in EVENTS if e[0] == "batch"]
    assert batches, "the small instances share batched launches"
    for sizes in batches:
        assert all(n < solo_min for n in sizes)
    # a finished instance is retired (its result read) after the next round was enqueued
    kinds = [e[0] for e in EVENTS]
    first_retire = kinds.index("retire")
    assert "step" in kinds[:first_retire]


def test_serving_admission_budget(fake_backend):
    from ocfd_b200.solver import footprint, set_parameters

    reqs = serving.make_stream(6, rate=0.0, seed=3, sizes=(16,), steps=(10, 10))
    p, _, _ = serving.request_setup(reqs[0], True)
    one = footprint(set_parameters(p))
    srv = serving.Server(mixed=True, hbm_budget=int(2.5 * one), max_slots=8, round_steps=10)
    out = srv.run(reqs, realtime=False)
    assert out["max_active"] == 2
    assert len(out["results"]) == 6


@pytest.mark.parametrize("mode,expect", [("per_kernel", False), ("persistent", True)])
def test_serving_forced_launch_mode(fake_backend, mode, expect):
    reqs = serving.make_stream(6, rate=0.0, seed=5, sizes=(8, 16), steps=(5, 12))
    srv = serving.Server(mixed=True, hbm_budget=1 << 40, max_slots=4, round_steps=4, solo_min=1000,
                         launch_mode=mode)
    out = srv.run(reqs, realtime=False)
    assert len(out["results"]) == 6
    calls = [e[1] for e in EVENTS if e[0] == "persistent"]
    assert calls and all(c is expect for c in calls)
    with pytest.raises(ValueError):
        serving.Server(mixed=True, hbm_budget=1 << 40, launch_mode="fastest")
