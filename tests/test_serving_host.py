"""
The serving loop's host logic on the CPU: admission by HBM footprint, continuous dispatch (a
request of a free shape overtakes one whose shape is busy), cancellation of queued and in-flight
requests, the per-shape slot cap, release of idle slots and the engine's tiles-per-CTA setting.
The GPU slot (a planned context, its stream and graphs) is replaced by a stand-in whose "volume"
completes a fixed time after launch; the GPU tests run the same engine on a B200.
"""

import time
import types

import numpy as np
import pytest

from qpop_diffraction_b200 import serving

SMALL, LARGE = (16, 16, 8), (64, 64, 32)
DURATION = {SMALL: 0.005, LARGE: 0.06}  # seconds a stand-in volume takes


class StandInEvent:
    def __init__(self):
        self.t_done = None

    def query(self):
        return self.t_done is not None and time.perf_counter() >= self.t_done


class StandInSlot:
    """A slot without a GPU: same constructor and fields as serving.Slot, volumes that take DURATION."""

    made = []

    def __init__(self, shape, spacing, nPhase, device, crystal_of, priority=0, cta_tiles=0):
        self.shape = tuple(shape)
        self.priority, self.cta_tiles = priority, cta_tiles
        self.request = None
        self.footprint = serving.Engine._footprint_estimate(types.SimpleNamespace(shape=self.shape))
        self.event = StandInEvent()
        self.launched = []
        self.closed = False
        StandInSlot.made.append(self)

    def launch(self, snap, hkl):
        self.launched.append((snap.id, tuple(hkl)))
        self.event.t_done = time.perf_counter() + DURATION[self.shape]

    def close(self):
        self.closed = True


@pytest.fixture
def engine_parts(monkeypatch):
    monkeypatch.setattr(serving, "Slot", StandInSlot)
    StandInSlot.made = []
    store = serving.SnapshotStore()
    params = types.SimpleNamespace(dx=0.39, dy=0.39, dz=0.4, nPhase=1)
    store.add(serving.Snapshot(0, "vortex", SMALL, params, {}))
    store.add(serving.Snapshot(1, "twin", LARGE, params, {}))
    return store


def footprint(shape):
    return serving.Engine._footprint_estimate(types.SimpleNamespace(shape=shape))


def test_admission_never_exceeds_the_budget(engine_parts):
    store = engine_parts
    budget = 2 * footprint(LARGE) + footprint(LARGE) // 2   # room for two large slots, not three
    eng = serving.Engine(store, budget, crystal_of=lambda p, h: None)
    reqs = [serving.Request(i, 1, (0, 0, 2), 0.0) for i in range(5)]
    done = eng.run(reqs)
    assert sorted(r.id for r in done) == list(range(5))
    assert eng.peak_slots == 2 and eng.used <= budget
    # five volumes through two slots: the last ones waited for a slot to free up
    assert max(r.start for r in done) >= DURATION[LARGE] * 0.9


def test_a_free_shape_overtakes_a_busy_one(engine_parts):
    store = engine_parts
    eng = serving.Engine(store, 1 << 40, crystal_of=lambda p, h: None, max_slots=1)
    reqs = [serving.Request(0, 1, (0, 0, 2), 0.0), serving.Request(1, 1, (1, 0, 3), 0.0),
            serving.Request(2, 0, (0, 0, 2), 0.0)]
    done = {r.id: r for r in eng.run(reqs)}
    # the second large request waits for the only large slot; the small one behind it starts at once
    assert done[2].start < done[0].done <= done[1].start
    assert len(eng.slots[LARGE]) == 1 and len(eng.slots[SMALL]) == 1


def test_cancel_a_queued_and_an_in_flight_request(engine_parts):
    store = engine_parts
    eng = serving.Engine(store, 1 << 40, crystal_of=lambda p, h: None, max_slots=1)
    reqs = [serving.Request(i, 1, (0, 0, 2), 0.0) for i in range(3)]
    done = eng.run(reqs, cancel=[(0.01, 0), (0.01, 2)])
    by = {r.id: r for r in done}
    assert by[0].cancelled and by[0].start is not None   # was on the device: runs to its end, result dropped
    assert by[2].cancelled and by[2].start is None       # still queued: never dispatched
    assert not by[1].cancelled and by[1].done is not None
    assert [r.id for r in done if not r.cancelled] == [1]
    assert all(s.request is None for s in eng.slots[LARGE])


def test_release_idle_returns_the_footprint(engine_parts):
    store = engine_parts
    eng = serving.Engine(store, 1 << 40, crystal_of=lambda p, h: None)
    eng.reserve(1, 2)
    eng.reserve(0, 1)
    assert eng.used == 2 * footprint(LARGE) + footprint(SMALL)
    assert eng.release_idle() == 0
    assert all(s.closed for s in StandInSlot.made)


def test_tiles_per_cta_setting(engine_parts):
    store = engine_parts
    assert serving.Engine(store, 1 << 30, priorities=True).cta_tiles == 4
    assert serving.Engine(store, 1 << 30).cta_tiles == 0
    eng = serving.Engine(store, 1 << 40, crystal_of=lambda p, h: None, cta_tiles=7)
    eng.reserve(0, 1)
    assert [s.cta_tiles for s in StandInSlot.made] == [7]


def test_latency_stats_leave_out_cancelled_requests():
    reqs = [serving.Request(i, 0, (0, 0, 2), arrival=0.001 * i) for i in range(10)]
    for i, r in enumerate(reqs):
        r.start, r.done = r.arrival, r.arrival + 0.002 * (i + 1)
    reqs[9].cancelled = True
    st = serving.latency_stats(reqs)
    lat = np.array([0.002 * (i + 1) for i in range(9)])
    assert st["p50_ms"] == pytest.approx(np.percentile(lat, 50) * 1e3)
    assert st["p99_ms"] == pytest.approx(np.percentile(lat, 99) * 1e3)
