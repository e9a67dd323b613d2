"""
The serving loop on a B200: every result is the same whether its request runs alone or among
others in flight, admission never exceeds the HBM budget, and served volumes meet the float32
contract against the oracle.
"""

import numpy as np
import pytest

from conftest import fp32_errors

pytestmark = pytest.mark.gpu

SHAPES = [(64, 64, 32), (32, 64, 68), (48, 32, 104)]
HKLS = [(0, 0, 2), (1, 0, 3), (1, 1, 3), (2, 0, 0)]


def make_store(torch, n_per_shape=2):
    from qpop_diffraction_b200 import workloads
    from qpop_diffraction_b200.serving import Snapshot, SnapshotStore
    store = SnapshotStore()
    i = 0
    for shape in SHAPES:
        for k in range(n_per_shape):
            kind = workloads.TEXTURES[i % 3]
            params, inputs = workloads.gpu_snapshot(kind, shape, seed=100 + i, device="cuda")
            store.add(Snapshot(i, kind, shape, params, inputs))
            i += 1
    return store


def oracle_inputs(snap):
    """Float64 reference-layout arrays holding the snapshot's packed values."""
    P = snap.inputs["P"].double().cpu().numpy()
    U = snap.inputs["U"].double().cpu().numpy()
    ph = snap.inputs["phase"].cpu().numpy().astype(np.int64)
    oPhase = np.stack([(ph == p).astype(np.float64) for p in range(2)]).ravel()
    return oPhase, P, U, np.ones(ph.size)


def test_same_result_alone_and_in_the_mix(gpu):
    torch = gpu
    from qpop_diffraction_b200.serving import Engine, poisson_requests
    store = make_store(torch)
    reqs = poisson_requests(24, 0, list(range(len(store))), HKLS, seed=7)
    alone, mixed = {}, {}
    eng = Engine(store, hbm_budget_bytes=4 << 30)
    try:
        for r in reqs:   # one at a time
            eng.run([type(r)(r.id, r.snapshot, r.hkl, 0.0)], result_of=lambda q, t: alone.__setitem__(q.id, t.cpu().numpy()))
        eng.run(reqs, result_of=lambda q, t: mixed.__setitem__(q.id, t.cpu().numpy()))
        assert eng.peak_slots > len(SHAPES)   # the mix really ran several volumes at once
    finally:
        eng.close()
    assert sorted(alone) == sorted(mixed) == [r.id for r in reqs]
    for r in reqs:
        np.testing.assert_array_equal(mixed[r.id], alone[r.id])


def test_admission_by_footprint(gpu):
    torch = gpu
    from qpop_diffraction_b200.serving import Engine, Request, Snapshot, SnapshotStore
    from qpop_diffraction_b200 import workloads
    store = SnapshotStore()
    params, inputs = workloads.gpu_snapshot("vortex", (64, 64, 104), 5, device="cuda")
    store.add(Snapshot(0, "vortex", (64, 64, 104), params, inputs))
    one_slot = Engine._footprint_estimate(store[0]) + (1 << 20)
    eng = Engine(store, hbm_budget_bytes=one_slot)
    try:
        done = eng.run([Request(i, 0, (0, 0, 2), 0.0) for i in range(5)])
        assert len(done) == 5 and eng.peak_slots == 1 and eng.used <= one_slot
    finally:
        eng.close()
    eng = Engine(store, hbm_budget_bytes=1024)   # nothing fits: requests wait, no slot is created
    assert eng.dispatch(Request(0, 0, (0, 0, 2), 0.0), 0.0) is False and eng.peak_slots == 0


def test_served_volume_meets_the_contract(gpu):
    torch = gpu
    from oracle import diffraction_oracle as oracle
    from qpop_diffraction_b200 import workloads
    from qpop_diffraction_b200.serving import Engine, Request
    store = make_store(torch, n_per_shape=1)
    out = {}
    eng = Engine(store, hbm_budget_bytes=4 << 30)
    try:
        eng.run([Request(i, i, HKLS[i % 4], 0.0) for i in range(len(store))],
                result_of=lambda q, t: out.__setitem__(q.id, t.cpu().numpy()))
    finally:
        eng.close()
    for i in range(len(store)):
        snap = store[i]
        oPhase, P, U, region = oracle_inputs(snap)
        ref = oracle.diffraction(snap.params, workloads.serving_crystal(HKLS[i % 4]), oPhase, P, U, region)[0]
        dmax, rel = fp32_errors(out[i], ref)
        assert dmax <= 1e-5 and rel <= 1e-3, (snap.shape, dmax, rel)


def test_cancel_queued_and_in_flight_requests(gpu):
    """A queued request cancelled never runs; one cancelled on the device finishes there with its
    result discarded; the slot serves the next request, which gives the same volume as when run alone;
    releasing idle slots returns their footprint to the budget."""
    torch = gpu
    from qpop_diffraction_b200.serving import Engine, Request
    store = make_store(torch, n_per_shape=1)
    shape_snap = 2  # (48, 32, 104)
    eng = Engine(store, hbm_budget_bytes=4 << 30)
    try:
        assert eng.reserve(shape_snap, 1) == 1
        budget_used = eng.budget = eng.used  # no room for a second slot: the shape has exactly one
        alone = {}
        eng.run([Request(9, shape_snap, (1, 0, 3), 0.0)], result_of=lambda q, t: alone.__setitem__(q.id, t.cpu().numpy()))
        assert len(eng.slots[store[shape_snap].shape]) == 1
        reqs = [Request(0, shape_snap, (0, 0, 2), 0.0), Request(1, shape_snap, (2, 0, 0), 0.0),
                Request(2, shape_snap, (1, 0, 3), 0.0)]
        got = {}
        out = eng.run(reqs, result_of=lambda q, t: got.__setitem__(q.id, t.cpu().numpy()),
                      cancel=[(0.0, 1), (0.0, 0)])
        by = {r.id: r for r in out}
        assert sorted(by) == [0, 1, 2]
        assert by[1].cancelled and by[1].start is None and by[1].done is None       # dropped from the queue
        assert by[0].cancelled and by[0].start is not None and by[0].done is not None  # finished, discarded
        assert not by[2].cancelled and by[2].done is not None
        assert sorted(got) == [2]
        np.testing.assert_array_equal(got[2], alone[9])
        assert not eng.busy() and eng.used == budget_used
        assert eng.release_idle() == 0
    finally:
        eng.close()


@pytest.mark.parametrize("shape", [(128, 128, 68), (96, 96, 104), (64, 64, 128)])
def test_cta_tiles_do_not_change_results(gpu, shape):
    """The serving loop caps the tiles per CTA of the persistent z stages (Plan.set_cta_tiles) so that
    CTAs retire while a large volume runs; the volume's bits do not depend on the cap.  These grids
    have more z-stage tiles than one wave of CTAs holds, so the caps really change the grid."""
    torch = gpu
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    params, inputs = workloads.gpu_snapshot(workloads.TEXTURES[0], shape, seed=11, device="cuda")
    crystal = crystal_from(params, workloads.serving_crystal((1, 0, 3)))
    outs = []
    for k in (0, 1, 3):
        with Plan(shape, (params.dx, params.dy, params.dz), params.nPhase, 3, precision="fp32") as plan:
            plan.set_crystal(crystal)
            plan.set_cta_tiles(k)
            out = torch.empty(shape, dtype=torch.float64, device="cuda")
            plan.run_device(inputs, out)
            torch.cuda.synchronize()
            plan.device_status()
            outs.append(out)
    for o in outs[1:]:
        assert torch.equal(o, outs[0])
