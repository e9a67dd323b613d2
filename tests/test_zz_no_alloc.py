"""
The allocation-free entry point qpd_run_device_noalloc, called through the C ABI.

Callers that cannot let a library allocate GPU memory (a framework allocator that owns the
device, a real-time loop with everything reserved up front) use this variant; it must give the
same volume as the allocating qpd_run_device on the same packed inputs, call after call, since
every call reuses one library-wide scratch array.  The file sorts last so that a run stopping at
the first failure has run every other test first.
"""

import numpy as np
import pytest

from conftest import fp32_errors

pytestmark = pytest.mark.gpu


def _several_groups_case(n_rx, seed=11, shape=(12, 10, 16)):
    """A random one-phase case whose atoms sit at n_rx distinct R_x (and a few R_y per R_x)."""
    from qpop_diffraction_b200 import workloads

    case = workloads.random_case(shape, seed, nAtom=n_rx + 2)
    xs = (np.arange(n_rx) + 0.5) / (n_rx + 1)
    xAtom = np.array([[xs[i % n_rx], 0.25 * (i // n_rx) + 0.1 * (i % 2), 0.1 * i] for i in range(n_rx + 2)],
                     dtype=np.float64)
    case.atoms.xAtom = xAtom
    return case


def _packed(torch, plan, case):
    dev = torch.device("cuda", 0)
    return plan.pack(*(torch.from_numpy(a).to(dev) for a in (case.oPhase, case.oStruc, case.u, case.region)))


def test_noalloc_matches_allocating_entry_point_twice(gpu):
    torch = gpu
    from oracle import diffraction_oracle as oracle
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    from qpop_diffraction_b200.noalloc import run_device_noalloc

    case = workloads.config2(shape=(32, 24, 104), hkl=(1, 0, 3))
    p = case.params
    spacing = (p.dx, p.dy, p.dz)
    crystal = crystal_from(p, case.atoms)
    dev = torch.device("cuda", 0)
    with Plan(case.shape, spacing, p.nPhase, p.nStruc, precision="fp32") as plan:
        plan.set_crystal(crystal)
        packed = _packed(torch, plan, case)
        assert packed["wdense"] is None
        ref = plan.run_device(packed).cpu().numpy()
    oracle_I = oracle.diffraction(*case.args())[0]
    for _ in range(2):
        out = torch.full(case.shape, -1.0, dtype=torch.float64, device=dev)
        run_device_noalloc(case.shape, spacing, crystal, packed, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        for want in (ref, oracle_I):
            dmax, rel = fp32_errors(got, want)
            assert dmax <= 1e-5 and rel <= 1e-3, (dmax, rel)


def test_noalloc_several_atom_groups_on_a_side_stream(gpu):
    """Six distinct R_x with several R_y each, enqueued on a non-default stream, twice in a row."""
    torch = gpu
    from oracle import diffraction_oracle as oracle
    from qpop_diffraction_b200 import Plan, crystal_from
    from qpop_diffraction_b200.noalloc import run_device_noalloc

    case = _several_groups_case(6)
    p = case.params
    spacing = (p.dx, p.dy, p.dz)
    crystal = crystal_from(p, case.atoms)
    assert len(np.unique(crystal.R[:, 0])) == 6
    dev = torch.device("cuda", 0)
    with Plan(case.shape, spacing, p.nPhase, p.nStruc, precision="fp32") as plan:
        plan.set_crystal(crystal)
        packed = _packed(torch, plan, case)
        ref = plan.run_device(packed).cpu().numpy()
    oracle_I = oracle.diffraction(*case.args())[0]
    side = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()
    for _ in range(2):
        with torch.cuda.stream(side):
            out = torch.full(case.shape, -1.0, dtype=torch.float64, device=dev)
            run_device_noalloc(case.shape, spacing, crystal, packed, out, stream=side.cuda_stream)
        side.synchronize()
        got = out.cpu().numpy()
        for want in (ref, oracle_I):
            dmax, rel = fp32_errors(got, want)
            assert dmax <= 1e-5 and rel <= 1e-3, (dmax, rel)


def test_noalloc_refuses_too_many_rx_groups_before_launching(gpu):
    """Fourteen distinct R_x need 28 inputs in the x-pass segment (at most 24): refused, nothing runs."""
    torch = gpu
    from qpop_diffraction_b200 import Plan, crystal_from, _native
    from qpop_diffraction_b200.noalloc import run_device_noalloc

    case = _several_groups_case(14, shape=(8, 8, 16))
    p = case.params
    spacing = (p.dx, p.dy, p.dz)
    crystal = crystal_from(p, case.atoms)
    assert len(np.unique(crystal.R[:, 0])) == 14
    dev = torch.device("cuda", 0)
    with Plan(case.shape, spacing, p.nPhase, p.nStruc, precision="fp32") as plan:
        plan.set_crystal(crystal)
        packed = _packed(torch, plan, case)
    out = torch.full(case.shape, -1.0, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    with pytest.raises(ValueError) as err:
        run_device_noalloc(case.shape, spacing, crystal, packed, out)
    assert err.value.code == _native.QPD_ERR_UNSUPPORTED
    assert "R_x" in str(err.value)
    torch.cuda.synchronize()
    assert bool((out == -1.0).all())


def test_noalloc_refuses_grids_beyond_its_scratch(gpu):
    torch = gpu
    from qpop_diffraction_b200 import crystal_from, workloads, _native
    from qpop_diffraction_b200.noalloc import run_device_noalloc

    shape = (256, 256, 64)  # 96 bytes of fields per cell: 400 MB, far beyond 32 MiB
    params = workloads.make_params(shape, (0.39, 0.39, 0.40), 2)
    crystal = crystal_from(params, workloads.config2_crystal(2, (0, 0, 2)))
    dev = torch.device("cuda", 0)
    tiny = {"P": torch.zeros(3, device=dev), "U": torch.zeros(3, device=dev),
            "phase": torch.zeros(1, dtype=torch.int8, device=dev), "weight": None, "wdense": None}
    out = torch.empty(shape, dtype=torch.float64, device=dev)
    with pytest.raises(MemoryError) as err:
        run_device_noalloc(shape, (params.dx, params.dy, params.dz), crystal, tiny, out)
    assert err.value.code == _native.QPD_ERR_NOMEM
    assert "QPD_NOALLOC_SCRATCH_BYTES" in str(err.value)
