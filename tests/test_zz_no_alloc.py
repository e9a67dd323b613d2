"""
The allocation-free entry point qpd_run_device_noalloc, called through the C ABI.

Callers that cannot let a library allocate GPU memory (a stream under graph capture, a framework
allocator that owns the device, a real-time loop with everything reserved up front) use this
variant; it must give the same volume as the allocating qpd_run_device on the same packed inputs,
call after call, since every call reuses one library-wide scratch array.  The file sorts last so
that a run stopping at the first failure has run every other test first.
"""

import numpy as np
import pytest

from conftest import fp32_errors

pytestmark = pytest.mark.gpu


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
        packed = plan.pack(*(torch.from_numpy(a).to(dev) for a in (case.oPhase, case.oStruc, case.u, case.region)))
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
