"""
Failure paths on a B200, none of which faults, traps or hangs the GPU.

* A bounded wait that runs out: qpd_probe_wait_timeout makes a kernel wait on a barrier that no copy
  ever completes, with a limit of a thousand polls; the device status word records the timeout, the
  host reads it as QPD_ERR_CUDA (the reference aborts through MPI_Abort instead,
  src/heffte/util.hpp:12-16), and the same context then computes the next volume normally.
* NaN inputs: the reference floors |S Amp|^2 with numpy.maximum, which propagates NaN
  (src/python/diffraction.py:111), and a NaN in one scattering cell reaches every voxel through the
  FFT; the CUDA path returns the same all-NaN volume in every precision and schedule.
"""

import numpy as np
import pytest

from conftest import fp32_errors

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_the_context_recovers(gpu):
    from qpop_diffraction_b200 import Plan, crystal_from, workloads, _native
    case = workloads.config2(shape=(32, 24, 104), hkl=(1, 0, 3))
    p = case.params
    with Plan(case.shape, (p.dx, p.dy, p.dz), p.nPhase, p.nStruc, precision="fp32") as plan:
        plan.set_crystal(crystal_from(p, case.atoms))
        before = plan.run_host(case.oPhase, case.oStruc, case.u, case.region)
        plan.probe_wait_timeout(1000)
        with pytest.raises(_native.QpdError) as err:
            plan.device_status()
        assert err.value.code == _native.QPD_ERR_CUDA
        assert "gave up waiting" in str(err.value)
        plan.device_status()  # the word was cleared by the read
        after = plan.run_host(case.oPhase, case.oStruc, case.u, case.region)
    np.testing.assert_array_equal(after, before)


def test_probe_rejects_bad_poll_counts(gpu):
    from qpop_diffraction_b200 import Plan, _native
    with Plan((8, 8, 8), (0.4, 0.4, 0.4), 1) as plan:
        for polls in (0, -5, (1 << 24) + 1):
            with pytest.raises(ValueError):
                plan.probe_wait_timeout(polls)
        assert plan.lib.qpd_probe_wait_timeout(None, 10) == _native.QPD_ERR_ARG


@pytest.mark.parametrize("precision,schedule", [("fp32", "fused"), ("fp64", "fused"), ("fp32", "plain"),
                                                ("fp64", "plain")])
def test_nan_input_propagates_like_the_reference(gpu, precision, schedule):
    from oracle import diffraction_oracle as oracle
    from qpop_diffraction_b200 import diffraction, workloads
    case = workloads.random_case((12, 10, 16), seed=21, nPhase=1, weights="onehot")
    n = case.params.n
    cell = int(np.flatnonzero(case.region > 0)[5])  # a cell that scatters
    for arr, comp in ((case.oStruc, 1), (case.u, 2)):
        bad = arr.copy()
        bad[comp * n + cell] = np.nan
        args = list(case.args())
        args[3 if arr is case.oStruc else 4] = bad
        ref = oracle.diffraction(*args)[0]
        assert np.isnan(ref).all()
        got = diffraction(*args, precision=precision, schedule=schedule)[0]
        assert np.isnan(got).all()
    # and the clean volume right after is unaffected
    ref = oracle.diffraction(*case.args())[0]
    got = diffraction(*case.args(), precision=precision, schedule=schedule)[0]
    dmax, rel = fp32_errors(got, ref)
    assert dmax <= 1e-5 and rel <= 1e-3
