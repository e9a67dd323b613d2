"""
The float64 direct-sum voxel check (tests/direct_dft.py) against the oracle's FFT restatement of the
reference's diffraction() (oracle/diffraction_oracle.py), on CPU tensors.  The direct sum is the
independent check of the 4000 x 4000 x 68 volume in test_gpu_parity.py, where the oracle cannot run.
"""

import numpy as np
import pytest

from direct_dft import crystal_constants, direct_intensity, fft_index_to_shifted, shifted_to_fft_index
from oracle import diffraction_oracle as oracle


def oracle_from_packed(torch, shape, spacing, consts, inputs, nPhase):
    G, qC, V, R, fAtom, su = consts
    n = int(np.prod(shape))
    ph = inputs["phase"].numpy().astype(np.int64)
    w = np.stack([(ph == p).astype(np.float64) for p in range(nPhase)])
    P = inputs["P"].double().numpy().reshape(3, n)
    U = inputs["U"].double().numpy().reshape(3, n)
    return oracle.intensity(shape, spacing, G, qC, V, R, fAtom, su, w, P, U)


@pytest.mark.parametrize("kind,nPhase", [("twin", 1), ("vortex", 2)])
def test_direct_sum_equals_the_oracle_at_every_voxel(kind, nPhase):
    import torch
    from qpop_diffraction_b200 import workloads
    shape = (12, 10, 8)
    params, inputs = workloads.gpu_snapshot(kind, shape, seed=4, device="cpu", n_phase=nPhase, n_domains=5)
    atoms = workloads.config3_crystal(3, (1, 1, 3)) if nPhase == 1 else workloads.config2_crystal(2, (1, 0, 3))
    spacing = (params.dx, params.dy, params.dz)
    consts = crystal_constants(params, atoms)
    ref = oracle_from_packed(torch, shape, spacing, consts, inputs, nPhase)      # fftshifted
    idx = np.stack(np.meshgrid(*[np.arange(s) for s in shape], indexing="ij"), axis=-1).reshape(-1, 3)
    got = direct_intensity(torch, shape, spacing, *consts, inputs["P"], inputs["U"], inputs["phase"], None, idx,
                           slab=5)
    pos = [fft_index_to_shifted(s) for s in shape]
    want = ref[pos[0][idx[:, 0]], pos[1][idx[:, 1]], pos[2][idx[:, 2]]]
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * want.max())


def test_shift_maps_are_inverse():
    for N in (7, 8, 68, 4000):
        a, b = fft_index_to_shifted(N), shifted_to_fft_index(N)
        assert np.array_equal(b[a], np.arange(N)) and np.array_equal(a[b], np.arange(N))
        x = np.arange(N) * 3.0
        assert np.array_equal(np.fft.fftshift(x)[a], x)
