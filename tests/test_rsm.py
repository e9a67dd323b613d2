"""
Reciprocal-space maps (qpop_diffraction_b200.rsm) against the oracle's restatement of the
reference's per-voxel histogram2d binning (oracle/rsm_oracle.py, src/python/rsm.py:69-104).
Sums in a different order: relative tolerance 1e-12 of the map's maximum.
"""

import numpy as np
import pytest

from oracle import rsm_oracle
from qpop_diffraction_b200 import rsm

CASES = [((12, 9, 7), None, "sum"), ((12, 9, 7), None, "mean"), ((12, 9, 7), 5, "sum"), ((12, 9, 7), 4, "mean"),
         ((1, 16, 20), None, "sum"), ((1, 16, 20), None, "mean"), ((6, 1, 5), 3, "mean")]


def volume(shape, seed=0):
    rng = np.random.default_rng(seed)
    I = rng.random(shape) ** 4 + 1e-50
    qC = rng.standard_normal(3)
    axes = [np.fft.fftshift(2 * np.pi * np.fft.fftfreq(n, h)) + c for n, h, c in zip(shape, (0.4, 0.39, 0.41), qC)]
    return I, axes


def assert_maps(got, want):
    assert set(got) == set(want)
    for stem in want:
        for g, w in zip(got[stem][:2], want[stem][:2]):
            assert np.array_equal(g, w), stem
        np.testing.assert_allclose(got[stem][2], want[stem][2], rtol=0, atol=1e-12 * want[stem][2].max())


@pytest.mark.parametrize("shape,bins,aggregation", CASES)
def test_rebinning_of_projections_matches_histogram2d(shape, bins, aggregation):
    I, axes = volume(shape)
    proj = [I.sum(axis=2), I.sum(axis=1), I.sum(axis=0)]
    assert_maps(rsm.maps_from_projections(proj, *axes, bins=bins, aggregation=aggregation),
                rsm_oracle.maps(I, *axes, bins=bins, aggregation=aggregation))


def test_bin_index_follows_numpy_histogram():
    rng = np.random.default_rng(1)
    v = rng.uniform(-1, 1, 500)
    e = np.linspace(-0.8, 0.9, 8)
    v[:3] = e[-1], e[0], e[3]
    idx = rsm.bin_index(v, e)
    counts = np.bincount(idx[idx >= 0], minlength=e.size - 1)
    assert np.array_equal(counts, np.histogram(v, bins=e)[0])


@pytest.mark.gpu
@pytest.mark.parametrize("shape,bins,aggregation", CASES + [((3, 5000, 4), None, "sum"), ((40, 30, 104), 16, "mean")])
def test_gpu_maps_match_the_oracle(gpu, shape, bins, aggregation):
    torch = gpu
    I, axes = volume(shape, seed=2)
    got = rsm.maps(torch.from_numpy(I).cuda(), *axes, bins=bins, aggregation=aggregation)
    assert_maps(got, rsm_oracle.maps(I, *axes, bins=bins, aggregation=aggregation))


@pytest.mark.gpu
def test_gpu_projections(gpu):
    torch = gpu
    I, _ = volume((33, 70, 45), seed=3)
    t = torch.from_numpy(I).cuda()
    xy, xz, yz = rsm.projections(t)
    torch.cuda.synchronize()
    for got, axis in ((xy, 2), (xz, 1), (yz, 0)):
        want = I.sum(axis=axis)
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-13, atol=0)
    again = rsm.projections(t)          # deterministic: no atomics
    assert all(torch.equal(a, b) for a, b in zip((xy, xz, yz), again))
