"""
Pin the oracle (oracle/diffraction_oracle.py) before trusting it as the checker.

1. Against golden fixtures made by running the reference's own diffraction() on the
   same inputs (tests/golden/make_golden.py): bit-exact q axes, intensity to 1e-12.
2. Against the reference test-suite's analytic known answers (tests/analytic.py),
   with the reference's own tolerances.
"""

import numpy as np
import pytest

import analytic
from conftest import golden_names, load_golden
from oracle import diffraction_oracle as oracle


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_golden(name):
    case, ref = load_golden(name)
    I, qx, qy, qz = oracle.diffraction(*case.args())
    for got, want in zip((qx, qy, qz), (ref.qx, ref.qy, ref.qz)):
        assert np.array_equal(got, want)
    assert I.shape == case.shape
    np.testing.assert_allclose(I, ref.I, rtol=1e-12, atol=1e-13 * ref.I.max())


def test_threaded_oracle_equals_serial():
    case, _ = load_golden("random_24x16x10_dense")
    a = oracle.diffraction(*case.args(), threads=1)[0]
    b = oracle.diffraction(*case.args(), threads=3)[0]
    np.testing.assert_allclose(a, b, rtol=1e-13, atol=1e-14 * a.max())


@pytest.mark.parametrize("hkl", analytic.REFLECTIONS, ids=lambda h: "".join(map(str, h)))
@pytest.mark.parametrize("variant", list(analytic.VARIANTS))
def test_structure_factor(variant, hkl):
    analytic.check_structure_factor(oracle.diffraction, variant, hkl)


def test_variant_symmetry():
    analytic.check_variant_symmetry(oracle.diffraction)


@pytest.mark.parametrize("variant", ["c+", "a1+", "a2+"])
def test_spontaneous_strain(variant):
    analytic.check_spontaneous_strain(oracle.diffraction, variant)


@pytest.mark.parametrize("p", [8, 16])
@pytest.mark.parametrize("t", [8, 16])
def test_thickness_fringes(t, p):
    analytic.check_thickness_fringes(oracle.diffraction, t, p)


@pytest.mark.parametrize("p", [8, 16])
@pytest.mark.parametrize("t", [8, 16])
def test_domain_satellites(t, p):
    analytic.check_domain_satellites(oracle.diffraction, t, p)


def test_planted_signals():
    analytic.check_uniform_p_peaks_at_g(oracle.diffraction)
    analytic.check_uz_ramp_shifts_peak(oracle.diffraction)
    analytic.check_stripe_satellites_along_x_only(oracle.diffraction)
    analytic.check_phase_and_region_weights(oracle.diffraction)


def test_planted_oracle_fails_on_a_planted_mistake():
    """The checks catch a wrong sign in the phase factor (planted in a copy of the oracle, on the CPU)."""
    def wrong(params, atoms, oPhase, oStruc, u, region):
        atoms2 = type(atoms)(**vars(atoms))
        atoms2.fAtom = np.conj(atoms.fAtom)
        return oracle.diffraction(params, atoms2, oPhase, oStruc, u, region)
    with pytest.raises(AssertionError):
        analytic.check_structure_factor(wrong, "c+", (0, 0, 2))
