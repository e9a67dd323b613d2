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


# ---------------- the FerroDyn example and the boundary-input preparation ----------------

def test_oracle_matches_reference_on_the_ferrodyn_example():
    """The disordered polar-vortex example, prepared as the CLI does, against the reference's own run."""
    from conftest import load_example
    from oracle import fields_oracle
    ex = load_example()
    oPhase, oStruc, u, region = fields_oracle.prepare(ex.P, ex.mat, ex.dc, ex.phase_of, ex.ramp_dz, region=ex.region)
    assert np.array_equal(u[2 * (u.size // 3):], ex.uz_ref)
    I, qx, qy, qz = oracle.diffraction(ex.params, ex.atoms, oPhase, oStruc, u, region)
    for got, want in zip((qx, qy, qz), (ex.qx, ex.qy, ex.qz)):
        assert np.array_equal(got, want)
    np.testing.assert_allclose(I, ex.I, rtol=1e-12, atol=1e-13 * ex.I.max())


def test_fields_oracle_restates_the_cli_prep():
    """prepare() against a literal transcription of src/python/cli.py:187-217 on a cropped two-material stack."""
    from oracle import fields_oracle
    rng = np.random.default_rng(5)
    nxf, nyf, nzf = 6, 5, 20
    lims = (1, 4), (0, 3), (3, 14)
    sl = tuple(slice(a, b + 1) for a, b in lims)
    mat_xyz = np.where(np.arange(nzf)[None, None, :] < 8, 0, 2) * np.ones((nxf, nyf, 1), dtype=int)
    mat_xyz[rng.random(mat_xyz.shape) < 0.1] = 1                       # air pockets: not FE
    fe_ids, dc_table, dz = [0, 2], np.array([-0.011, 0.0, 0.024]), 0.4
    P_xyz = rng.standard_normal((3, nxf, nyf, nzf)).astype(np.float32)
    u_xyz = (rng.standard_normal((3, nxf, nyf, nzf)) * 1e-11).astype(np.float32)
    reg_xyz = rng.random((nxf, nyf, nzf)).astype(np.float32)
    # the reference's arithmetic, step by step
    oPhase = np.stack([mat_xyz[sl] == m for m in fe_ids]).astype(np.float64)
    region = oPhase.sum(axis=0).ravel() * reg_xyz[sl].astype(np.float64).ravel()
    dc = dc_table[mat_xyz]
    uz_ref = ((np.cumsum(dc, axis=2) - 0.5 * dc) * dz)[sl].ravel()
    u = np.stack([c[sl] for c in u_xyz]).astype(np.float64).ravel() / 1e-9
    n = region.size
    u[2 * n:] += uz_ref
    oStruc = np.stack([c[sl] for c in P_xyz]).astype(np.float64).ravel()
    # the oracle, from file-order arrays
    f = lambda a: np.ascontiguousarray(a.transpose(*range(a.ndim - 3), a.ndim - 1, a.ndim - 2, a.ndim - 3))
    cut = (sl[2], sl[1], sl[0])
    got = fields_oracle.prepare(f(P_xyz)[(slice(None),) + cut], f(mat_xyz[sl[0], sl[1], :]), dc_table, [0, -1, 1], dz,
                                z0=lims[2][0], u=f(u_xyz)[(slice(None),) + cut], region=f(reg_xyz)[cut],
                                u_scale=1e9)
    for g, w in zip(got, (oPhase.ravel(), oStruc, u, region)):  # u: x * 1e9 (native u_scale) vs x / 1e-9
        np.testing.assert_allclose(g, w, rtol=1e-15, atol=1e-15 * np.abs(w).max())
