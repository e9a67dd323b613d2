"""
Analytic known answers of the reference's own test-suite, restated as direct calls.

The reference checks its CLI end to end on synthetic FerroDyn runs
(tests/test_single_domain.py, tests/test_a1a2_domains.py, tests/test_planted.py).
HDF5 is not available here, so the same runs are built in memory with the same
constants (tests/test_planted.py:21-45) and passed to ``diffraction()`` directly.
"""

import math

import numpy as np

from qpop_diffraction_b200 import workloads

DX = 1.0         # nm, one cell (tests/test_planted.py:22)
A = 0.4          # nm, lattice constant of parameter.atom.in (tests/test_planted.py:23)
POS = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]])
FORM = np.array([19.3678 + 0.746466j, 40.5697 + 1.67439j, 8.035 + 0.021j, 8.035 + 0.021j, 8.035 + 0.021j])
SHIFT = np.array([[1.01, 1.01, 1.01], [-0.56, -0.56, -0.56],
                  [-3.66, -3.15, -3.15], [-3.15, -3.66, -3.15], [-3.15, -3.15, -3.66]]) * 1e-11  # m per C/m^2
PS = 0.75        # C/m^2 (tests/test_single_domain.py:24)
VARIANTS = {"c+": (0, 0, 1), "c-": (0, 0, -1), "a1+": (1, 0, 0), "a1-": (-1, 0, 0), "a2+": (0, 1, 0), "a2-": (0, -1, 0)}
REFLECTIONS = [(0, 0, 2), (2, 0, 0), (0, 2, 0), (1, 1, 1)]


def reciprocal(hkl):
    return 2 * math.pi * np.array(hkl, dtype=float) / A


def structure_factor(q, P):
    """sum_a f_a exp(-i q . (R_a + d_a)), positions in nm, P in C/m^2 (tests/test_single_domain.py:36-39)."""
    r = POS * A + SHIFT * np.asarray(P) / 1e-9
    return np.sum(FORM * np.exp(-1j * (r @ q)))


def atoms_for(q00):
    """The PbTiO3 cell of the reference's fixtures: su per atom along P, converted m -> nm (AtomList.setup)."""
    su = np.zeros((3, 3, 1, len(POS)))
    for d in range(3):
        su[d, d, 0, :] = SHIFT[:, d] / 1e-9
    return workloads.make_atoms(np.eye(3) * A, q00, POS, FORM[None, :], su)


L0 = 1e-9        # src/python/constants.py:8
DX_SI = 1e-9     # m, Mesh DX/DY/DZ of the reference fixtures (tests/test_planted.py:22)
A_SI = 4e-10     # m, LatticeConstants of both materials (tests/test_planted.py:59)


def boundary(P, u_si, q00, mat=None, fe=(1,), region=None, phase=None, thin_film=False):
    """
    The arguments the reference CLI hands to diffraction() for a synthetic FerroDyn run
    (src/python/cli.py:174-221), restated with its arithmetic:

    - grid spacing lx / nx with lx = nx DX / L0 (src/python/size_context.py:79-81, :185-187);
    - u in nm from metres (src/python/io_utils.py:71);
    - one-hot phases of the FE materials, region = their sum times the region weight
      (src/python/cli.py:189-199);
    - strainAvg and the out-of-plane mismatch dc = c_m(T) / aC_z - 1 per material
      (src/python/size_context.py:124-159), the u_z ramp (cumsum_z dc - dc / 2) dz
      (src/python/cli.py:207-217).

    P is (3, nx, ny, nz) in C/m^2 and u_si in metres; mat (nx, ny, nz) material indices
    (default: all material 1, the film).  Both materials have lattice constant A_SI.
    """
    shape = P.shape[1:]
    nx, ny, nz = shape
    n = int(np.prod(shape))
    spacing = [(m * DX_SI / L0) / m for m in shape]
    params = workloads.make_params(shape, spacing, len(fe))
    atoms = atoms_for(q00)
    lattice = A_SI * (1.0 + 0.0) / L0
    aC = np.diag(atoms.aC)
    params.strainAvg = np.zeros(6)
    params.strainAvg[:2] = np.array([lattice, lattice]) / aC[:2] - 1.0
    dc_m = np.array([lattice, lattice]) / aC[2] - 1.0
    mat = np.ones(shape, dtype=int) if mat is None else mat
    onehot = np.stack([(mat == m) for m in fe]).astype(np.float64)
    reg = onehot.sum(axis=0).ravel()
    oPhase = onehot.ravel() if phase is None else np.asarray(phase, dtype=np.float32).astype(np.float64).ravel()
    if region is not None:
        reg = reg * np.asarray(region, dtype=np.float32).astype(np.float64).ravel()
    dc = dc_m[mat]
    uz_ref = ((np.cumsum(dc, axis=2) - 0.5 * dc) * spacing[2]).ravel()
    u = (np.asarray(u_si, dtype=np.float64) / L0).reshape(3, n)
    u[2] += uz_ref
    return params, atoms, oPhase, P.reshape(-1).astype(np.float64), u.reshape(-1), reg


def run_case(P, u, q00, region=None, phase=None):
    """A bulk run of the film material everywhere; u in nm (DX = 1 nm cells)."""
    return boundary(P, np.asarray(u) * L0, q00, region=region, phase=phase)


def at(I, axes, target):
    """Intensity at the grid point nearest the q target (tests/test_planted.py:126-129)."""
    idx = [int(np.argmin(np.abs(ax - t))) for ax, t in zip(axes, target)]
    return I[tuple(idx)]


def peak(I, axes):
    i = np.unravel_index(np.argmax(I), I.shape)
    return np.array([axes[d][i[d]] for d in range(3)])


def single_domain(P, hkl, shape=(40, 30, 20), strain=None):
    """Uniform P around reflection hkl; strain (axis, e) adds u_axis = e r_axis (tests/test_single_domain.py:42-54)."""
    fields = np.zeros((3,) + shape)
    for d in range(3):
        fields[d] = P[d]
    u = np.zeros((3,) + shape)
    if strain is not None:
        d, e = strain
        r = np.arange(shape[d]) * DX
        u[d] = e * r.reshape([-1 if i == d else 1 for i in range(3)])
    return run_case(fields, u, reciprocal(hkl))


def a1a2_film(t, p, shape=(32, 48, 32), substrate=8):
    """a1/a2 stripes of period p in a film t cells thick on a non-scattering substrate (tests/test_a1a2_domains.py:38-47)."""
    nx, ny, nz = shape
    i = np.arange(nx)[:, None, None]
    j = np.arange(ny)[None, :, None]
    a1 = np.broadcast_to(((i + j) % p) < p // 2, shape)
    P = np.zeros((3,) + shape)
    P[0] = PS * a1
    P[1] = PS * ~a1
    mat = np.zeros(shape, dtype=int)
    mat[:, :, substrate:substrate + t] = 1
    G = np.array([2 * math.pi * 2 / A, 0.0, 0.0])
    return boundary(P, np.zeros_like(P), G, mat=mat), G


# ---------------------------------------------------------------------------------------------
# Checks, each taking the diffraction callable under test.  rtol / floor: tolerances of the
# reference's own tests for a float64 path, relaxed to the float32 contract by the caller.
# ---------------------------------------------------------------------------------------------

def check_structure_factor(diffraction, variant, hkl, rtol=1e-9):
    """Peak at G and I(G) = |F(G)|^2 / V^2 (tests/test_single_domain.py:51-58)."""
    P = PS * np.array(VARIANTS[variant])
    G = reciprocal(hkl)
    I, *axes = diffraction(*single_domain(P, hkl))
    np.testing.assert_allclose(peak(I, axes), G, atol=1e-9)
    np.testing.assert_allclose(at(I, axes, G), abs(structure_factor(G, P)) ** 2 / A ** 6, rtol=rtol)


def check_variant_symmetry(diffraction, rtol=1e-12):
    """Cubic symmetry, shifts perpendicular to G invisible, Friedel's law broken (tests/test_single_domain.py:61-78)."""
    I = {}
    for name, P in list(VARIANTS.items()) + [("0", (0, 0, 0))]:
        for hkl in [(0, 0, 2), (2, 0, 0), (0, 2, 0)]:
            out, *axes = diffraction(*single_domain(PS * np.array(P), hkl))
            I[name, hkl] = at(out, axes, reciprocal(hkl))
    for sign in "+-":
        parallel = [I["c" + sign, (0, 0, 2)], I["a1" + sign, (2, 0, 0)], I["a2" + sign, (0, 2, 0)]]
        np.testing.assert_allclose(parallel, parallel[0], rtol=rtol)
        perpendicular = [I["a1" + sign, (0, 0, 2)], I["a2" + sign, (0, 0, 2)], I["c" + sign, (2, 0, 0)]]
        np.testing.assert_allclose(perpendicular, I["0", (0, 0, 2)], rtol=rtol)
    assert abs(I["c+", (0, 0, 2)] / I["c-", (0, 0, 2)] - 1) > 1e-3


def check_spontaneous_strain(diffraction, variant):
    """A strain e along P moves the reflections along P to G (1 - e) (tests/test_single_domain.py:81-96)."""
    e = 0.02
    shape = (40, 30, 20)
    axis = int(np.argmax(np.abs(VARIANTS[variant])))
    for hkl in [(0, 0, 2), (2, 0, 0), (0, 2, 0)]:
        I, *axes = diffraction(*single_domain(PS * np.array(VARIANTS[variant]), hkl, shape, strain=(axis, e)))
        G = reciprocal(hkl)
        expected = G.copy()
        expected[axis] = G[axis] / (1 + e)
        dq = 2 * math.pi / (np.array(shape) * DX)
        assert np.all(np.abs(peak(I, axes) - expected) < dq / 2), (hkl, peak(I, axes), expected)


def check_thickness_fringes(diffraction, t, p, rtol=1e-6, zero=1e-20):
    """Laue fringes sinc^2(k_z T / 2) |F(G + k_z)|^2 / |F(G)|^2 along q_z (tests/test_a1a2_domains.py:50-62)."""
    args, G = a1a2_film(t, p)
    I, *axes = diffraction(*args)
    F1 = lambda q: structure_factor(q, (PS, 0.0, 0.0))
    F2 = lambda q: structure_factor(q, (0.0, PS, 0.0))
    F = lambda q: (F1(q) + F2(q)) / 2
    I0 = at(I, axes, G)
    for kz in 2 * math.pi * np.fft.fftfreq(32, 1.0):
        qz = G + np.array([0.0, 0.0, kz])
        expected = np.sinc(kz * t / (2 * math.pi)) ** 2 * abs(F(qz)) ** 2 / abs(F(G)) ** 2
        if expected > 1e-8:
            np.testing.assert_allclose(at(I, axes, qz) / I0, expected, rtol=rtol)
        elif expected < 1e-20:
            assert at(I, axes, qz) < zero * I0, kz


def check_domain_satellites(diffraction, t, p, zero=1e-20):
    """First-order satellites along (1,1,0) with the square-wave intensity; none along (1,-1,0) nor at second
    order (tests/test_a1a2_domains.py:65-80)."""
    args, G = a1a2_film(t, p)
    I, *axes = diffraction(*args)
    F1 = lambda q: structure_factor(q, (PS, 0.0, 0.0))
    F2 = lambda q: structure_factor(q, (0.0, PS, 0.0))
    kappa = 2 * math.pi / p
    k1 = kappa * np.array([1.0, 1.0, 0.0])
    c1 = np.mean(np.where(np.arange(p) < p // 2, 1.0, 0.0) * np.exp(-2j * math.pi * np.arange(p) / p))
    S = np.sinc(kappa / (2 * math.pi)) ** 2
    expected = S ** 2 * abs(c1) ** 2 * abs(F1(G + k1) - F2(G + k1)) ** 2 / abs((F1(G) + F2(G)) / 2) ** 2
    I0 = at(I, axes, G)
    np.testing.assert_allclose(at(I, axes, G + k1) / I0, expected, rtol=1e-2)
    np.testing.assert_allclose(at(I, axes, G - k1) / I0, abs(c1) ** 2 * S ** 2 * abs(F1(G - k1) - F2(G - k1)) ** 2
                               / abs((F1(G) + F2(G)) / 2) ** 2, rtol=1e-2)
    assert at(I, axes, G + kappa * np.array([1.0, -1.0, 0.0])) < zero * I0
    assert at(I, axes, G + 2 * k1) < zero * I0


PLANTED = (48, 32, 20)  # tests/test_planted.py:21
G002 = 2 * math.pi * 2 / A


def check_uniform_p_peaks_at_g(diffraction):
    """tests/test_planted.py:141-146."""
    P = np.zeros((3,) + PLANTED)
    P[2] = 0.5
    I, *axes = diffraction(*run_case(P, np.zeros_like(P), (0.0, 0.0, G002)))
    np.testing.assert_allclose(peak(I, axes), [0.0, 0.0, G002], atol=1e-9)


def check_uz_ramp_shifts_peak(diffraction):
    """u_z = e z moves the 002 peak to G (1 - e) (tests/test_planted.py:149-158)."""
    e = 0.02
    u = np.zeros((3,) + PLANTED)
    u[2] = e * DX * np.arange(PLANTED[2])[None, None, :]
    I, *axes = diffraction(*run_case(np.zeros_like(u), u, (0.0, 0.0, G002)))
    dqz = 2 * math.pi / (PLANTED[2] * DX)
    assert abs(peak(I, axes)[2] - G002 * (1 - e)) < dqz


def check_stripe_satellites_along_x_only(diffraction, ratio=1e6):
    """180-degree Pz stripes along x give satellites on q_x only (tests/test_planted.py:161-173)."""
    L = 16
    P = np.zeros((3,) + PLANTED)
    P[2] = np.where((np.arange(PLANTED[0]) // (L // 2)) % 2 == 0, 0.5, -0.5)[:, None, None]
    I, *axes = diffraction(*run_case(P, np.zeros_like(P), (0.0, 0.0, G002)))
    k = 2 * math.pi / (L * DX)
    on_x = at(I, axes, (k, 0.0, G002))
    on_y = at(I, axes, (0.0, k, G002))
    assert on_x > 1e-6 * I.max()
    assert on_x > ratio * on_y


def check_phase_and_region_weights(diffraction, rtol=1e-6, lit=1e-20):
    """Weight = phase fraction x region: uniform 0.6, 0.5 scale I by 0.3^2; a half region halves the amplitude
    (tests/test_planted.py:206-219)."""
    P = np.zeros((3,) + PLANTED)
    P[2] = 0.5
    u = np.zeros_like(P)
    q00 = (0.0, 0.0, G002)
    plain, *axes = diffraction(*run_case(P, u, q00))
    uniform, *_ = diffraction(*run_case(P, u, q00, phase=np.full(PLANTED, 0.6), region=np.full(PLANTED, 0.5)))
    half = (np.arange(PLANTED[0]) < PLANTED[0] // 2)[:, None, None] * np.ones(PLANTED)
    halved, *_ = diffraction(*run_case(P, u, q00, region=half))
    # Above the 1e-50 floor only: for these uniform fields the reference's own FFT returns exact zeros
    # off the Bragg peak, so floored voxels are 1e-50 in both runs and cannot scale by 0.09.
    mask = plain > lit * plain.max()
    np.testing.assert_allclose(uniform[mask], 0.09 * plain[mask], rtol=rtol)
    np.testing.assert_allclose(at(halved, axes, (0.0, 0.0, G002)), 0.25 * at(plain, axes, (0.0, 0.0, G002)), rtol=rtol)
