"""
Parity of the CUDA path with the reference, through the C ABI, on a B200.

Tolerances (written per test):
  * float64 (QPD_FP64): the reference's own mgpu-vs-Python bar, I rtol 1e-9 with atol 1e-12 I_max
    (tests/test_mgpu.py:53 of the reference); q axes bit-exact.
  * float32 (QPD_FP32, float64 phase reduction): max |dI| / I_max <= 1e-5 and relative error
    <= 1e-3 on voxels above 1e-6 I_max; q axes bit-exact.
"""

import numpy as np
import pytest

import analytic
from conftest import fp32_errors, golden_names, load_golden

pytestmark = pytest.mark.gpu

MODES = [("fp32", "fused"), ("fp64", "fused"), ("fp64", "plain"), ("fp32", "plain")]


def run(case, precision, schedule):
    from qpop_diffraction_b200 import diffraction
    return diffraction(*case.args(), precision=precision, schedule=schedule)


def assert_parity(I, ref, precision):
    if precision == "fp64":
        np.testing.assert_allclose(I, ref, rtol=1e-9, atol=1e-12 * ref.max())
    else:
        dmax, rel = fp32_errors(I, ref)
        assert dmax <= 1e-5, dmax
        assert rel <= 1e-3, rel


@pytest.mark.parametrize("precision,schedule", MODES)
@pytest.mark.parametrize("name", golden_names())
def test_matches_reference_golden(gpu, name, precision, schedule):
    case, ref = load_golden(name)
    I, qx, qy, qz = run(case, precision, schedule)
    for got, want in zip((qx, qy, qz), (ref.qx, ref.qy, ref.qz)):
        assert np.array_equal(got, want)
    assert I.shape == case.shape and I.dtype == np.float64
    assert_parity(I, ref.I, precision)


def test_device_path_equals_host_path(gpu):
    torch = gpu
    from qpop_diffraction_b200 import Plan, crystal_from
    case, ref = load_golden("random_24x16x10_dense")
    p = case.params
    with Plan(case.shape, (p.dx, p.dy, p.dz), p.nPhase, p.nStruc) as plan:
        plan.set_crystal(crystal_from(p, case.atoms))
        host = plan.run_host(case.oPhase, case.oStruc, case.u, case.region)
        dev = torch.device("cuda", 0)
        packed = plan.pack(*(torch.from_numpy(a).to(dev) for a in (case.oPhase, case.oStruc, case.u, case.region)))
        assert packed["wdense"] is not None  # overlapping phase fractions
        out = plan.run_device(packed)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), host)


def test_plan_reuse_and_second_reflection(gpu):
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    from oracle import diffraction_oracle as oracle
    a = workloads.config2(shape=(16, 16, 104), hkl=(0, 0, 2))
    b = workloads.config2(shape=(16, 16, 104), hkl=(1, 0, 3))
    p = a.params
    with Plan(a.shape, (p.dx, p.dy, p.dz), p.nPhase, p.nStruc, precision="fp64") as plan:
        out = {}
        for case in (a, b, a):
            plan.set_crystal(crystal_from(case.params, case.atoms))
            out.setdefault(case.name, []).append(plan.run_host(case.oPhase, case.oStruc, case.u, case.region))
        assert np.array_equal(out[a.name][0], out[a.name][1])
        for case in (a, b):
            ref = oracle.diffraction(*case.args())[0]
            assert_parity(out[case.name][0], ref, "fp64")


@pytest.mark.parametrize("shape,precisions", [
    ((1, 1, 1), ("fp64", "fp32")), ((1, 1, 7), ("fp64", "fp32")), ((5, 1, 1), ("fp64", "fp32")),
    ((2, 3, 1), ("fp64", "fp32")), ((64, 1, 9), ("fp64", "fp32")), ((3, 37, 2), ("fp64", "fp32")),
    ((41, 2, 3), ("fp64", "fp32")), ((4, 4, 2048), ("fp64", "fp32")), ((2, 2, 4096), ("fp32",))])
def test_edge_shapes(gpu, shape, precisions):
    """Axes of length 1, prime lengths without a specialised radix (37, 41), the longest z per precision."""
    from qpop_diffraction_b200 import workloads
    from oracle import diffraction_oracle as oracle
    case = workloads.random_case(shape, seed=sum(shape), nPhase=1, weights="region")
    ref = oracle.diffraction(*case.args())[0]
    for precision in precisions:
        I = run(case, precision, "fused")[0]
        assert_parity(I, ref, precision)


@pytest.mark.parametrize("shape", [(512, 2, 104), (2, 512, 104), (256, 128, 64), (128, 256, 68), (1024, 2, 32),
                                   (2, 1024, 128), (32, 64, 128), (64, 32, 32), (512, 2, 7), (2, 256, 9),
                                   (4000, 2, 68), (2, 4000, 68), (3, 4000, 1)])
def test_specialised_axis_lengths(gpu, shape):
    """Every axis length with a compile-time kernel, in both strided positions, even and odd nz."""
    from qpop_diffraction_b200 import workloads
    from oracle import diffraction_oracle as oracle
    case = workloads.random_case(shape, seed=sum(shape) + 7, nPhase=2, weights="onehot", strain=True)
    ref = oracle.diffraction(*case.args())[0]
    for precision in ("fp32", "fp64"):
        assert_parity(run(case, precision, "fused")[0], ref, precision)


def test_specialised_equals_generic(gpu, monkeypatch):
    """The compile-time kernels and the generic ones compute the same volume (QPOP_B200_GENERIC=1)."""
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    case = workloads.config2(shape=(64, 64, 104), hkl=(1, 0, 3))
    p = case.params
    out = []
    for generic in ("0", "1"):
        monkeypatch.setenv("QPOP_B200_GENERIC", generic)
        with Plan(case.shape, (p.dx, p.dy, p.dz), p.nPhase, p.nStruc) as plan:
            plan.set_crystal(crystal_from(p, case.atoms))
            out.append(plan.run_host(case.oPhase, case.oStruc, case.u, case.region))
    dmax = np.abs(out[0] - out[1]).max() / out[1].max()
    assert dmax <= 1e-6, dmax


def test_nothing_scatters(gpu):
    """All weights zero: every voxel is the 1e-50 floor, as in the reference (src/python/diffraction.py:111)."""
    from qpop_diffraction_b200 import workloads
    case = workloads.random_case((6, 5, 4), seed=3)
    case.region = np.zeros_like(case.region)
    for precision in ("fp32", "fp64"):
        I = run(case, precision, "fused")[0]
        assert np.all(I == 1e-50)


def test_errors_are_exceptions_not_aborts(gpu):
    from qpop_diffraction_b200 import Plan, crystal_from, workloads, _native
    case = workloads.random_case((6, 5, 4), seed=3)
    p = case.params
    with Plan(case.shape, (p.dx, p.dy, p.dz), 1) as plan:
        with pytest.raises(RuntimeError):
            plan.run_host(case.oPhase, case.oStruc, case.u, case.region)   # no crystal yet
        plan.set_crystal(crystal_from(p, case.atoms))
        with pytest.raises(ValueError):
            plan.run_host(case.oPhase[:-1], case.oStruc, case.u, case.region)
    with pytest.raises(ValueError):
        Plan((4, 4, 5000), (1, 1, 1), 1)          # z longer than the z stage handles
    with pytest.raises(ValueError):
        Plan((4, 4, 4), (1, 1, 1), 9)             # more phases than the packed layout holds
    with Plan(case.shape, (p.dx, p.dy, p.dz), 1, hbm_budget=4096) as plan:
        with pytest.raises(MemoryError):
            plan.set_crystal(crystal_from(p, case.atoms))
    with pytest.raises(_native.QpdError):
        Plan(case.shape, (p.dx, p.dy, p.dz), 1, device=1 << 20)


# ---------------- the reference's analytic known answers on the GPU ----------------

def ours(precision):
    from qpop_diffraction_b200 import diffraction

    def call(*args):
        return diffraction(*args, precision=precision)
    return call


@pytest.mark.parametrize("hkl", analytic.REFLECTIONS, ids=lambda h: "".join(map(str, h)))
@pytest.mark.parametrize("variant", list(analytic.VARIANTS))
def test_structure_factor(gpu, variant, hkl):
    analytic.check_structure_factor(ours("fp64"), variant, hkl)
    analytic.check_structure_factor(ours("fp32"), variant, hkl, rtol=1e-5)


def test_variant_symmetry(gpu):
    analytic.check_variant_symmetry(ours("fp64"))
    analytic.check_variant_symmetry(ours("fp32"), rtol=1e-5)


@pytest.mark.parametrize("variant", ["c+", "a1+", "a2+"])
def test_spontaneous_strain(gpu, variant):
    analytic.check_spontaneous_strain(ours("fp64"), variant)
    analytic.check_spontaneous_strain(ours("fp32"), variant)


@pytest.mark.parametrize("p", [8, 16])
@pytest.mark.parametrize("t", [8, 16])
def test_thickness_fringes(gpu, t, p):
    analytic.check_thickness_fringes(ours("fp64"), t, p)
    # float32: fringes to the fp32 contract, zeros below the float32 noise floor
    analytic.check_thickness_fringes(ours("fp32"), t, p, rtol=1e-3, zero=1e-9)


@pytest.mark.parametrize("p", [8, 16])
@pytest.mark.parametrize("t", [8, 16])
def test_domain_satellites(gpu, t, p):
    analytic.check_domain_satellites(ours("fp64"), t, p)
    analytic.check_domain_satellites(ours("fp32"), t, p, zero=1e-9)


def test_planted_signals(gpu):
    for precision, ratio in (("fp64", 1e6), ("fp32", 1e3)):
        f = ours(precision)
        analytic.check_uniform_p_peaks_at_g(f)
        analytic.check_uz_ramp_shifts_peak(f)
        analytic.check_stripe_satellites_along_x_only(f, ratio=ratio)
        if precision == "fp64":
            analytic.check_phase_and_region_weights(f)
        else:  # float32: voxels above its noise floor
            analytic.check_phase_and_region_weights(f, rtol=1e-5, lit=1e-6)


@pytest.mark.parametrize("shape,weights", [((64, 48, 104), "onehot"), ((40, 36, 68), "region"), ((24, 30, 68), "onehot")])
def test_prime_factor_z_stage_equals_stockham(gpu, monkeypatch, shape, weights):
    """The register-fused prime-factor z stage (zstage_pfa) and the Stockham one compute the same volume."""
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    from oracle import diffraction_oracle as oracle
    case = workloads.random_case(shape, seed=sum(shape), nPhase=2, weights=weights, strain=True, hkl=(1, 0, 3))
    p = case.params
    out = []
    for knob in ("0", "1"):
        monkeypatch.setenv("QPOP_B200_ZPFA", knob)
        with Plan(case.shape, (p.dx, p.dy, p.dz), p.nPhase, p.nStruc) as plan:
            plan.set_crystal(crystal_from(p, case.atoms))
            out.append(plan.run_host(case.oPhase, case.oStruc, case.u, case.region))
    assert np.abs(out[0] - out[1]).max() / out[0].max() <= 1e-6
    ref = oracle.diffraction(*case.args())[0]
    assert_parity(out[1], ref, "fp32")


def test_y_fastest_route_at_4000x4000x68(gpu, monkeypatch):
    """The 4000 x 4000 x 68 route (z stage writing y-fastest fields, bulk y pass, swapped x pass)
    against the z-fastest route of the same kernels, on the full config-3 volume, with the
    shared-memory Stockham 4000-point passes (QPOP_B200_N4K=0), whose two routes round differently.
    The register-resident passes compute both routes with the same arithmetic (tested below)."""
    torch = gpu
    monkeypatch.setenv("QPOP_B200_N4K", "0")
    torch.cuda.empty_cache()  # blocks an earlier test left in the caching allocator
    free, _ = torch.cuda.mem_get_info(0)
    if free < 160e9:
        pytest.skip("needs about 150 GB of free device memory")
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    shape = (4000, 4000, 68)
    params, inputs = workloads.gpu_snapshot("twin", shape, seed=3, device="cuda:0", n_phase=1)
    crystal = crystal_from(params, workloads.config3_crystal(3, (1, 1, 3)))
    out = torch.empty(shape, dtype=torch.float64, device="cuda:0")
    for knob in ("0", "1"):
        monkeypatch.setenv("QPOP_B200_YFAST", knob)
        with Plan(shape, (params.dx, params.dy, params.dz), 1, 3, precision="fp32") as plan:
            plan.set_crystal(crystal)
            plan.run_device(inputs, out)
            torch.cuda.synchronize()
            plan.device_status()
        if knob == "0":
            ref = out.clone()
        else:
            dmax = ((out - ref).abs().max() / ref.max()).item()
            assert dmax <= 1e-6, dmax
            # the routes round differently (two-level twiddles in the bulk y pass): identical bits would
            # mean the y-fastest route did not run
            assert not torch.equal(out, ref)


def test_register_4000_point_passes_at_4000x4000x68(gpu, monkeypatch):
    """The register-resident 4000-point y and x passes (qpd_n4000.cu, the default) against the
    shared-memory Stockham passes (QPOP_B200_N4K=0) on the full config-3 volume."""
    torch = gpu
    torch.cuda.empty_cache()  # blocks an earlier test left in the caching allocator
    free, _ = torch.cuda.mem_get_info(0)
    if free < 160e9:
        pytest.skip("needs about 150 GB of free device memory")
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    shape = (4000, 4000, 68)
    params, inputs = workloads.gpu_snapshot("twin", shape, seed=3, device="cuda:0", n_phase=1)
    crystal = crystal_from(params, workloads.config3_crystal(3, (1, 1, 3)))
    out = torch.empty(shape, dtype=torch.float64, device="cuda:0")
    for knob in ("0", "1"):
        monkeypatch.setenv("QPOP_B200_N4K", knob)
        with Plan(shape, (params.dx, params.dy, params.dz), 1, 3, precision="fp32") as plan:
            plan.set_crystal(crystal)
            plan.run_device(inputs, out)
            torch.cuda.synchronize()
            plan.device_status()
        if knob == "0":
            ref = out.clone()
        else:
            dmax = ((out - ref).abs().max() / ref.max()).item()
            assert dmax <= 1e-6, dmax
            # different twiddle and butterfly rounding: identical bits would mean the new passes did not run
            assert not torch.equal(out, ref)
    # with the register-resident passes the z-fastest route (strided y pass) gives the same bits as the
    # y-fastest one (bulk y pass): the same transforms and folds in the same order
    monkeypatch.setenv("QPOP_B200_N4K", "1")
    for knob, dst in (("0", ref), ("1", out)):
        monkeypatch.setenv("QPOP_B200_YFAST", knob)
        with Plan(shape, (params.dx, params.dy, params.dz), 1, 3, precision="fp32") as plan:
            plan.set_crystal(crystal)
            plan.run_device(inputs, dst)
            torch.cuda.synchronize()
            plan.device_status()
    assert torch.equal(out, ref)


def test_direct_sum_voxels_at_4000x4000x68(gpu):
    """The full 4000 x 4000 x 68 volume (default route) against float64 direct sums over all 1.088e9
    cells at 64 voxels: the 32 brightest of the result and 32 drawn at random.  Independent of every
    FFT kernel; the per-precision contract is the float32 one of the smaller grids."""
    torch = gpu
    torch.cuda.empty_cache()  # blocks an earlier test left in the caching allocator
    free, _ = torch.cuda.mem_get_info(0)
    if free < 160e9:
        pytest.skip("needs about 150 GB of free device memory")
    from direct_dft import crystal_constants, direct_intensity, fft_index_to_shifted, shifted_to_fft_index
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    shape = (4000, 4000, 68)
    params, inputs = workloads.gpu_snapshot("twin", shape, seed=3, device="cuda:0", n_phase=1)
    atoms = workloads.config3_crystal(3, (1, 1, 3))
    out = torch.empty(shape, dtype=torch.float64, device="cuda:0")
    with Plan(shape, (params.dx, params.dy, params.dz), 1, 3, precision="fp32") as plan:
        plan.set_crystal(crystal_from(params, atoms))
        plan.run_device(inputs, out)
        torch.cuda.synchronize()
        plan.device_status()
    top = torch.topk(out.view(-1), 32).indices.cpu().numpy()
    sx, sy, sz = np.unravel_index(top, shape)
    inv = [shifted_to_fft_index(s) for s in shape]
    bright = np.stack([inv[0][sx], inv[1][sy], inv[2][sz]], axis=1)
    rng = np.random.default_rng(11)
    rand = np.stack([rng.integers(0, s, 32) for s in shape], axis=1)
    vox = np.concatenate([bright, rand])
    pos = [fft_index_to_shifted(s) for s in shape]
    sel = [torch.from_numpy(pos[d][vox[:, d]]).to(out.device) for d in range(3)]
    got = out[sel[0], sel[1], sel[2]].cpu().numpy()
    del out
    torch.cuda.empty_cache()
    spacing = (params.dx, params.dy, params.dz)
    want = direct_intensity(torch, shape, spacing, *crystal_constants(params, atoms), inputs["P"], inputs["U"],
                            inputs["phase"], inputs["weight"], vox)
    Imax = want.max()
    big = want > 1e-6 * Imax
    dmax = np.abs(got - want).max() / Imax
    rel = (np.abs(got - want)[big] / want[big]).max()
    print(f"direct sums at {len(vox)} voxels: max |dI|/I_max {dmax:.2e}, max rel {rel:.2e} over {big.sum()} voxels")
    assert dmax <= 1e-5 and big.sum() >= 32 and rel <= 1e-3, (dmax, rel, big.sum())
