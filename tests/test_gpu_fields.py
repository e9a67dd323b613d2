"""
Boundary-input preparation on the GPU (qpd_pack_fields) against the oracle's restatement of the
reference CLI (oracle/fields_oracle.py, src/python/cli.py:174-217) and against the reference's own
run of its FerroDyn polar-vortex example.

Tolerances: the packed inputs are bit-exact with qpd_pack_device on the oracle-prepared float64
arrays (same rounding steps, in the same order); intensities follow the per-precision contract of
test_gpu_parity.py.
"""

import numpy as np
import pytest

from conftest import fp32_errors, load_example
from oracle import diffraction_oracle as oracle
from oracle import fields_oracle

pytestmark = pytest.mark.gpu


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def stack_case(seed, phase_file=False, displacement=True):
    """A cropped film-on-substrate stack: three materials (one of them air), dc != 0, region weights."""
    from qpop_diffraction_b200 import workloads
    rng = np.random.default_rng(seed)
    full = (30, 26, 50)                     # (nx, ny, nz) of the FerroDyn grid
    x0, y0, z0 = 3, 4, 12
    shape = (24, 20, 30)                    # crop
    nzf, nyf, nxf = full[2], full[1], full[0]
    mat = np.where(np.arange(nzf)[:, None, None] < 20, 0, 2) * np.ones((1, nyf, nxf), dtype=np.int8)
    mat[rng.random(mat.shape) < 0.08] = 1   # air: does not scatter
    mat = mat.astype(np.int8)
    dc = np.array([-0.0125, 0.0, 0.0213])
    phase_of = np.array([0, -1, 1], dtype=np.int32)
    crop = (slice(z0, z0 + shape[2]), slice(y0, y0 + shape[1]), slice(x0, x0 + shape[0]))
    f = lambda *s: rng.standard_normal(s).astype(np.float32)
    P = f(3, nzf, nyf, nxf)[(slice(None),) + crop] * np.float32(0.4)
    u = (f(3, nzf, nyf, nxf) * np.float32(2e-11))[(slice(None),) + crop] if displacement else None
    region = rng.random((nzf, nyf, nxf)).astype(np.float32)[crop]
    phase = None
    if phase_file:
        a = rng.random((nzf, nyf, nxf)).astype(np.float32)[crop]
        phase = np.stack([a, (1 - a).astype(np.float32)])
    spacing = (0.4, 0.4, 0.41)
    case = dict(P=np.ascontiguousarray(P), u=None if u is None else np.ascontiguousarray(u),
                phase=phase, region=np.ascontiguousarray(region),
                mat=np.ascontiguousarray(mat[:, crop[1], crop[2]]), z0=z0, dc=dc, phase_of=phase_of,
                ramp_dz=spacing[2])
    params = workloads.make_params(shape, spacing, 2, np.array([0.002, 0.002, 0, 0, 0, 0]))
    return shape, params, case


def prepared(case):
    return fields_oracle.prepare(case["P"], case["mat"], case["dc"], case["phase_of"], case["ramp_dz"], z0=case["z0"],
                                 u=case["u"], phase=case["phase"], region=case["region"], u_scale=1e9)


def pack_both(torch, plan, case):
    """(qpd_pack_fields on the fields, qpd_pack_device on the oracle-prepared float64 arrays)."""
    d = lambda a: None if a is None else to_dev(torch, a)
    got = plan.pack_fields(d(case["P"]), d(case["mat"]), case["dc"], case["phase_of"], case["ramp_dz"],
                           z0=case["z0"], u=d(case["u"]), phase=d(case["phase"]), region=d(case["region"]))
    oPhase, oStruc, u, region = prepared(case)
    want = plan.pack(*(to_dev(torch, a) for a in (oPhase, oStruc, u, region)))
    return got, want, (oPhase, oStruc, u, region)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("phase_file,displacement", [(False, True), (True, True), (False, False)])
def test_pack_fields_equals_pack_of_the_cli_prep(gpu, precision, phase_file, displacement):
    torch = gpu
    from qpop_diffraction_b200 import Plan
    shape, params, case = stack_case(21, phase_file, displacement)
    with Plan(shape, (params.dx, params.dy, params.dz), 2, precision=precision) as plan:
        got, want, _ = pack_both(torch, plan, case)
        torch.cuda.synchronize()
        for key in ("P", "U", "phase", "weight", "wdense"):
            assert (got[key] is None) == (want[key] is None), key
            if got[key] is not None:
                assert torch.equal(got[key], want[key]), key
        assert (got["wdense"] is not None) == phase_file


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_stack_through_the_hot_path_matches_the_oracle(gpu, precision):
    torch = gpu
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    shape, params, case = stack_case(22, phase_file=False)
    atoms = workloads.random_case(shape, seed=22, nPhase=2, weights="onehot", strain=True, hkl=(1, 0, 3)).atoms
    with Plan(shape, (params.dx, params.dy, params.dz), 2, precision=precision) as plan:
        plan.set_crystal(crystal_from(params, atoms))
        got, _, args = pack_both(torch, plan, case)
        I = plan.run_device(got).cpu().numpy()
        plan.device_status()
    ref = oracle.diffraction(params, atoms, *args)[0]
    if precision == "fp64":
        np.testing.assert_allclose(I, ref, rtol=1e-9, atol=1e-12 * ref.max())
    else:
        dmax, rel = fp32_errors(I, ref)
        assert dmax <= 1e-5 and rel <= 1e-3, (dmax, rel)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ferrodyn_example_matches_the_reference_run(gpu, precision):
    """The reference's disordered polar-vortex example, from its FerroDyn fields to the intensity."""
    torch = gpu
    from qpop_diffraction_b200 import Plan, crystal_from
    ex = load_example()
    p = ex.params
    with Plan(ex.shape, (p.dx, p.dy, p.dz), p.nPhase, p.nStruc, precision=precision) as plan:
        plan.set_crystal(crystal_from(p, ex.atoms))
        packed = plan.pack_fields(to_dev(torch, ex.P), to_dev(torch, ex.mat), ex.dc, ex.phase_of, ex.ramp_dz,
                                  region=to_dev(torch, ex.region))
        I = plan.run_device(packed).cpu().numpy()
        plan.device_status()
    if precision == "fp64":
        np.testing.assert_allclose(I, ex.I, rtol=1e-9, atol=1e-12 * ex.I.max())
    else:
        dmax, rel = fp32_errors(I, ex.I)
        assert dmax <= 1e-5 and rel <= 1e-3, (dmax, rel)


def test_bad_material_and_crop_are_errors(gpu):
    torch = gpu
    from qpop_diffraction_b200 import Plan
    shape, params, case = stack_case(23)
    with Plan(shape, (params.dx, params.dy, params.dz), 2) as plan:
        d = lambda a: to_dev(torch, a)
        mat = case["mat"].copy()
        mat[case["z0"] + 3, 5, 7] = 9                      # not in the 3-entry tables
        with pytest.raises(ValueError):
            plan.pack_fields(d(case["P"]), d(mat), case["dc"], case["phase_of"], case["ramp_dz"], z0=case["z0"])
        with pytest.raises(ValueError):                    # crop runs past the stack
            plan.pack_fields(d(case["P"]), d(case["mat"]), case["dc"], case["phase_of"], case["ramp_dz"],
                             z0=case["mat"].shape[0] - shape[2] + 1)
        with pytest.raises(ValueError):                    # phase index beyond nPhase
            plan.pack_fields(d(case["P"]), d(case["mat"]), case["dc"], np.array([0, -1, 2], dtype=np.int32),
                             case["ramp_dz"], z0=case["z0"])
        # a valid call still works on the same plan afterwards
        out = plan.pack_fields(d(case["P"]), d(case["mat"]), case["dc"], case["phase_of"], case["ramp_dz"], z0=case["z0"])
        assert out["P"].numel() == 3 * plan.n
