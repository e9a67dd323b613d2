"""
The hand-written adjoint (qpd_adjoint_device behind qpop_diffraction_b200.autograd.intensity)
against a float64 PyTorch complex128 autograd reference (tests/torch_reference.py) and against
central finite differences of the loss through the float64 forward.

Loss: L = sum_q (log10 I - log10 I_target)^2, I_target from an unperturbed field, evaluated at
P + N(0, 0.05), u + N(0, 0.001 nm).
Tolerances (max |g - g_ref| / max |g_ref| per gradient):
  float64 adjoint vs complex128 autograd: 1e-8;  float32 adjoint: 2e-3.
  Finite differences on 64 voxels (relative to the largest of them): float64 1e-5, float32 2e-3.
"""

import numpy as np
import pytest

import torch_reference as tref
from conftest import load_golden

pytestmark = pytest.mark.gpu


def problem(torch, shape, precision, seed, weights="dense", nPhase=2):
    """A Plan, the packed perturbed inputs as leaf tensors, the target intensity and the dense weights."""
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    case = workloads.random_case(shape, seed=seed, nPhase=nPhase, weights=weights, strain=True, hkl=(1, 0, 3))
    p = case.params
    plan = Plan(shape, (p.dx, p.dy, p.dz), p.nPhase, p.nStruc, precision=precision)
    crystal = crystal_from(p, case.atoms)
    plan.set_crystal(crystal)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(a).to(dev)
    target = plan.run_device(plan.pack(t(case.oPhase), t(case.oStruc), t(case.u), t(case.region))).clone()
    rng = np.random.default_rng(seed + 100)
    n = case.region.size
    oStruc = (case.oStruc + rng.normal(0, 0.05, case.oStruc.size)).astype(np.float32).astype(np.float64)
    u = (case.u + rng.normal(0, 0.001, case.u.size)).astype(np.float32).astype(np.float64)
    packed = plan.pack(t(case.oPhase), t(oStruc), t(u), t(case.region))
    W = (case.oPhase.reshape(p.nPhase, n) * case.region).reshape((p.nPhase,) + shape)
    return plan, crystal, packed, target, t(W), case


def grads_ours(torch, plan, packed, target):
    from qpop_diffraction_b200 import autograd
    shape4 = (3,) + plan.shape
    P = packed["P"].view(shape4).clone().requires_grad_(True)
    U = packed["U"].view(shape4).clone().requires_grad_(True)
    I = autograd.intensity(plan, P, U, phase=packed["phase"], weight=packed["weight"], wdense=packed["wdense"])
    L = tref.log_loss(I, target)
    L.backward()
    plan.device_status()
    return L.item(), P.grad.double(), U.grad.double()


def grads_torch(torch, plan, crystal, packed, target, W):
    shape4 = (3,) + plan.shape
    P = packed["P"].double().view(shape4).clone().requires_grad_(True)
    U = packed["U"].double().view(shape4).clone().requires_grad_(True)
    I = tref.intensity(P, U, W, crystal, plan.shape, plan.spacing)
    L = tref.log_loss(I, target)
    L.backward()
    return L.item(), P.grad, U.grad


def rel(a, b):
    return ((a - b).abs().max() / b.abs().max()).item()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32", 2e-3)])
@pytest.mark.parametrize("shape,weights,nPhase", [((24, 20, 16), "dense", 2), ((16, 12, 10), "onehot", 2),
                                                  ((20, 8, 13), "region", 1), ((12, 10, 104), "onehot", 2),
                                                  ((10, 12, 64), "region", 1)])
def test_adjoint_matches_complex128_autograd(gpu, precision, tol, shape, weights, nPhase):
    torch = gpu
    plan, crystal, packed, target, W, _ = problem(torch, shape, precision, seed=sum(shape), weights=weights,
                                                  nPhase=nPhase)
    with plan:
        L, gP, gU = grads_ours(torch, plan, packed, target)
        Lr, rP, rU = grads_torch(torch, plan, crystal, packed, target, W)
    assert abs(L - Lr) <= 1e-6 * abs(Lr) + (1e-12 if precision == "fp64" else 1e-3 * abs(Lr))
    assert rel(gP, rP) <= tol, rel(gP, rP)
    assert rel(gU, rU) <= tol, rel(gU, rU)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-5), ("fp32", 2e-3)])
def test_adjoint_matches_finite_differences(gpu, precision, tol):
    """Central differences of L through the float64 forward on 64 random voxels (P and u components)."""
    torch = gpu
    shape = (32, 24, 20)
    plan, crystal, packed, target, W, _ = problem(torch, shape, precision, seed=5)
    with plan:
        _, gP, gU = grads_ours(torch, plan, packed, target)
    fplan, _, fpacked, ftarget, _, _ = problem(torch, shape, "fp64", seed=5)
    rng = np.random.default_rng(9)
    n = plan.n
    picks = [(name, int(rng.integers(3)), int(rng.integers(n))) for name in ("P", "U") for _ in range(32)]
    fd, ad = [], []
    with fplan:
        for name, comp, cell in picks:
            h = 1e-4 if name == "P" else 1e-5
            vals = []
            for sgn in (1, -1):
                x = {k: (v.clone() if v is not None else None) for k, v in fpacked.items()}
                x[name][comp * n + cell] += sgn * h
                vals.append(tref.log_loss(fplan.run_device(x), ftarget).item())
            fd.append((vals[0] - vals[1]) / (2 * h))
            ad.append((gP if name == "P" else gU).reshape(-1)[comp * n + cell].item())
    fd, ad = np.array(fd), np.array(ad)
    err = np.abs(fd - ad).max() / np.abs(fd).max()
    assert err <= tol, err


def test_floor_passes_no_gradient(gpu):
    torch = gpu
    plan, crystal, packed, target, W, case = problem(torch, (8, 6, 5), "fp32", seed=1, weights="region", nPhase=1)
    packed["weight"] = torch.zeros_like(packed["phase"], dtype=plan.torch_dtype)   # nothing scatters
    with plan:
        from qpop_diffraction_b200 import autograd
        P = packed["P"].view((3,) + plan.shape).clone().requires_grad_(True)
        U = packed["U"].view((3,) + plan.shape).clone().requires_grad_(True)
        I = autograd.intensity(plan, P, U, phase=packed["phase"], weight=packed["weight"])
        assert torch.all(I == 1e-50)
        (I.sum()).backward()
        assert torch.count_nonzero(P.grad) == 0 and torch.count_nonzero(U.grad) == 0


def test_adjoint_needs_the_fused_schedule(gpu):
    torch = gpu
    from qpop_diffraction_b200 import Plan, crystal_from
    case, _ = load_golden("random_15x13x7_region")
    p = case.params
    with Plan(case.shape, (p.dx, p.dy, p.dz), p.nPhase, p.nStruc, precision="fp64", schedule="plain") as plan:
        plan.set_crystal(crystal_from(p, case.atoms))
        t = lambda a: torch.from_numpy(a).cuda()
        packed = plan.pack(t(case.oPhase), t(case.oStruc), t(case.u), t(case.region))
        with pytest.raises(ValueError):
            plan.adjoint(packed, torch.ones(plan.n, dtype=torch.float64, device="cuda"))


def config5(torch, precision, seed=5):
    """256 x 256 x 64 polar-vortex film, target from the unperturbed field, P + N(0, 0.05), u + N(0, 0.001 nm)."""
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    shape = (256, 256, 64)
    params, inputs = workloads.gpu_snapshot("vortex", shape, seed=seed, device="cuda:0")
    crystal = crystal_from(params, workloads.config2_crystal(2, (1, 0, 3)))
    plan = Plan(shape, (params.dx, params.dy, params.dz), params.nPhase, 3, precision=precision)
    plan.set_crystal(crystal)
    g = torch.Generator(device="cuda:0")
    g.manual_seed(seed + 1)
    dt = plan.torch_dtype
    base = {k: (v.to(dt) if v is not None and v.is_floating_point() else v) for k, v in inputs.items()}
    target = plan.run_device(base).clone()
    P = (inputs["P"].reshape(-1) + torch.randn(3 * plan.n, generator=g, device="cuda:0") * 0.05).float()
    U = (inputs["U"].reshape(-1) + torch.randn(3 * plan.n, generator=g, device="cuda:0") * 0.001).float()
    packed = dict(base, P=P.to(dt), U=U.to(dt))
    w = torch.ones(plan.n, dtype=torch.float64, device="cuda:0") if inputs["weight"] is None else inputs["weight"].double()
    W = torch.stack([(inputs["phase"].long() == p).double() * w for p in range(params.nPhase)]).view((params.nPhase,) + shape)
    return plan, crystal, packed, target, W


def test_config5_full_size_against_complex128_and_finite_differences(gpu):
    """The 256 x 256 x 64 differentiation workload: float32 adjoint vs complex128 autograd and 64-voxel FD."""
    torch = gpu
    plan, crystal, packed, target, W = config5(torch, "fp32")
    with plan:
        _, gP, gU = grads_ours(torch, plan, packed, target)
        _, rP, rU = grads_torch(torch, plan, crystal, packed, target, W)
    assert rel(gP, rP) <= 2e-3, rel(gP, rP)
    assert rel(gU, rU) <= 2e-3, rel(gU, rU)
    del rP, rU
    torch.cuda.empty_cache()
    fplan, _, fpacked, _, _ = config5(torch, "fp64")
    ftarget = target                        # the same loss: only the forward's precision differs
    rng = np.random.default_rng(64)
    n = fplan.n
    fd, ad = [], []
    with fplan:
        for name in ("P", "U"):
            for _ in range(32):
                comp, cell = int(rng.integers(3)), int(rng.integers(n))
                h = 1e-4 if name == "P" else 1e-5
                vals = []
                for sgn in (1, -1):
                    x = dict(fpacked)
                    x[name] = fpacked[name].clone()
                    x[name][comp * n + cell] += sgn * h
                    vals.append(tref.log_loss(fplan.run_device(x), ftarget).item())
                fd.append((vals[0] - vals[1]) / (2 * h))
                ad.append((gP if name == "P" else gU).reshape(-1)[comp * n + cell].item())
    fd, ad = np.array(fd), np.array(ad)
    assert np.abs(fd - ad).max() / np.abs(fd).max() <= 2e-3
