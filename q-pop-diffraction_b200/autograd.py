"""
Differentiation through the hot path: ``intensity(plan, P, U, ...)`` returns I as a torch tensor
whose gradient flows to the order parameter P and the displacement U.

The backward pass is the library's hand-written adjoint (qpd_adjoint_device): it recomputes the
forward transforms pass by pass instead of keeping intermediates, seeds dL/dconj(Amp) in the last
forward pass, runs the transposed x and y passes and finishes with the z transform fused with the
transpose of the source kernel.  The reference has no gradient; the model differentiated is its
diffraction() (src/python/diffraction.py:62-113).
"""

from __future__ import annotations

import torch


class _Intensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P, U, plan, phase, weight, wdense):
        inputs = {"P": P.detach().reshape(-1).contiguous(), "U": U.detach().reshape(-1).contiguous(),
                  "phase": phase, "weight": weight, "wdense": wdense}
        I = plan.run_device(inputs)
        ctx.plan, ctx.inputs, ctx.shapes = plan, inputs, (P.shape, U.shape)
        return I

    @staticmethod
    def backward(ctx, grad_I):
        dP, dU = ctx.plan.adjoint(ctx.inputs, grad_I.to(torch.float64))
        return dP.view(ctx.shapes[0]), dU.view(ctx.shapes[1]), None, None, None, None


def intensity(plan, P, U, phase=None, weight=None, wdense=None):
    """
    I (nx, ny, nz) float64, fftshifted, for the packed inputs of a Plan: P and U (3, nx, ny, nz) in
    the plan precision (``plan.torch_dtype``) on its device, and either the phase index with an
    optional weight (single-phase cells) or dense weights (nPhase, nx, ny, nz).  Differentiable with
    respect to P and U.
    """
    for name, t in (("P", P), ("U", U)):
        if t.dtype != plan.torch_dtype or t.numel() != 3 * plan.n or not t.is_cuda:
            raise ValueError(f"{name}: expected 3 x {plan.shape} {plan.torch_dtype} values on the GPU")
    if (phase is None) == (wdense is None):
        raise ValueError("give either phase (with an optional weight) or wdense")
    flat = lambda t: None if t is None else t.reshape(-1).contiguous()
    return _Intensity.apply(P, U, plan, flat(phase), flat(weight), flat(wdense))
