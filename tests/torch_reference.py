"""
The diffraction model in plain PyTorch complex128, differentiable by autograd: the float64
reference gradient for the adjoint kernels.  TEST INFRASTRUCTURE ONLY.

It restates src/python/diffraction.py:62-113 (as the oracle does in NumPy) on torch tensors:
u_ap = u + su[:, :, p, a] . P;  fE = sum_p w_p f_pa exp(-i qC . u_ap);  fU = fE-weighted u_ap;
Amp = sum_a exp(-i (k + G) . R_a) / V [fftn(fE)/n - i k . fftn(fU)/n];
I = fftshift(max(|S Amp|^2, 1e-50)).
"""

import math

import numpy as np
import torch


def intensity(P, U, W, crystal, shape, spacing):
    """P, U: (3, nx, ny, nz) float64; W: (nPhase, nx, ny, nz) float64 weights; returns I (nx, ny, nz)."""
    dev = P.device
    n = int(np.prod(shape))
    k = [torch.as_tensor(2 * math.pi * np.fft.fftfreq(m, h), dtype=torch.float64, device=dev)
         for m, h in zip(shape, spacing)]
    kb = [k[0].view(-1, 1, 1), k[1].view(1, -1, 1), k[2].view(1, 1, -1)]
    qC = torch.as_tensor(crystal.qC, dtype=torch.float64, device=dev)
    su = torch.as_tensor(crystal.su, dtype=torch.float64, device=dev)
    f = torch.as_tensor(crystal.fAtom, dtype=torch.complex128, device=dev)
    R = crystal.R
    nS = su.shape[1]
    amp = torch.zeros(shape, dtype=torch.complex128, device=dev)
    for a in range(R.shape[0]):
        fE = torch.zeros(shape, dtype=torch.complex128, device=dev)
        fU = [torch.zeros(shape, dtype=torch.complex128, device=dev) for _ in range(3)]
        for p in range(W.shape[0]):
            ua = [U[d] + sum(su[d, s, p, a] * P[s] for s in range(nS)) for d in range(3)]
            theta = qC[0] * ua[0] + qC[1] * ua[1] + qC[2] * ua[2]
            e = W[p] * f[p, a] * torch.exp(-1j * theta)
            fE = fE + e
            fU = [fU[d] + e * ua[d] for d in range(3)]
        FE = torch.fft.fftn(fE) / n
        FU = [torch.fft.fftn(x) / n for x in fU]
        ph = torch.exp(-1j * ((kb[0] + crystal.G[0]) * R[a, 0] + (kb[1] + crystal.G[1]) * R[a, 1]
                              + (kb[2] + crystal.G[2]) * R[a, 2])) / crystal.V
        amp = amp + ph * (FE - 1j * (kb[0] * FU[0] + kb[1] * FU[1] + kb[2] * FU[2]))
    S = 1.0
    for d, h in enumerate(spacing):
        S = S * torch.sinc(kb[d] * h / (2 * math.pi))
    I = torch.clamp((S * amp).abs() ** 2, min=1e-50)
    return torch.fft.fftshift(I)


def log_loss(I, I_target):
    """sum_q (log10 I - log10 I_target)^2."""
    return ((torch.log10(I) - torch.log10(I_target)) ** 2).sum()
