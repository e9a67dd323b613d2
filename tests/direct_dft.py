"""
Direct-sum intensities at chosen voxels, in float64 torch: the independent check of the 3-D FFT path
at sizes the NumPy oracle cannot hold (4000 x 4000 x 68 needs about 425 GB there).  TEST
INFRASTRUCTURE ONLY.

The amplitude at one voxel k (FFT-order indices (i, j, l)) is the model of
oracle/diffraction_oracle.py (src/python/diffraction.py:97-112) written as a sum over cells instead
of an FFT:

    Amp(k) = sum_a exp(-i (k + G) . R_a) / (V n) sum_r e(k, r) [fE_a(r) - i k . fU_a(r)],
    e(k, r) = exp(-2 pi i (i x / nx + j y / ny + l z / nz)),

with fE_a, fU_a the per-cell sources of the packed inputs (float32 P and u promoted to float64, the
int8 phase index and optional weight).  The sum over r is separable: for each x slab a batched
product with the (voxel, y) factors, then the z and x factors.  Nothing is shared with the CUDA
kernels: no FFT, no folding, no tables.
"""

from __future__ import annotations

import math

import numpy as np


def fft_index_to_shifted(N):
    """pos[i]: where FFT index i lands in the fftshifted axis of length N."""
    return np.argsort(np.fft.fftshift(np.arange(N)))


def shifted_to_fft_index(N):
    """idx[m]: the FFT index at fftshifted position m."""
    return np.fft.fftshift(np.arange(N))


def direct_intensity(torch, shape, spacing, G, qC, V, R, fAtom, su, P, U, phase, weight, vox, slab=16):
    """
    Float64 intensities max(|S Amp|^2, 1e-50) at voxels `vox` ((nv, 3) FFT-order indices).

    P, U: flat (3 n) tensors in any float type; phase: (n,) int8 (-1: the cell does not scatter);
    weight: (n,) or None (1); su: (3, nStruc, nPhase, nAtom); fAtom: (nPhase, nAtom).
    """
    nx, ny, nz = (int(s) for s in shape)
    n = nx * ny * nz
    dev = P.device
    vox = np.asarray(vox, dtype=np.int64).reshape(-1, 3)
    nv = vox.shape[0]
    k = [2 * math.pi * np.fft.fftfreq(m, d) for m, d in zip(shape, spacing)]
    kv = np.stack([k[d][vox[:, d]] for d in range(3)], axis=1)                     # (nv, 3)

    def factors(N, idx):                                                            # (nv, N)
        return torch.from_numpy(np.exp(-2j * math.pi * np.outer(idx, np.arange(N)) / N)).to(dev)

    ex, ey, ez = factors(nx, vox[:, 0]), factors(ny, vox[:, 1]), factors(nz, vox[:, 2])
    R = np.asarray(R, dtype=np.float64)
    G = np.asarray(G, dtype=np.float64)
    shift = np.exp(-1j * ((kv + G) @ R.T)) / (V * n)                                # (nv, nAtom)
    cE = torch.from_numpy(shift).to(dev)
    cU = [torch.from_numpy(-1j * kv[:, d:d + 1] * shift).to(dev) for d in range(3)]
    nPhase, nAtom = fAtom.shape
    nStruc = su.shape[1]
    qCt = torch.tensor(np.asarray(qC, dtype=np.float64), device=dev)
    P3 = P.view(3, nx, ny, nz)
    U3 = U.view(3, nx, ny, nz)
    ph = phase.view(nx, ny, nz)
    W3 = None if weight is None else weight.view(nx, ny, nz)
    amp = torch.zeros((nv, nAtom), dtype=torch.complex128, device=dev)
    for x0 in range(0, nx, slab):
        x1 = min(nx, x0 + slab)
        p = P3[:nStruc, x0:x1].double()
        u = U3[:, x0:x1].double()
        phs = ph[x0:x1].long()
        w = torch.ones_like(u[0]) if W3 is None else W3[x0:x1].double()
        exs = ex[:, x0:x1]
        for pi in range(nPhase):
            wp = torch.where(phs == pi, w, torch.zeros_like(w))
            if not bool((wp != 0).any()):
                continue
            for a in range(nAtom):
                sa = torch.from_numpy(np.ascontiguousarray(su[:, :, pi, a])).to(dev)      # (3, nStruc)
                ua = u + torch.einsum("dk,kxyz->dxyz", sa, p)
                e = wp * torch.exp(-1j * torch.einsum("d,dxyz->xyz", qCt, ua)) * complex(fAtom[pi, a])
                for F, cf in ((e, cE[:, a]), (e * ua[0], cU[0][:, a]), (e * ua[1], cU[1][:, a]),
                              (e * ua[2], cU[2][:, a])):
                    T = torch.einsum("vy,xyz->vxz", ey, F)                          # sum over y
                    amp[:, a] += cf * torch.einsum("vxz,vx,vz->v", T, exs, ez)     # then z and x
    S = np.ones(nv)
    for d, h in enumerate(spacing):
        S = S * np.sinc(kv[:, d] * h / (2 * math.pi))
    A = amp.sum(dim=1).cpu().numpy()
    return np.maximum(np.abs(S * A) ** 2, 1e-50)


def crystal_constants(params, atoms):
    """(G, qC, V, R, fAtom, su) of the reference's diffraction() for these params and atoms."""
    from oracle import diffraction_oracle as oracle
    G, qC = oracle.reciprocal_centre(atoms.aC, atoms.q00, params.strainAvg)
    V = float(np.linalg.det(atoms.aC))
    R = atoms.xAtom @ atoms.aC
    su = np.stack([atoms.su1, atoms.su2, atoms.su3])
    return G, qC, V, R, np.asarray(atoms.fAtom), su
