"""
CPU oracle for the kinematic-diffraction hot path.  TEST INFRASTRUCTURE ONLY.

This module restates, in NumPy float64, the reference's standard-build compute
call ``diffraction(params, atoms, oPhase, oStruc, u, region)``
(src/python/diffraction.py:62-113).  It is the checker for the CUDA path and the
timed CPU baseline; the product (the ``qpop_diffraction_b200`` package and its
CUDA library) never imports, links or runs it.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / ``--impl reference``
legs may use it.

Pinning: the golden fixtures under ``tests/golden/`` were produced by running the
reference's own ``diffraction()`` on the same seeded inputs
(``tests/golden/make_golden.py``); ``tests/test_oracle.py`` checks this module
against them, and against the reference's analytic known answers
(tests/test_single_domain.py:51-78, tests/test_a1a2_domains.py:50-80,
tests/test_planted.py:141-219 of the reference).

The model, as the reference computes it (docs/method.md:11-26):

    u_ap(r) = u(r) + su[:, :, p, a] . P(r)
    fE_a(r) = sum_p w_p(r) f_pa exp(-i qC . u_ap(r))
    fU_a(r) = sum_p w_p(r) f_pa exp(-i qC . u_ap(r)) u_ap(r)
    Amp(k)  = sum_a exp(-i (k + G) . R_a) / V [FFT(fE_a)/n - i k . FFT(fU_a)/n]
    I       = fftshift(max(|S(k) Amp(k)|^2, 1e-50)),  S(k) = prod_d sinc(k_d h_d / 2)
"""

from __future__ import annotations

import math
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np


def strain_tensor(strain_avg):
    """Voigt (xx, yy, zz, yz, xz, xy) -> symmetric 3x3, as src/python/diffraction.py:44-45 orders it."""
    e = np.asarray(strain_avg, dtype=np.float64)
    return np.array([[e[0], e[5], e[4]],
                     [e[5], e[1], e[3]],
                     [e[4], e[3], e[2]]])


def reciprocal_centre(aC, q00, strain_avg):
    """G nearest q00 and qC = G - eps G in nm^-1 (src/python/diffraction.py:36-48)."""
    aC = np.asarray(aC, dtype=np.float64)
    hkl = np.round(aC @ np.asarray(q00, dtype=np.float64) / (2 * math.pi))
    G = hkl @ (2 * math.pi * np.linalg.inv(aC).T)
    return G, G - strain_tensor(strain_avg) @ G


def wavevectors(shape, spacing):
    """2 pi fftfreq per axis, FFT order (src/python/diffraction.py:51-54)."""
    return [2 * math.pi * np.fft.fftfreq(m, d) for m, d in zip(shape, spacing)]


def q_axes(shape, spacing, qC):
    """fftshifted 1-D q axes (src/python/diffraction.py:57-59)."""
    return tuple(np.fft.fftshift(kd) + qC[d] for d, kd in enumerate(wavevectors(shape, spacing)))


def _broadcast(kd, axis):
    return kd.reshape([-1 if i == axis else 1 for i in range(3)])


def _atom_amplitude(a, shape, k, G, qC, V, R, fAtom, su, w, P, U):
    """One atom's term of the amplitude sum (src/python/diffraction.py:97-109)."""
    n = int(np.prod(shape))
    nPhase = w.shape[0]
    fE = np.zeros(n, dtype=np.complex128)
    fU = np.zeros((3, n), dtype=np.complex128)
    for p in range(nPhase):
        ua = U + su[:, :, p, a] @ P
        e = fAtom[p, a] * w[p] * np.exp(-1j * (qC @ ua))
        fE += e
        fU += e * ua
    FE = np.fft.fftn(fE.reshape(shape)) / n
    FU = np.fft.fftn(fU.reshape(3, *shape), axes=(1, 2, 3)) / n
    kx, ky, kz = (_broadcast(k[d], d) for d in range(3))
    shift = np.exp(-1j * (kx + G[0]) * R[a, 0]) * np.exp(-1j * (ky + G[1]) * R[a, 1]) \
        * np.exp(-1j * (kz + G[2]) * R[a, 2]) / V
    return shift * (FE - 1j * (kx * FU[0] + ky * FU[1] + kz * FU[2]))


def intensity(shape, spacing, G, qC, V, R, fAtom, su, weights, P, U, threads=1):
    """
    The fftshifted intensity (nx, ny, nz), float64.

    Args:
        shape:   (nx, ny, nz)
        spacing: (dx, dy, dz) in nm
        G, qC:   reciprocal lattice point and its strain-corrected centre, nm^-1
        V:       unit-cell volume, nm^3
        R:       (nAtom, 3) atom positions in nm
        fAtom:   (nPhase, nAtom) complex form factors
        su:      (3, nStruc, nPhase, nAtom) ionic shifts, nm per C/m^2
        weights: (nPhase, n) phase fraction x region weight
        P:       (nStruc, n) order parameter, C/m^2
        U:       (3, n) displacement, nm
        threads: atoms evaluated concurrently (NumPy releases the GIL in its
                 ufunc loops and FFTs); 1 reproduces the reference's serial loop.
    """
    shape = tuple(int(s) for s in shape)
    k = wavevectors(shape, spacing)
    nAtom = R.shape[0]
    args = (shape, k, np.asarray(G), np.asarray(qC), V, R, fAtom, su, weights, P, U)
    amp = np.zeros(shape, dtype=np.complex128)
    if threads <= 1:
        for a in range(nAtom):
            amp += _atom_amplitude(a, *args)
    else:
        with ThreadPoolExecutor(max_workers=threads) as pool:
            for part in pool.map(lambda a: _atom_amplitude(a, *args), range(nAtom)):
                amp += part
    S = np.ones(shape)
    for d, h in enumerate(spacing):
        S = S * np.sinc(_broadcast(k[d], d) * h / (2 * math.pi))
    return np.fft.fftshift(np.maximum(np.abs(S * amp) ** 2, 1e-50))


def diffraction(params, atoms, oPhase, oStruc, u, region, threads=1):
    """
    Same call as the reference's standard build (src/python/diffraction.py:62-113):
    ``params`` needs nx, ny, nz, n, dx, dy, dz, nPhase, nStruc, strainAvg; ``atoms``
    needs aC, q00, xAtom, fAtom, su1, su2, su3, nAtom.  Returns (I, qx, qy, qz).
    """
    shape = (params.nx, params.ny, params.nz)
    spacing = (params.dx, params.dy, params.dz)
    n = params.n
    G, qC = reciprocal_centre(atoms.aC, atoms.q00, params.strainAvg)
    V = np.linalg.det(atoms.aC)
    R = atoms.xAtom @ atoms.aC
    su = np.stack([atoms.su1, atoms.su2, atoms.su3])
    weights = oPhase.reshape(params.nPhase, n) * region
    P = oStruc.reshape(params.nStruc, n)
    U = u.reshape(3, n)
    I = intensity(shape, spacing, G, qC, V, R, atoms.fAtom, su, weights, P, U, threads=threads)
    return (I,) + q_axes(shape, spacing, qC)


def default_threads(nAtom):
    """Host threads the threaded oracle can use: one per atom, at most the cores present."""
    return max(1, min(int(nAtom), os.cpu_count() or 1))
