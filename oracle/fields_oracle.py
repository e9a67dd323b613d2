"""
CPU oracle for the boundary-input preparation.  TEST INFRASTRUCTURE ONLY.

Restates, in NumPy float64, how the reference turns Q-POP-FerroDyn fields into the arguments of
``diffraction(params, atoms, oPhase, oStruc, u, region)``:

- the cropped (nz, ny, nx) datasets are read and transposed to (x, y, z) order, float64
  (src/python/io_utils.py:30-40, 54-92); P is divided by OS0 = 1 (src/python/cli.py:176) and the
  displacement scaled from metres to nm (src/python/io_utils.py:71; u_scale of the native
  program, src/heffte/params.hpp:20);
- the phases are one-hot over the FE materials of the cropped material field and the region
  weight is their sum times the optional region file; an optional phase file replaces the
  one-hot phases (src/python/cli.py:187-200);
- the u_z reference ramp (cumsum_z dc[mat] - dc[mat] / 2) dz is summed over the FULL material
  stack and then cropped (src/python/cli.py:207-217; the native twin is the `columns` kernel,
  src/heffte/kernels.cuh:34-50, which also sets phase = phaseOf[mat]).

Only ``tests/`` may import this module.
"""

from __future__ import annotations

import numpy as np


def to_xyz(a):
    """(nz, ny, nx) file order -> (x, y, z) float64."""
    return np.asarray(a).astype(np.float64).transpose(2, 1, 0)


def prepare(P, mat, dc, phase_of, ramp_dz, z0=0, u=None, phase=None, region=None, p_scale=1.0, u_scale=1.0):
    """
    Arguments of diffraction() from FerroDyn-layout fields.

    P: (nStruc, nz, ny, nx); u: (3, nz, ny, nx) in metres, or None; phase: (nPhase, nz, ny, nx)
    phase fractions or None; region: (nz, ny, nx) or None -- all already cropped.  mat:
    (nz_full, ny, nx) material indices of the full stack over the crop's columns; z0 the crop's
    first layer in it.  dc[m] = c_m / aC_z - 1 and phase_of[m] (phase index, -1 for a material
    that does not scatter) per material.  Returns (oPhase, oStruc, u, region), flat float64 in
    component-major (x, y, z) C order.
    """
    nStruc = P.shape[0]
    nz, ny, nx = P.shape[1:]
    n = nx * ny * nz
    mat_xyz = np.asarray(mat).astype(np.int64).transpose(2, 1, 0)          # (nx, ny, nz_full)
    phase_of = np.asarray(phase_of, dtype=np.int64)
    dcm = np.asarray(dc, dtype=np.float64)[mat_xyz]
    ramp = ((np.cumsum(dcm, axis=2) - 0.5 * dcm) * ramp_dz)[:, :, z0:z0 + nz]
    m = mat_xyz[:, :, z0:z0 + nz]
    nPhase = int(phase_of.max()) + 1 if phase is None else phase.shape[0]
    onehot = np.stack([phase_of[m] == p for p in range(nPhase)]).astype(np.float64)
    reg = (phase_of[m] >= 0).astype(np.float64).ravel()
    if phase is not None:
        onehot = np.stack([to_xyz(f) for f in phase])
    if region is not None:
        reg = reg * to_xyz(region).ravel()
    oStruc = np.stack([to_xyz(c) * p_scale for c in P]).ravel()
    uu = np.zeros((3, n)) if u is None else np.stack([to_xyz(c) * u_scale for c in u]).reshape(3, n)
    uu[2] += ramp.ravel()
    assert oStruc.size == nStruc * n
    return onehot.ravel(), oStruc, uu.ravel(), reg
