"""
CPU oracle for the reciprocal-space maps.  TEST INFRASTRUCTURE ONLY.

Restates the reference's per-voxel binning (src/python/rsm.py:69-104, 150-156): the q vector of
every voxel is broadcast from the three 1-D axes (src/python/io_utils.py:201-206) and each pair of
components is binned with numpy.histogram2d, weighted by I, summed or averaged per bin.  Only
``tests/`` may import this module.
"""

from __future__ import annotations

import numpy as np


def edges(values, n_bins=None):
    if n_bins is not None:
        e = np.linspace(values.min(), values.max(), n_bins + 1)
        return e, 0.5 * (e[:-1] + e[1:])
    u = np.unique(np.round(values, decimals=10))
    if u.size == 1:
        return np.array([u[0] - 0.5, u[0] + 0.5]), u.copy()
    mid = 0.5 * (u[:-1] + u[1:])
    return np.concatenate(([u[0] - 0.5 * (u[1] - u[0])], mid, [u[-1] + 0.5 * (u[-1] - u[-2])])), u


def maps(I, qx, qy, qz, bins=None, aggregation="sum"):
    shape = I.shape
    q = [np.broadcast_to(np.asarray(a).reshape([-1 if d == i else 1 for i in range(3)]), shape).reshape(-1)
         for d, a in enumerate((qx, qy, qz))]
    w = I.reshape(-1)
    out = {}
    for a, b, stem in ((0, 1, "qx_qy"), (0, 2, "qx_qz"), (1, 2, "qy_qz")):
        ea, ca = edges(q[a], bins)
        eb, cb = edges(q[b], bins)
        s, _, _ = np.histogram2d(q[a], q[b], bins=(ea, eb), weights=w)
        if aggregation == "mean":
            c, _, _ = np.histogram2d(q[a], q[b], bins=(ea, eb))
            s = np.divide(s, c, out=np.zeros_like(s), where=c > 0)
        out[stem] = (ca, cb, s)
    return out
