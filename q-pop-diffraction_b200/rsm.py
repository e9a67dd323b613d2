"""
Reciprocal-space maps of an intensity volume, projected on the GPU.

The reference (src/python/rsm.py:22-178) bins all n voxels with ``numpy.histogram2d`` over each
pair of broadcast q components (qx-qy, qx-qz, qy-qz), summing or averaging I per bin.  The q grid
is the tensor product of three 1-D axes, so a voxel's bin in the (a, b) map depends only on its
index along a and along b: each map is the projection of I over the third axis (qpd_rsm_project,
on the GPU, over the resident volume) re-binned along the two 1-D axes (here, on maps of nx*ny
values at most).  Bin edges and centres follow src/python/rsm.py:69-85; the bin of a value follows
numpy.histogram (half-open bins, the last edge inclusive, values outside dropped).

    python -m qpop_diffraction_b200.rsm -d diffraction.h5 [-o reciprocal_space_maps] [--bins N]
                                        [--aggregation sum|mean]

writes ``qx_qy.npz``, ``qx_qz.npz`` and ``qy_qz.npz`` with the reference's keys (q_a, q_b,
q_units, intensity, log10_intensity; src/python/rsm.py:107-117).  The reference's PNG figures need
matplotlib, which this package does not use: plot the npz files.
"""

from __future__ import annotations

import argparse
import ctypes
import sys
from pathlib import Path

import numpy as np

from . import _native as nat
from . import hdf5

PAIRS = ((0, 1, "qx_qy"), (0, 2, "qx_qz"), (1, 2, "qy_qz"))


def build_edges(values, n_bins=None):
    """(edges, centres) of one map axis (src/python/rsm.py:69-85)."""
    values = np.asarray(values, dtype=np.float64)
    if n_bins is not None:
        edges = np.linspace(values.min(), values.max(), n_bins + 1)
        return edges, 0.5 * (edges[:-1] + edges[1:])
    centres = np.unique(np.round(values, decimals=10))
    if centres.size == 1:
        return np.array([centres[0] - 0.5, centres[0] + 0.5]), centres.copy()
    first = centres[0] - 0.5 * (centres[1] - centres[0])
    last = centres[-1] + 0.5 * (centres[-1] - centres[-2])
    return np.concatenate(([first], 0.5 * (centres[:-1] + centres[1:]), [last])), centres


def bin_index(values, edges):
    """Bin of each value as numpy.histogram assigns it: [e_i, e_i+1), the last bin closed; -1 outside."""
    values = np.asarray(values, dtype=np.float64)
    nb = edges.size - 1
    idx = np.searchsorted(edges, values, side="right") - 1
    idx[values == edges[-1]] = nb - 1
    idx[(values < edges[0]) | (values > edges[-1])] = -1
    return idx


def _rebin(proj, ia, ib, na, nb):
    out = np.zeros((na, nb))
    ok_a, ok_b = ia >= 0, ib >= 0
    sub = proj[np.ix_(ok_a, ok_b)]
    np.add.at(out, (ia[ok_a][:, None], ib[ok_b][None, :]), sub)
    return out


def projections(I, stream=None):
    """The three projections (xy, xz, yz) of a float64 (nx, ny, nz) CUDA tensor, on the GPU."""
    import torch
    if not isinstance(I, torch.Tensor) or not I.is_cuda or I.dtype != torch.float64 or I.dim() != 3:
        raise ValueError("I must be a float64 (nx, ny, nz) CUDA tensor")
    I = I.contiguous()
    nx, ny, nz = I.shape
    kw = dict(dtype=torch.float64, device=I.device)
    xy, xz, yz = torch.empty((nx, ny), **kw), torch.empty((nx, nz), **kw), torch.empty((ny, nz), **kw)
    lib = nat.load()
    st = stream if stream is not None else torch.cuda.current_stream(I.device).cuda_stream
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    nat.check(lib, None, lib.qpd_rsm_project(p(I), nx, ny, nz, p(xy), p(xz), p(yz), ctypes.c_void_p(st)))
    return xy, xz, yz


def maps(I, qx, qy, qz, bins=None, aggregation="sum", stream=None):
    """
    The three reciprocal-space maps of intensity I: ``{stem: (centres_a, centres_b, map)}`` with
    stem in qx_qy, qx_qz, qy_qz (src/python/rsm.py:88-104, 150-156).  I is a float64 (nx, ny, nz)
    CUDA tensor (a NumPy array is copied to the current device first).
    """
    import torch
    if aggregation not in ("sum", "mean"):
        raise ValueError("aggregation must be 'sum' or 'mean'")
    if isinstance(I, np.ndarray):
        I = torch.from_numpy(np.ascontiguousarray(I, dtype=np.float64)).cuda()
    axes = [np.asarray(q, dtype=np.float64) for q in (qx, qy, qz)]
    if tuple(I.shape) != tuple(a.size for a in axes):
        raise ValueError(f"I has shape {tuple(I.shape)}, the q axes {tuple(a.size for a in axes)}")
    proj = projections(I, stream)
    if stream is not None:      # the copies below run on the current stream
        torch.cuda.synchronize(I.device)
    return maps_from_projections([t.cpu().numpy() for t in proj], *axes, bins=bins, aggregation=aggregation)


def maps_from_projections(proj, qx, qy, qz, bins=None, aggregation="sum"):
    """The maps from the projections (xy, xz, yz) of I: the re-binning along the 1-D q axes."""
    axes = [np.asarray(q, dtype=np.float64) for q in (qx, qy, qz)]
    grid = [build_edges(a, bins) for a in axes]
    index = [bin_index(a, e) for a, (e, _) in zip(axes, grid)]
    out = {}
    for (a, b, stem), pr in zip(PAIRS, proj):
        na, nb = grid[a][0].size - 1, grid[b][0].size - 1
        total = _rebin(pr, index[a], index[b], na, nb)
        if aggregation == "mean":
            third = axes[3 - a - b].size
            ca = np.bincount(index[a][index[a] >= 0], minlength=na).astype(np.float64)
            cb = np.bincount(index[b][index[b] >= 0], minlength=nb).astype(np.float64)
            counts = np.outer(ca, cb) * third
            total = np.divide(total, counts, out=np.zeros_like(total), where=counts > 0)
        out[stem] = (grid[a][1], grid[b][1], total)
    return out


def save_map_data(path, q_a, q_b, data):
    """The reference's npz layout (src/python/rsm.py:107-117)."""
    np.savez(path, q_a=q_a, q_b=q_b, q_units="nm^-1", intensity=data,
             log10_intensity=np.log10(np.maximum(data, np.finfo(np.float64).tiny)))


def main(argv=None):
    ap = argparse.ArgumentParser(description="Reciprocal-space maps of a Q-POP-Diffraction output file (GPU).")
    ap.add_argument("--diffraction", "-d", type=Path, required=True, metavar="HDF5")
    ap.add_argument("--output-dir", "-o", type=Path, default=Path("reciprocal_space_maps"))
    ap.add_argument("--bins", type=int, default=None)
    ap.add_argument("--aggregation", choices=("sum", "mean"), default="sum")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    import torch
    I, qx, qy, qz, _ = hdf5.load_diffraction_output(args.diffraction)
    args.output_dir.mkdir(parents=True, exist_ok=True)
    dev = torch.device("cuda", args.device)
    result = maps(torch.from_numpy(np.ascontiguousarray(I)).to(dev), qx, qy, qz, args.bins, args.aggregation)
    for stem, (ca, cb, data) in result.items():
        save_map_data(args.output_dir / f"{stem}.npz", ca, cb, data)
        print(f"Wrote {stem}.npz with shape {data.shape} to {args.output_dir}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
