"""
Single-GPU consumer of the reference's multi-GPU parameter file, a drop-in for the
``qpop_diffraction_mgpu <out>_params.h5`` program (src/heffte/qpop_diffraction_mgpu.cu:37-200).

``qpop-diffraction --mgpu`` (src/python/cli.py:106-146) writes ``<out>_params.h5``
(src/python/io_utils.py:144-183, read by src/heffte/params.hpp:66-108) and the output skeleton
``<out>.h5`` with the q axes (src/python/io_utils.py:106-141).  This runner reads the same file,
loads the cropped FerroDyn fields it names (hyperslabs of src/heffte/hdf5_io.hpp:33-62), prepares
them on the GPU (qpd_pack_fields: scale, one-hot phases, region, u_z ramp), runs the hot path on
one B200 and writes ``/intensity`` (nz, ny, nx) with the q axes and attributes into ``<out>.h5``
(src/heffte/hdf5_io.hpp:64-97).  One GPU holds what the reference spreads over several ranks.

    python -m qpop_diffraction_b200.params_runner <out>_params.h5 [--precision fp32|fp64] [--device 0]
"""

from __future__ import annotations

import argparse
import math
import os
import sys
import time
from pathlib import Path
from types import SimpleNamespace

import numpy as np

from . import hdf5
from .plan import Crystal, Plan


def read_params(path):
    """The content of <out>_params.h5, as mgpuParams::read takes it (src/heffte/params.hpp:66-108)."""
    d = lambda name: hdf5.read_dataset(path, name)
    attrs = hdf5.read_attrs(path)
    su = np.asarray(d("su"), dtype=np.float64)
    prm = SimpleNamespace(
        full=tuple(int(v) for v in d("grid")), crop=tuple(int(v) for v in d("crop")),
        spacing=tuple(float(v) for v in d("spacing")), G=np.asarray(d("G"), dtype=np.float64),
        qC=np.asarray(d("qC"), dtype=np.float64), V=float(d("V")[0]), u_scale=float(d("u_scale")[0]),
        R=np.asarray(d("R"), dtype=np.float64),
        fAtom=np.asarray(d("fAtom_re"), dtype=np.float64) + 1j * np.asarray(d("fAtom_im"), dtype=np.float64),
        su=su, phase_of=np.asarray(d("phase_of"), dtype=np.int32), dc=np.asarray(d("dc"), dtype=np.float64),
        **{k: (attrs[k] if attrs.get(k) else None) for k in ("platt_file", "platt_prefix", "displacement_file",
                                                            "material_file", "phase_file", "region_file",
                                                            "output_file")})
    if su.ndim != 4 or su.shape[0] != 3 or su.shape[1] != 3:
        raise ValueError(f"{path}: expects nStruc = 3 (P_x, P_y, P_z), su has shape {su.shape}")
    prm.nAtom, prm.nPhase = prm.R.shape[0], prm.fAtom.shape[0]
    prm.shape = tuple(prm.crop[2 * d + 1] - prm.crop[2 * d] + 1 for d in range(3))
    for d in range(3):
        if not 0 <= prm.crop[2 * d] <= prm.crop[2 * d + 1] < prm.full[d]:
            raise ValueError(f"{path}: crop {prm.crop} outside the grid {prm.full}")
    if not prm.platt_file or not prm.material_file or not prm.output_file:
        raise ValueError(f"{path}: platt_file, material_file and output_file are required")
    return prm


def _float32(path, name, full):
    """A (nz, ny, nx) FerroDyn dataset, float32 as FerroDyn writes it (src/python/io_utils.py:30-40)."""
    a = hdf5.read_dataset(path, name)
    if a.shape != full[::-1]:
        raise ValueError(f"{path}:/{name} has shape {a.shape}, expected (nz, ny, nx) = {full[::-1]}")
    if a.dtype != np.float32:
        raise ValueError(f"{path}:/{name} is {a.dtype}; FerroDyn fields are float32")
    return a


def load_fields(prm):
    """Cropped float32 fields in file order and the material stack over the crop's columns."""
    x0, x1, y0, y1, z0, z1 = prm.crop
    cut = (slice(z0, z1 + 1), slice(y0, y1 + 1), slice(x0, x1 + 1))
    crop = lambda a: np.ascontiguousarray(a[cut])
    prefix = prm.platt_prefix or "P_Lattice"
    P = np.stack([crop(_float32(prm.platt_file, f"{prefix}_{c}", prm.full)) for c in "xyz"])
    u = None
    if prm.displacement_file:
        u = np.stack([crop(_float32(prm.displacement_file, f"Displacement_{c}", prm.full)) for c in "xyz"])
    phase = None
    if prm.phase_file:
        phase = np.stack([crop(_float32(prm.phase_file, f"phase_{p + 1}", prm.full)) for p in range(prm.nPhase)])
    region = crop(_float32(prm.region_file, "region", prm.full)) if prm.region_file else None
    mat = hdf5.read_dataset(prm.material_file, "materialField")
    if mat.shape != prm.full[::-1]:
        raise ValueError(f"{prm.material_file}:/materialField has shape {mat.shape}, expected {prm.full[::-1]}")
    mat = np.ascontiguousarray(mat[:, cut[1], cut[2]])
    if mat.size and (mat.min() < 0 or mat.max() >= prm.dc.size):
        raise ValueError(f"materialField holds material {int(mat.max())}, outside the run's {prm.dc.size} materials")
    return SimpleNamespace(P=P, u=u, phase=phase, region=region, material=mat.astype(np.int8), z0=z0)


def q_axes(shape, spacing, qC):
    """1-D q axes of the fftshifted intensity (src/python/diffraction.py:51-59)."""
    return tuple(np.fft.fftshift(2 * math.pi * np.fft.fftfreq(m, h)) + qC[d]
                 for d, (m, h) in enumerate(zip(shape, spacing)))


def run(path, precision="fp32", device=0, out=None, verbose=True):
    """Run a parameter file on one GPU; writes <output_file> (and its .xdmf) and returns the intensity."""
    import torch

    t0 = time.perf_counter()
    prm = read_params(path)
    f = load_fields(prm)
    dev = torch.device("cuda", device)
    to = lambda a: None if a is None else torch.from_numpy(a).to(dev)
    t1 = time.perf_counter()
    crystal = Crystal(G=prm.G, qC=prm.qC, V=prm.V, R=prm.R, fAtom=prm.fAtom, su=prm.su)
    with Plan(prm.shape, prm.spacing, prm.nPhase, 3, precision=precision, device=device) as plan:
        plan.set_crystal(crystal)
        packed = plan.pack_fields(to(f.P), to(f.material), prm.dc, prm.phase_of, prm.spacing[2], z0=f.z0,
                                  u=to(f.u), phase=to(f.phase), region=to(f.region), p_scale=1.0,
                                  u_scale=prm.u_scale)
        I = plan.run_device(packed).cpu().numpy()
        plan.device_status()
        workspace = plan.workspace_bytes
    t2 = time.perf_counter()
    output = Path(out or prm.output_file)
    base = str(output.with_suffix("")) if output.suffix == ".h5" else str(output)
    step = 0
    qx, qy, qz = q_axes(prm.shape, prm.spacing, prm.qC)
    if os.path.exists(base + ".h5"):   # the skeleton written by qpop-diffraction --mgpu: keep its axes and step
        names = hdf5.list_datasets(base + ".h5")
        if {"q_x", "q_y", "q_z"} <= set(names):
            qx, qy, qz = (hdf5.read_dataset(base + ".h5", f"q_{c}") for c in "xyz")
        step = int(hdf5.read_attrs(base + ".h5").get("Timestep", 0))
    else:
        step = int(hdf5.read_attrs(prm.platt_file).get("Timestep", 0))
    hdf5.write_diffraction_output(base, I, qx, qy, qz, step)
    t3 = time.perf_counter()
    if verbose:
        nx, ny, nz = prm.shape
        print(f"grid {nx} x {ny} x {nz} on 1 GPU ({precision}), device workspace {workspace / 1e9:.2f} GB")
        print(f"read {t1 - t0:.2f} s, amplitude + intensity {t2 - t1:.2f} s, write {t3 - t2:.2f} s -> {base}.h5")
    return I


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("params", help="<out>_params.h5 written by qpop-diffraction --mgpu")
    ap.add_argument("--precision", choices=("fp32", "fp64"), default="fp32")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--output", default=None, help="write here instead of the file's output_file")
    args = ap.parse_args(argv)
    run(args.params, precision=args.precision, device=args.device, out=args.output)
    return 0


if __name__ == "__main__":
    sys.exit(main())
