"""
Python binding of qpd_run_device_noalloc, the allocation-free variant of the device path.

It is for callers that must not let a library allocate GPU memory: a framework whose caching
allocator owns the device's memory, or a real-time loop that reserves all of its memory up front.  The float32 fused computation is
the same as ``Plan.run_device``; the intermediate fields and tables live in one fixed device
array inside the library (``QPD_NOALLOC_SCRATCH_BYTES``, 32 MiB, held by every GPU that loads
the library until the process exits), so only small grids fit and larger ones are refused with
a MemoryError; crystals with more than 12 distinct R_x are refused with a ValueError.  All calls share that array: calls that can overlap on the GPU race, so the
caller serialises them.  The first call on a device looks up the array's address; make it
before any stream capture.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat
from .plan import Crystal

SCRATCH_BYTES = nat.QPD_NOALLOC_SCRATCH_BYTES


def run_device_noalloc(shape, spacing, crystal: Crystal, inputs, out, stream=None):
    """
    Enqueue one float32 volume on the current device without allocating device memory.

    inputs: packed single-phase-mode tensors as ``Plan.pack`` returns them (float32 P, U, int8
    phase, float32 weight or None); out: a contiguous float64 device tensor of nx*ny*nz values.
    """
    import torch
    lib = nat.load()
    if inputs.get("wdense") is not None:
        raise ValueError("the allocation-free call takes the single-phase mode (phase index and weight)")
    if out.dtype != torch.float64 or not out.is_contiguous() or out.numel() != int(np.prod(shape)):
        raise ValueError("out must be a contiguous float64 tensor of nx*ny*nz values")
    grid = nat.QpdGrid(*(int(s) for s in shape), *(float(h) for h in spacing))
    R = np.ascontiguousarray(crystal.R, dtype=np.float64)
    fr = np.ascontiguousarray(crystal.fAtom.real, dtype=np.float64)
    fi = np.ascontiguousarray(crystal.fAtom.imag, dtype=np.float64)
    su = np.ascontiguousarray(crystal.su, dtype=np.float64)
    dp = ctypes.POINTER(ctypes.c_double)
    k = nat.QpdCrystal(crystal.nAtom, crystal.nPhase, crystal.nStruc,
                       (ctypes.c_double * 3)(*map(float, crystal.G)), (ctypes.c_double * 3)(*map(float, crystal.qC)),
                       float(crystal.V), R.ctypes.data_as(dp), fr.ctypes.data_as(dp), fi.ctypes.data_as(dp),
                       su.ctypes.data_as(dp))

    def p(t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    rc = lib.qpd_run_device_noalloc(ctypes.byref(grid), ctypes.byref(k), p(inputs["P"]), p(inputs["U"]),
                                    p(inputs["phase"]), p(inputs.get("weight")), p(out), st)
    nat.check(lib, None, rc)
    return out
