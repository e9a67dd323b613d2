"""
ctypes binding of libqpopdiff.so (C ABI in include/qpopdiff.h).

The library must have been built (``qpop_diffraction_b200.build.build()``); there
is no fallback: importing a compute entry point without it raises.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int, c_int8, c_int32, c_int64, c_uint32, c_uint64, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libqpopdiff.so"

QPD_OK = 0
QPD_ERR_ARG = -1
QPD_ERR_CUDA = -2
QPD_ERR_NOMEM = -3
QPD_ERR_UNSUPPORTED = -4
QPD_ERR_STATE = -5

QPD_FP32 = 0
QPD_FP64 = 1
QPD_SCHED_FUSED = 0
QPD_SCHED_PLAIN = 1
QPD_NOALLOC_SCRATCH_BYTES = 32 << 20

PRECISIONS = {"fp32": QPD_FP32, "fp64": QPD_FP64}
SCHEDULES = {"fused": QPD_SCHED_FUSED, "plain": QPD_SCHED_PLAIN}

# Every symbol include/qpopdiff.h declares.
EXPORTS = ("qpd_create", "qpd_destroy", "qpd_last_error", "qpd_plan", "qpd_set_crystal", "qpd_run_host",
           "qpd_pack_device", "qpd_pack_fields", "qpd_run_device", "qpd_adjoint_device", "qpd_device_status", "qpd_probe_wait_timeout", "qpd_workspace_bytes", "qpd_launch_count", "qpd_set_cta_tiles", "qpd_enable_timing",
           "qpd_stage_times", "qpd_run_device_noalloc", "qpd_rsm_project", "qpd_axis_radices")

# Kernel kinds of qpd_stage_times (QPD_K_*), in index order.
KERNEL_KINDS = ("zstage", "ypass", "xpass", "pack", "source", "fftz", "axis", "accumulate", "intensity", "adj_seed",
                "adj_axis", "adj_z")


class QpdGrid(ctypes.Structure):
    _fields_ = [("nx", c_int64), ("ny", c_int64), ("nz", c_int64), ("dx", c_double), ("dy", c_double),
                ("dz", c_double)]


class QpdCrystal(ctypes.Structure):
    _fields_ = [("nAtom", c_int32), ("nPhase", c_int32), ("nStruc", c_int32), ("G", c_double * 3),
                ("qC", c_double * 3), ("V", c_double), ("R", POINTER(c_double)), ("f_re", POINTER(c_double)),
                ("f_im", POINTER(c_double)), ("su", POINTER(c_double))]


class QpdFields(ctypes.Structure):
    _fields_ = [("P", c_void_p * 3), ("u", c_void_p * 3), ("phase", c_void_p), ("region", c_void_p),
                ("material", c_void_p), ("nz_full", c_int64), ("z0", c_int64), ("n_material", c_int32),
                ("dc", POINTER(c_double)), ("phase_of", POINTER(c_int32)), ("ramp_dz", c_double),
                ("p_scale", c_double), ("u_scale", c_double)]


class QpdError(RuntimeError):
    """A failed libqpopdiff call: ``code`` is the QPD_ERR_* value."""

    def __init__(self, code, message):
        super().__init__(f"libqpopdiff error {code}: {message}")
        self.code = code


class QpdValueError(QpdError, ValueError):
    """Invalid argument or unsupported shape (QPD_ERR_ARG / QPD_ERR_UNSUPPORTED)."""


class QpdMemoryError(QpdError, MemoryError):
    """The workspace does not fit the device or the budget (QPD_ERR_NOMEM)."""


_lib = None


def load(path=None):
    """Load libqpopdiff.so once and declare its signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is not built: run qpop_diffraction_b200.build.build() (nvcc, sm_100a) first")
    lib = ctypes.CDLL(str(p))
    sig = {
        "qpd_create": (c_int, [c_int, c_uint64, POINTER(c_void_p)]),
        "qpd_destroy": (c_int, [c_void_p]),
        "qpd_last_error": (c_char_p, [c_void_p]),
        "qpd_plan": (c_int, [c_void_p, POINTER(QpdGrid), c_int32, c_int32, c_int32, c_int32]),
        "qpd_set_crystal": (c_int, [c_void_p, POINTER(QpdCrystal)]),
        "qpd_run_host": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
        "qpd_pack_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_void_p, c_void_p, c_int32, POINTER(c_uint32), c_void_p]),
        "qpd_pack_fields": (c_int, [c_void_p, POINTER(QpdFields), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_int32, POINTER(c_uint32), c_void_p]),
        "qpd_run_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p]),
        "qpd_adjoint_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_void_p]),
        "qpd_device_status": (c_int, [c_void_p]),
        "qpd_probe_wait_timeout": (c_int, [c_void_p, c_int64]),
        "qpd_workspace_bytes": (c_uint64, [c_void_p]),
        "qpd_launch_count": (c_uint64, [c_void_p]),
        "qpd_set_cta_tiles": (c_int, [c_void_p, c_int32]),
        "qpd_enable_timing": (c_int, [c_void_p, c_int32]),
        "qpd_stage_times": (c_int, [c_void_p, POINTER(c_double), POINTER(c_uint64), c_int32]),
        "qpd_run_device_noalloc": (c_int, [POINTER(QpdGrid), POINTER(QpdCrystal), c_void_p, c_void_p, c_void_p,
                                           c_void_p, c_void_p, c_void_p]),
        "qpd_rsm_project": (c_int, [c_void_p, c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
        "qpd_axis_radices": (c_int, [c_int64, POINTER(c_int32), c_int32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(lib, ctx, code):
    if code == QPD_OK:
        return
    msg = (lib.qpd_last_error(ctx) or b"").decode(errors="replace")
    if code in (QPD_ERR_ARG, QPD_ERR_UNSUPPORTED):
        raise QpdValueError(code, msg)
    if code == QPD_ERR_NOMEM:
        raise QpdMemoryError(code, msg)
    raise QpdError(code, msg)


def axis_radices(n):
    """FFT stage radices the library plans for an axis of length n (no GPU needed)."""
    lib = load()
    buf = (c_int32 * 64)()
    k = lib.qpd_axis_radices(int(n), buf, 64)
    if k < 0:
        raise QpdValueError(k, f"axis length {n}")
    return list(buf[:k])


__all__ = ["load", "check", "axis_radices", "QpdGrid", "QpdCrystal", "QpdFields", "QpdError", "QpdValueError", "QpdMemoryError",
           "EXPORTS", "KERNEL_KINDS", "PRECISIONS", "SCHEDULES", "c_int8"]
