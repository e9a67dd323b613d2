"""
Plans: a libqpopdiff context bound to one grid, precision and schedule.

``Plan`` keeps the device workspace between calls, so a snapshot grid is planned
once and then evaluated for any number of reflections.  Two ways to run it:

* ``run_host``: the reference-facing call, float64 host arrays in the layout
  ``diffraction()`` receives (src/python/diffraction.py:62-74), intensity back on
  the host;
* ``pack`` + ``run_device``: inputs resident on the GPU as torch tensors (packed
  float32/float64 fields, phase index), intensity into a device tensor, asynchronous
  on the current torch stream.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _native as nat


@dataclass
class Crystal:
    """Reflection and crystal constants the kernels need (the content of _params.h5, src/heffte/params.hpp:13-35)."""
    G: np.ndarray       # (3,) nm^-1
    qC: np.ndarray      # (3,) nm^-1
    V: float            # nm^3
    R: np.ndarray       # (nAtom, 3) nm
    fAtom: np.ndarray   # (nPhase, nAtom) complex
    su: np.ndarray      # (3, nStruc, nPhase, nAtom) nm per C/m^2

    @property
    def nAtom(self):
        return self.R.shape[0]

    @property
    def nPhase(self):
        return self.fAtom.shape[0]

    @property
    def nStruc(self):
        return self.su.shape[1]


def strain_tensor(strain_avg):
    """Voigt (xx, yy, zz, yz, xz, xy) -> 3x3, the order of src/python/diffraction.py:44-45."""
    e = np.asarray(strain_avg, dtype=np.float64)
    return np.array([[e[0], e[5], e[4]], [e[5], e[1], e[3]], [e[4], e[3], e[2]]])


def reciprocal_centre(aC, q00, strain_avg):
    """G nearest q00 and qC = G - eps G (src/python/diffraction.py:36-48), host float64."""
    aC = np.asarray(aC, dtype=np.float64)
    G = np.round(aC @ np.asarray(q00, dtype=np.float64) / (2 * math.pi)) @ (2 * math.pi * np.linalg.inv(aC).T)
    return G, G - strain_tensor(strain_avg) @ G


def crystal_from(params, atoms):
    """Crystal constants from the reference's SizeContext / AtomList objects (after setup())."""
    G, qC = reciprocal_centre(atoms.aC, atoms.q00, params.strainAvg)
    return Crystal(G=G, qC=qC, V=float(np.linalg.det(atoms.aC)), R=np.asarray(atoms.xAtom @ atoms.aC, dtype=np.float64),
                   fAtom=np.asarray(atoms.fAtom, dtype=np.complex128),
                   su=np.stack([atoms.su1, atoms.su2, atoms.su3]).astype(np.float64))


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class Plan:
    """A planned grid on one GPU.  Not thread-safe: use one Plan per host thread."""

    def __init__(self, shape, spacing, nPhase, nStruc=3, precision="fp32", schedule="fused", device=0,
                 hbm_budget=0):
        if precision not in nat.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(nat.PRECISIONS)}")
        if schedule not in nat.SCHEDULES:
            raise ValueError(f"schedule must be one of {sorted(nat.SCHEDULES)}")
        self.lib = nat.load()
        self.shape = tuple(int(s) for s in shape)
        self.spacing = tuple(float(h) for h in spacing)
        self.n = int(np.prod(self.shape))
        self.nPhase, self.nStruc = int(nPhase), int(nStruc)
        self.precision, self.schedule, self.device = precision, schedule, int(device)
        self._ctx = ctypes.c_void_p()
        nat.check(self.lib, None, self.lib.qpd_create(self.device, int(hbm_budget), ctypes.byref(self._ctx)))
        grid = nat.QpdGrid(*self.shape, *self.spacing)
        try:
            self._check(self.lib.qpd_plan(self._ctx, ctypes.byref(grid), self.nPhase, self.nStruc,
                                          nat.PRECISIONS[precision], nat.SCHEDULES[schedule]))
        except Exception:
            self.close()
            raise
        self.crystal = None

    def _check(self, code):
        nat.check(self.lib, self._ctx, code)

    def close(self):
        if self._ctx:
            self.lib.qpd_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def launches(self):
        return int(self.lib.qpd_launch_count(self._ctx))

    @property
    def workspace_bytes(self):
        return int(self.lib.qpd_workspace_bytes(self._ctx))

    def device_status(self):
        """Raise if a kernel of this plan gave up on a bounded wait (reads and clears the device status)."""
        self._check(self.lib.qpd_device_status(self._ctx))

    def probe_wait_timeout(self, polls=1000):
        """Run the bounded-wait failure path once (qpd_probe_wait_timeout); device_status() then raises."""
        self._check(self.lib.qpd_probe_wait_timeout(self._ctx, int(polls)))

    def set_cta_tiles(self, tiles):
        """At most `tiles` tiles per CTA of the persistent z stages (0: one wave of CTAs, the default), so
        that kernels on higher-priority streams get SMs while this volume's z stage runs."""
        self._check(self.lib.qpd_set_cta_tiles(self._ctx, int(tiles)))

    def enable_timing(self, on=True):
        """Record CUDA events around every kernel launch (see stage_times)."""
        self._check(self.lib.qpd_enable_timing(self._ctx, int(bool(on))))

    def stage_times(self):
        """{kernel kind: (summed device ms, launches)} since the last call; waits for the events."""
        k = len(nat.KERNEL_KINDS)
        ms = (ctypes.c_double * k)()
        cnt = (ctypes.c_uint64 * k)()
        self._check(self.lib.qpd_stage_times(self._ctx, ms, cnt, k))
        return {name: (ms[i], int(cnt[i])) for i, name in enumerate(nat.KERNEL_KINDS) if cnt[i]}

    def set_crystal(self, crystal: Crystal):
        if crystal.nPhase != self.nPhase or crystal.nStruc != self.nStruc:
            raise ValueError(f"crystal has nPhase {crystal.nPhase}, nStruc {crystal.nStruc}; "
                             f"the plan {self.nPhase}, {self.nStruc}")
        R = np.ascontiguousarray(crystal.R, dtype=np.float64)
        fr = np.ascontiguousarray(crystal.fAtom.real, dtype=np.float64)
        fi = np.ascontiguousarray(crystal.fAtom.imag, dtype=np.float64)
        su = np.ascontiguousarray(crystal.su, dtype=np.float64)
        dp = ctypes.POINTER(ctypes.c_double)
        k = nat.QpdCrystal(crystal.nAtom, crystal.nPhase, crystal.nStruc,
                           (ctypes.c_double * 3)(*map(float, crystal.G)), (ctypes.c_double * 3)(*map(float, crystal.qC)),
                           float(crystal.V), R.ctypes.data_as(dp), fr.ctypes.data_as(dp), fi.ctypes.data_as(dp),
                           su.ctypes.data_as(dp))
        self._check(self.lib.qpd_set_crystal(self._ctx, ctypes.byref(k)))
        self.crystal = crystal

    # ---------------- host path ----------------
    def _host(self, a, count, name):
        arr = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        if arr.size != count:
            raise ValueError(f"{name} has {arr.size} values, expected {count}")
        return arr

    def run_host(self, oPhase, oStruc, u, region, out=None):
        """I (nx, ny, nz) float64 from float64 host arrays in the reference layout."""
        if self.crystal is None:
            raise RuntimeError("set_crystal() first")
        n = self.n
        oPhase = self._host(oPhase, self.nPhase * n, "oPhase")
        oStruc = self._host(oStruc, self.nStruc * n, "oStruc") if self.nStruc else None
        u = self._host(u, 3 * n, "u")
        region = self._host(region, n, "region") if region is not None else None
        I = out if out is not None else np.empty(self.shape, dtype=np.float64)
        if I.dtype != np.float64 or not I.flags.c_contiguous or I.size != n:
            raise ValueError("out must be a C-contiguous float64 array of n values")
        self._check(self.lib.qpd_run_host(self._ctx, _ptr(oPhase), _ptr(oStruc), _ptr(u), _ptr(region), _ptr(I)))
        return I

    # ---------------- device path (torch tensors) ----------------
    @property
    def torch_dtype(self):
        import torch
        return torch.float32 if self.precision == "fp32" else torch.float64

    def pack(self, oPhase, oStruc, u, region=None, stream=None):
        """
        Pack float64 device tensors (reference layout) into kernel inputs.  Returns a dict with
        P, U and either phase + weight (weight None when every weight is 0 or 1) or wdense.
        """
        import torch
        dev = torch.device("cuda", self.device)
        n = self.n
        f64 = dict(dtype=torch.float64, device=dev)

        def flat(t, count, name):
            t = t.reshape(-1)
            if t.numel() != count or t.dtype != torch.float64 or t.device != dev:
                raise ValueError(f"{name}: expected {count} float64 values on {dev}")
            return t.contiguous()

        oPhase = flat(oPhase, self.nPhase * n, "oPhase")
        oStruc = flat(oStruc, self.nStruc * n, "oStruc") if self.nStruc else torch.zeros(1, **f64)
        u = flat(u, 3 * n, "u")
        region = flat(region, n, "region") if region is not None else None
        dt = self.torch_dtype
        P = torch.empty(3 * n, dtype=dt, device=dev)
        U = torch.empty(3 * n, dtype=dt, device=dev)
        phase = torch.empty(n, dtype=torch.int8, device=dev)
        weight = torch.empty(n, dtype=dt, device=dev)
        flags = ctypes.c_uint32(0)
        st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream)

        def call(dense, wd):
            self._check(self.lib.qpd_pack_device(
                self._ctx, ctypes.c_void_p(oPhase.data_ptr()), ctypes.c_void_p(oStruc.data_ptr()),
                ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(region.data_ptr()) if region is not None else None,
                ctypes.c_void_p(P.data_ptr()), ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(phase.data_ptr()),
                ctypes.c_void_p(weight.data_ptr()), ctypes.c_void_p(wd.data_ptr()) if wd is not None else None,
                int(dense), ctypes.byref(flags), st))

        call(False, None)
        if flags.value & 1:
            wdense = torch.empty(self.nPhase * n, dtype=dt, device=dev)
            call(True, wdense)
            return {"P": P, "U": U, "phase": None, "weight": None, "wdense": wdense}
        return {"P": P, "U": U, "phase": phase, "weight": weight if flags.value & 2 else None, "wdense": None}

    def adjoint(self, inputs, grad_I, stream=None):
        """
        dL/dP and dL/dU (each 3 * n in the plan precision) for packed inputs and dL/dI, a float64 CUDA
        tensor of n values laid out like I (fftshifted).  The forward is recomputed on the device.
        """
        import torch
        if self.crystal is None:
            raise RuntimeError("set_crystal() first")
        dev = torch.device("cuda", self.device)
        g = grad_I.reshape(-1)
        if g.dtype != torch.float64 or g.numel() != self.n or g.device != dev:
            raise ValueError(f"grad_I: expected {self.n} float64 values on {dev}")
        g = g.contiguous()
        dP = torch.empty(3 * self.n, dtype=self.torch_dtype, device=dev)
        dU = torch.empty(3 * self.n, dtype=self.torch_dtype, device=dev)

        def p(t):
            return ctypes.c_void_p(t.data_ptr()) if t is not None else None

        st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream)
        self._check(self.lib.qpd_adjoint_device(self._ctx, p(inputs["P"]), p(inputs["U"]), p(inputs.get("phase")),
                                                p(inputs.get("weight")), p(inputs.get("wdense")), p(g), p(dP),
                                                p(dU), st))
        return dP, dU

    def pack_fields(self, P, material, dc, phase_of, ramp_dz, z0=0, u=None, phase=None, region=None,
                    p_scale=1.0, u_scale=1e9, stream=None):
        """
        Pack Q-POP-FerroDyn fields resident on the GPU into kernel inputs (qpd_pack_fields): the
        preparation of src/python/cli.py:174-217 on the device.

        P (nStruc planes), u (3 planes, metres; None: 0), phase (nPhase planes; None: one-hot from
        the material) and region (None: 1) are float32 CUDA tensors in file order (nz, ny, nx),
        cropped to the plan's grid; material is int8 (nz_full, ny, nx): the crop's columns over the
        full stack, of which the crop starts at layer z0.  dc and phase_of are per-material tables
        (c_m / aC_z - 1; phase index or -1).  Returns the same dict as pack().
        """
        import torch
        dev = torch.device("cuda", self.device)
        nx, ny, nz = self.shape
        plane = nz * ny * nx
        keep = []

        def f32(t, count, name):
            if t.dtype != torch.float32 or t.device != dev or t.numel() != count:
                raise ValueError(f"{name}: expected {count} float32 values on {dev} in (nz, ny, nx) order")
            t = t.contiguous()
            keep.append(t)
            return t.data_ptr()

        def planes(ts, k, name):
            if isinstance(ts, torch.Tensor):
                ts = [ts[i] for i in range(ts.shape[0])] if ts.dim() == 4 else [ts]
            if len(ts) < k:
                raise ValueError(f"{name}: expected {k} planes")
            return [f32(t, plane, f"{name}[{i}]") for i, t in enumerate(ts[:k])]

        fields = nat.QpdFields()
        for i, ptr in enumerate(planes(P, self.nStruc, "P") if self.nStruc else []):
            fields.P[i] = ptr
        if u is not None:
            for i, ptr in enumerate(planes(u, 3, "u")):
                fields.u[i] = ptr
        if phase is not None:
            fields.phase = f32(phase, self.nPhase * plane, "phase")
        if region is not None:
            fields.region = f32(region, plane, "region")
        if material.dtype != torch.int8 or material.device != dev or material.dim() != 3 or \
                tuple(material.shape[1:]) != (ny, nx):
            raise ValueError(f"material: expected an int8 (nz_full, {ny}, {nx}) tensor on {dev}")
        material = material.contiguous()
        keep.append(material)
        fields.material = material.data_ptr()
        fields.nz_full, fields.z0 = int(material.shape[0]), int(z0)
        dc = np.ascontiguousarray(dc, dtype=np.float64)
        phase_of = np.ascontiguousarray(phase_of, dtype=np.int32)
        if dc.shape != phase_of.shape or dc.ndim != 1:
            raise ValueError("dc and phase_of: one entry per material")
        fields.n_material = int(dc.size)
        fields.dc = dc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        fields.phase_of = phase_of.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        fields.ramp_dz, fields.p_scale, fields.u_scale = float(ramp_dz), float(p_scale), float(u_scale)

        n = self.n
        dt = self.torch_dtype
        Pout = torch.empty(3 * n, dtype=dt, device=dev)
        Uout = torch.empty(3 * n, dtype=dt, device=dev)
        phase_idx = torch.empty(n, dtype=torch.int8, device=dev)
        weight = torch.empty(n, dtype=dt, device=dev)
        flags = ctypes.c_uint32(0)
        st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream)

        def call(dense, wd):
            self._check(self.lib.qpd_pack_fields(
                self._ctx, ctypes.byref(fields), ctypes.c_void_p(Pout.data_ptr()), ctypes.c_void_p(Uout.data_ptr()),
                ctypes.c_void_p(phase_idx.data_ptr()), ctypes.c_void_p(weight.data_ptr()),
                ctypes.c_void_p(wd.data_ptr()) if wd is not None else None, int(dense), ctypes.byref(flags), st))

        call(False, None)
        if flags.value & 1:
            wdense = torch.empty(self.nPhase * n, dtype=dt, device=dev)
            call(True, wdense)
            return {"P": Pout, "U": Uout, "phase": None, "weight": None, "wdense": wdense}
        return {"P": Pout, "U": Uout, "phase": phase_idx, "weight": weight if flags.value & 2 else None, "wdense": None}

    def run_device(self, inputs, out=None, stream=None):
        """Enqueue the hot path on device-resident packed inputs; returns the (nx, ny, nz) float64 tensor."""
        import torch
        if self.crystal is None:
            raise RuntimeError("set_crystal() first")
        dev = torch.device("cuda", self.device)
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float64, device=dev)
        if out.dtype != torch.float64 or out.numel() != self.n or not out.is_contiguous():
            raise ValueError("out must be a contiguous float64 tensor of n values")

        def p(t):
            return ctypes.c_void_p(t.data_ptr()) if t is not None else None

        st = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream)
        self._check(self.lib.qpd_run_device(self._ctx, p(inputs["P"]), p(inputs["U"]), p(inputs.get("phase")),
                                            p(inputs.get("weight")), p(inputs.get("wdense")), p(out), st))
        return out
