#!/usr/bin/env python3
"""
Throughput of the kinematic-diffraction hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one 3-D intensity volume: one (snapshot, reflection) evaluation of all atoms,
their four FFT components and the |S Amp|^2 + fftshift epilogue.  The workload is the
two-phase polar-vortex film of 512 x 512 x 104 cells (5 atoms, 2 phases), alternating
between the reflections G = (0,0,2) and (1,0,3) on one resident snapshot; the inputs are
seeded synthetic fields (qpop_diffraction_b200.workloads.config2_*), since the reference
ships no dataset at this size.

Printed (rank 0, one JSON line):
  value     Gcells/s over all ranks, inputs resident in HBM (packed float32 P, u, int8 phase)
            and the intensity left in HBM; device time by CUDA events, max over ranks;
  e2e       the same metric through the reference-facing C-ABI call qpd_run_host: float64
            host arrays in pinned memory, host->device copies, packing, the transform and the
            float64 intensity copied back, all inside the timed region;
  roofline  the dominant kernel's algorithmic bytes per launch / its mean event-timed duration,
            against the measured HBM copy bandwidth;
  cpu_baseline  the reference's own NumPy diffraction() (the unmodified package installed under
            baseline/_ref) on the full 512 x 512 x 104 grid, one run on this host; its result is also
            the float64 oracle of the full-grid accuracy figures;
  fp64      the same hand-written kernels in float64, fused and plain (the reference's own
            per-atom, per-component schedule), for the float32-vs-float64 comparison;
  accuracy  float32 against float64: the reference itself at G=002 on the full grid, the float64
            oracle per workload (configs 1, 2 at G=103, serving grids, the config-5 forward, direct
            sums at 1024 x 1024 x 68), and the same kernels in float64;
  config3   the 4000 x 4000 x 68 twin film on one GPU: per-pass times and roofline fractions,
            device memory and float64 direct sums at 64 voxels (bench.py --config 3 adds one
            end-to-end volume from float64 host arrays through qpd_run_host).

With --impl reference only the reference's own diffraction() runs (rank 0, NumPy with its own
threading, as the reference computes), on a bounded crop of the workload per step; the oracle
port stands in when baseline/_ref is absent.
Under torchrun each rank evaluates its own volumes on its own GPU (replicas: the path has no
cross-volume exchange), so scaling is weak.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GRID = (512, 512, 104)
REFLECTIONS = ((0, 0, 2), (1, 0, 3))
METRIC = "Gcells/s per 3-D volume at 512x512x104 (float32 source+FFT, float64 phase reduction)"
UNIT = "Gcells/s"
REF_SAMPLE = (128, 128, 104)        # --impl reference: one step, so K + W steps end in minutes
FALLBACK_HBM = 6650.0


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--grid", type=int, nargs=3, default=GRID)
    ap.add_argument("--e2e-steps", type=int, default=None, help="steps of the host-buffer leg (default: min(K, 20))")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the float64 comparison leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving (request loop) leg")
    ap.add_argument("--serving-requests", type=int, default=400)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiation (adjoint) leg")
    ap.add_argument("--config", type=int, default=2, choices=(2, 3),
                    help="3: the 4000x4000x68 twin film on one GPU (device-resident, per-pass roofline)")
    ap.add_argument("--validate", action="store_true", help="with --config 3: compare against a float64 plain run")
    ap.add_argument("--no-config3", action="store_true", help="skip the 4000x4000x68 leg of the default run")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the per-workload float32-vs-float64-oracle leg of the default run")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id):
        self.device_id = device_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device_id), "-lms", "50"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
            except ValueError:
                continue
            for name, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def atom_groups(R):
    """Field counts of the fused schedule: g1 = distinct (R_x, R_y), g2 = distinct R_x."""
    return len({(r[0], r[1]) for r in R}), len({r[0] for r in R})


def kernel_bytes(n, g1, g2, weight):
    """Algorithmic HBM bytes per launch of each fused kernel (float32 inputs, complex64 fields, float64 I)."""
    b_in = 24 + 1 + (4 if weight else 0)
    return {"zstage": n * (b_in + 3 * g1 * 8), "ypass": n * (3 * g1 * 8 + 2 * g2 * 8), "xpass": n * (2 * g2 * 8 + 8)}


def profiled_traffic():
    """DRAM bytes per cell of each fused kernel from the committed ncu summary (profiles/), if present."""
    out = {}
    for p in sorted((ROOT / "profiles").glob("*.md")):
        for line in p.read_text().splitlines():
            if line.startswith("traffic_bytes_per_cell"):
                for item in line.split()[1:]:
                    k, _, v = item.partition("=")
                    out[k] = float(v)
    return out


def host_cpu():
    """CPU model and core count of this host."""
    model = "unknown CPU"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{model}, {os.cpu_count()} cores"


def reference_diffraction():
    """
    The reference's own diffraction() (baseline/_ref or a source checkout), or None.  Called with its
    progress prints (G, qC) sent to /dev/null, so the JSON line stays the last line of the output.
    """
    import contextlib
    sys.path.insert(0, str(ROOT / "tests"))
    import reference_pkg
    mods = reference_pkg.load("diffraction")
    if mods is None:
        return None
    fn = mods[0].diffraction

    def quiet(*a, **k):
        with open(os.devnull, "w") as null, contextlib.redirect_stdout(null):
            return fn(*a, **k)
    return quiet


def run_reference(args, rank):
    """
    The reference arm: the unmodified reference diffraction() (src/python/diffraction.py:62-113, NumPy
    with its own threading, as the reference runs) on a crop of the config-2 snapshot, both reflections
    alternating.
    """
    if rank != 0:
        return
    from qpop_diffraction_b200 import workloads
    diffraction = reference_diffraction()
    kind, cores = "reference", os.cpu_count()  # as the reference runs: NumPy's own threading
    if diffraction is None:  # no install and no checkout: the oracle port, the same algorithm restated
        from oracle import diffraction_oracle as oracle
        diffraction, kind = oracle.diffraction, "port"
    cases = [workloads.config2(shape=REF_SAMPLE, hkl=h) for h in REFLECTIONS]
    for i in range(args.warmup):
        diffraction(*cases[i % 2].args())
    t = time.perf_counter()
    for i in range(args.steps):
        diffraction(*cases[i % 2].args())
    dt = time.perf_counter() - t
    n = cases[0].params.n
    value = args.steps * n / dt / 1e9
    who = "the reference's own diffraction() (baseline/_ref, unmodified, NumPy as installed)" if kind == "reference" else \
          "the oracle port of the reference's diffraction() (NumPy)"
    sample = (f"{who} on the config-2 snapshot cropped to {'x'.join(map(str, REF_SAMPLE))}, G=002,103 alternating, "
              f"one crop per step; host {host_cpu()}")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"two-phase polar-vortex film {'x'.join(map(str, GRID))}, 5 atoms, 2 phases, "
                               f"G=002,103 alternating", "grid": list(GRID), "cells": int(np.prod(GRID)), "atoms": 5,
                   "phases": 2, "precision": "fp64 (NumPy, as the reference computes)", "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


CONFIG3 = (4000, 4000, 68)


def intensity_errors(I, ref):
    """Float32-contract figures of I against a float64 reference volume (numpy or torch)."""
    I = np.asarray(I, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    imax = ref.max()
    strong = ref > 1e-6 * imax
    dlog = np.abs(np.log10(I[strong]) - np.log10(ref[strong]))
    return {"max_abs_dI_over_Imax": float(np.abs(I - ref).max() / imax),
            "max_rel_err_above_1e-6_Imax": float((np.abs(I - ref)[strong] / ref[strong]).max()),
            "max_abs_dlog10I_above_1e-6_Imax": float(dlog.max()),
            "voxels_above_1e-6_Imax": int(strong.sum()),
            "contract": "max |dI|/I_max <= 1e-5, rel <= 1e-3 above 1e-6 I_max"}


def pick_voxels(torch, out, nbright=32, nrandom=32, seed=11):
    """FFT-order indices of the brightest and of random voxels of a shifted volume, and their values."""
    sys.path.insert(0, str(ROOT / "tests"))
    from direct_dft import fft_index_to_shifted, shifted_to_fft_index
    shape = tuple(out.shape)
    top = torch.topk(out.view(-1), nbright).indices.cpu().numpy()
    sx, sy, sz = np.unravel_index(top, shape)
    inv = [shifted_to_fft_index(m) for m in shape]
    bright = np.stack([inv[0][sx], inv[1][sy], inv[2][sz]], axis=1)
    rng = np.random.default_rng(seed)
    vox = np.concatenate([bright, np.stack([rng.integers(0, m, nrandom) for m in shape], axis=1)])
    pos = [fft_index_to_shifted(m) for m in shape]
    sel = [torch.from_numpy(pos[d][vox[:, d]]).to(out.device) for d in range(3)]
    return vox, out[sel[0], sel[1], sel[2]].cpu().numpy()


def direct_errors(torch, params, atoms, inputs, vox, got):
    """The values `got` at voxels `vox` against float64 direct sums over all cells (tests/direct_dft.py)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from direct_dft import crystal_constants, direct_intensity
    shape = (params.nx, params.ny, params.nz)
    t = time.perf_counter()
    want = direct_intensity(torch, shape, (params.dx, params.dy, params.dz), *crystal_constants(params, atoms),
                            inputs["P"], inputs["U"], inputs["phase"], inputs["weight"], vox)
    imax = want.max()
    big = want > 1e-6 * imax
    return {"voxels": int(len(vox)), "voxels_above_1e-6_Imax": int(big.sum()),
            "max_abs_dI_over_Imax": float(np.abs(got - want).max() / imax),
            "max_rel_err_above_1e-6_Imax": float((np.abs(got - want)[big] / want[big]).max()),
            "max_abs_dlog10I_above_1e-6_Imax": float(np.abs(np.log10(got[big]) - np.log10(want[big])).max()),
            "seconds": time.perf_counter() - t,
            "against": f"float64 direct sums over all cells (no FFT), {len(vox) // 2} brightest + "
                       f"{len(vox) - len(vox) // 2} random voxels"}


def oracle_arrays(params, inputs):
    """Float64 host arrays (oPhase, oStruc, u, region) in the reference layout holding packed device inputs."""
    ph = inputs["phase"].cpu().numpy().astype(np.int64)
    oPhase = np.concatenate([(ph == p).astype(np.float64) for p in range(params.nPhase)])
    region = np.ones(ph.size) if inputs["weight"] is None else inputs["weight"].double().cpu().numpy()
    return oPhase, inputs["P"].double().cpu().numpy(), inputs["U"].double().cpu().numpy(), region


def accuracy_leg(torch, dev, config2=None):
    """
    The float32 fused path against the float64 oracle (the reference's diffraction() restated in NumPy,
    pinned to the reference's own outputs by the golden tests) on each workload's own inputs:
    config 1 through the drop-in diffraction() call, the config-2 grid at G=103 (G=002 is compared
    with the reference itself by the CPU baseline), two serving grids, the config-5 forward, and the
    1024 x 1024 x 68 serving grid by float64 direct sums at 64 voxels.  config2: (params, host arrays,
    float32 volume at G=103) of the bench's config-2 snapshot.
    """
    import qpop_diffraction_b200 as qpd
    from oracle import diffraction_oracle as oracle
    from qpop_diffraction_b200 import Plan, crystal_from, workloads
    threads = oracle.default_threads(5)
    out = {}

    def entry(name, I32, params, atoms, arrays):
        t = time.perf_counter()
        ref = oracle.diffraction(params, atoms, *arrays, threads=threads)[0]
        out[name] = dict(intensity_errors(I32, ref), oracle_seconds=time.perf_counter() - t)

    case = workloads.config1()
    I32 = qpd.diffraction(*case.args(), device=dev.index)[0]
    entry("config 1: 64x64x32 perovskite stripes, G=002 (drop-in diffraction())", I32, case.params, case.atoms,
          (case.oPhase, case.oStruc, case.u, case.region))
    if config2 is not None:
        params, arrays, I32 = config2
        entry(f"config 2: {'x'.join(map(str, GRID))} polar-vortex film, G=103", I32, params,
              workloads.config2_crystal(2, (1, 0, 3)), arrays)
    for kind, shape, seed, hkl, label in (("vortex", (128, 128, 128), 1000, (0, 0, 2), "serving"),
                                          ("twin", (256, 256, 64), 1005, (1, 1, 3), "serving"),
                                          ("vortex", (256, 256, 64), 5, (1, 0, 3), "config 5 forward")):
        params, inputs = workloads.gpu_snapshot(kind, shape, seed=seed, device=dev)
        atoms = workloads.serving_crystal(hkl)
        with Plan(shape, (params.dx, params.dy, params.dz), params.nPhase, 3, precision="fp32",
                  device=dev.index) as plan:
            plan.set_crystal(crystal_from(params, atoms))
            I32 = plan.run_device(inputs).cpu().numpy()
        entry(f"{label}: {'x'.join(map(str, shape))} {kind} (seed {seed}), G={''.join(map(str, hkl))}", I32, params,
              atoms, oracle_arrays(params, inputs))
        del inputs
    shape, hkl = (1024, 1024, 68), (1, 0, 3)
    params, inputs = workloads.gpu_snapshot("twophase", shape, seed=1002, device=dev)
    atoms = workloads.serving_crystal(hkl)
    with Plan(shape, (params.dx, params.dy, params.dz), params.nPhase, 3, precision="fp32", device=dev.index) as plan:
        plan.set_crystal(crystal_from(params, atoms))
        vox, got = pick_voxels(torch, plan.run_device(inputs))
    out[f"serving: {'x'.join(map(str, shape))} twophase (seed 1002), G=103, direct sums"] = \
        direct_errors(torch, params, atoms, inputs, vox, got)
    del inputs
    torch.cuda.empty_cache()
    return {"threads": threads, "cases": out,
            "against": "float64 oracle on the same inputs (full volume), or float64 direct sums where marked"}


def config3_leg(args, torch, dev, rank, world, shape=CONFIG3, steps=3, warmup=1, validate=False, direct=True,
                e2e=True):
    """
    The 4000 x 4000 x 68 three-variant Voronoi twin film (1.09e9 cells, one phase, G = 113) on one
    GPU: generated on the device, float32 fused schedule, inputs resident; per-pass event times.
    direct: float64 direct sums over all cells at 64 voxels (32 brightest, 32 random) against the
    volume (tests/direct_dft.py, no FFT).  e2e: one volume from float64 host arrays in the reference
    layout through qpd_run_host (host arrays of about 78 GB), timed with its copies.  validate: the
    same volume in float64 with the plain schedule, compared on the GPU.
    """
    from qpop_diffraction_b200 import Plan, crystal_from, replicas, workloads
    params, inputs = workloads.gpu_snapshot("twin", shape, seed=3 + rank, device=dev, n_phase=1)
    atoms = workloads.config3_crystal(3, (1, 1, 3))
    crystal = crystal_from(params, atoms)
    spacing = (params.dx, params.dy, params.dz)
    n = params.n
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    torch.cuda.reset_peak_memory_stats(dev)
    plan = Plan(shape, spacing, 1, 3, precision="fp32", device=dev.index)
    plan.set_crystal(crystal)
    out = torch.empty(shape, dtype=torch.float64, device=dev)
    for _ in range(warmup):
        plan.run_device(inputs, out)
    torch.cuda.synchronize(dev)
    plan.device_status()
    plan.stage_times()
    plan.enable_timing(True)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.run_device(inputs, out)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    plan.device_status()
    ms = replicas.slowest(e0.elapsed_time(e1), dev) / steps
    stage = plan.stage_times()
    plan.enable_timing(False)
    hbm, hbm_src = peaks()
    g1, g2 = atom_groups(crystal.R)
    kb = kernel_bytes(n, g1, g2, False)
    kernels = {k: {"avg_ms": t / c, "bytes_per_launch": kb[k], "gbs": kb[k] / (t / c * 1e-3) / 1e9,
                   "frac": kb[k] / (t / c * 1e-3) / 1e9 / hbm} for k, (t, c) in stage.items() if k in kb}
    res = {"workload": f"three-variant Voronoi twin film {'x'.join(map(str, shape))}, 200 domains, 5 atoms, "
                       f"1 phase, G=113, generated on the GPU", "cells": n, "steps": steps, "warmup": warmup,
           "ms_per_volume": ms, "value": replicas.throughput(n, ms * 1e-3, world) / 1e9, "unit": UNIT,
           "kernels": kernels, "peak_gbs": hbm, "peak_source": f"hbm_gbs of {hbm_src}",
           "device_memory_peak_gb": (torch.cuda.max_memory_allocated(dev) + plan.workspace_bytes) / 1e9}
    # the model schedule's bytes (3 passes per atom and component, b_in = 25): A (25 + 144) per cell; the fused
    # schedule moves about 290, so this fraction can exceed 1
    model_cell = len(crystal.R) * (25 + 144)
    res["model_roofline"] = {"bytes_per_cell": model_cell, "achieved_gbs": n * model_cell / (ms * 1e-3) / 1e9,
                             "frac": n * model_cell / (ms * 1e-3) / 1e9 / hbm}
    if direct:
        vox, got = pick_voxels(torch, out)
        plan.close()
        del out
        torch.cuda.empty_cache()
        res["direct_sums"] = direct_errors(torch, params, atoms, inputs, vox, got)
    else:
        plan.close()
        del out
    if validate:
        torch.cuda.empty_cache()
        out32 = None
        p32 = Plan(shape, spacing, 1, 3, precision="fp32", device=dev.index)
        p32.set_crystal(crystal)
        out32 = p32.run_device(inputs).cpu()
        p32.close()
        in64 = {"P": inputs["P"].double(), "U": inputs["U"].double(), "phase": inputs["phase"], "weight": None,
                "wdense": None}
        torch.cuda.empty_cache()
        p64 = Plan(shape, spacing, 1, 3, precision="fp64", schedule="plain", device=dev.index)
        p64.set_crystal(crystal)
        t = time.perf_counter()
        I64 = p64.run_device(in64)
        torch.cuda.synchronize(dev)
        p64.device_status()
        res["validation"] = dict(intensity_errors(out32.numpy(), I64.cpu().numpy()),
                                 against="float64 plain schedule of the same kernels on the full grid",
                                 fp64_plain_seconds=time.perf_counter() - t)
        p64.close()
        del in64, I64
        torch.cuda.empty_cache()
    if e2e:
        import psutil
        if psutil.virtual_memory().available < 120e9:
            res["e2e"] = {"skipped": "needs about 90 GB of free host memory for the float64 host arrays"}
        else:
            # the reference layout on the host: float64 oPhase, oStruc (P), u, region, as cli.py hands them over
            host = {"oStruc": inputs["P"].reshape(-1).cpu().numpy().astype(np.float64),
                    "u": inputs["U"].reshape(-1).cpu().numpy().astype(np.float64)}
            ph = inputs["phase"].reshape(-1).cpu().numpy()
            host["oPhase"] = (ph == 0).astype(np.float64)
            host["region"] = (ph >= 0).astype(np.float64)
            del ph, inputs
            torch.cuda.empty_cache()
            I_host = np.empty(shape, dtype=np.float64)
            ph = Plan(shape, spacing, 1, 3, precision="fp32", device=dev.index)
            ph.set_crystal(crystal)
            ph.run_host(host["oPhase"], host["oStruc"], host["u"], host["region"], out=I_host)  # workspace, ring
            ph.stage_times()
            ph.enable_timing(True)
            t = time.perf_counter()
            ph.run_host(host["oPhase"], host["oStruc"], host["u"], host["region"], out=I_host)
            total = time.perf_counter() - t
            kern = sum(v[0] for v in ph.stage_times().values())
            h2d = sum(a.nbytes for a in host.values())
            res["e2e"] = {"value": n / total / 1e9, "unit": UNIT, "seconds": total, "kernels_ms": kern,
                          "host_transfer_and_pack_ms": total * 1e3 - kern, "h2d_bytes": h2d, "d2h_bytes": I_host.nbytes,
                          "call": "qpd_run_host: float64 host arrays in the reference layout (pageable), the intensity "
                                  "back in a float64 host array"}
            ph.close()
            del host, I_host
    return res


def run_config3(args, torch, dev, rank, world):
    """bench.py --config 3: the config-3 leg alone, one JSON line (--validate adds the float64 run)."""
    shape = tuple(args.grid) if tuple(args.grid) != GRID else CONFIG3
    res = config3_leg(args, torch, dev, rank, world, shape=shape, steps=args.steps, warmup=args.warmup,
                      validate=args.validate, direct=shape == CONFIG3, e2e=shape == CONFIG3 and args.e2e_steps != 0)
    if rank == 0:
        line = {"metric": f"Gcells/s per 3-D volume at {'x'.join(map(str, shape))} (float32, one GPU)",
                "value": res["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": res["ms_per_volume"], "higher_is_better": True, "scaling": "weak", "dtype": "f32",
                "data": "synthetic (seeded Voronoi twin film, generated on the GPU)",
                "config": {"workload": res["workload"], "cells": res["cells"]}}
        line.update({k: v for k, v in res.items() if k not in ("value", "workload", "cells")})
        print(json.dumps(line), flush=True)


SERVING_SHAPES = ((128, 128, 128), (256, 256, 64), (512, 512, 104), (1024, 1024, 68))
SERVING_HKLS = ((0, 0, 2), (1, 0, 3), (1, 1, 3), (2, 0, 0))


# Engine options of the serving leg: stream priorities by grid size and at most two volumes in flight per
# grid (measured on one B200: capacity 306 against 219 volumes/s with unlimited slots and no priorities,
# p50 at 80% load 3.8 against 9.9 ms); with priorities the engine also caps the tiles per CTA of the
# persistent z stages (Engine cta_tiles), so a small volume does not wait out a large one's z stage
SERVING_POLICY = {"priorities": True, "max_slots": 2}


def serving_leg(args, torch, device, policy=None):
    """
    32 resident snapshots (8 per grid of the serving mix, vortex / twin / two-phase textures) and
    Poisson requests over them and the 4 reflections.  Capacity: every request queued at once; then
    an open-loop run at 80% of that rate.  Latency is arrival to completion, on the device.
    """
    from qpop_diffraction_b200 import workloads
    from qpop_diffraction_b200.serving import Engine, Snapshot, SnapshotStore, latency_stats, poisson_requests
    store = SnapshotStore()
    for i in range(32):
        shape = SERVING_SHAPES[i % 4]
        kind = workloads.TEXTURES[(i // 4) % 3]
        params, inputs = workloads.gpu_snapshot(kind, shape, seed=1000 + i, device=f"cuda:{device}")
        store.add(Snapshot(i, kind, shape, params, inputs))
    free, total = torch.cuda.mem_get_info(device)
    budget = int(min(free - (8 << 30), 64 << 30))
    policy = SERVING_POLICY if policy is None else policy
    eng = Engine(store, budget, device=device, **policy)
    try:
        for i in range(4):                      # two slots per grid where the budget allows
            eng.reserve(i, 2)
        eng.warm([(i, h) for i in range(32) for h in SERVING_HKLS])
        ids = list(range(32))
        shape_of = lambda r: "x".join(map(str, store[r.snapshot].shape))
        cap = latency_stats(eng.run(poisson_requests(args.serving_requests, 0, ids, SERVING_HKLS, seed=1)))
        loads = {}
        for i, frac in enumerate((0.5, 0.8, 0.95)):
            rate = frac * cap["volumes_per_s"]
            st = latency_stats(eng.run(poisson_requests(args.serving_requests, rate, ids, SERVING_HKLS, seed=2 + i)),
                               key=shape_of)
            loads[f"{int(frac * 100)}%"] = dict(st, offered_rate_per_s=rate)
        load = loads["80%"]
        out = {"grids": [list(s) for s in SERVING_SHAPES], "snapshots": 32, "reflections": [list(h) for h in SERVING_HKLS],
               "capacity_volumes_per_s": cap["volumes_per_s"], "offered_rate_per_s": load["offered_rate_per_s"],
               "p50_ms": load["p50_ms"], "p99_ms": load["p99_ms"], "volumes_per_s": load["volumes_per_s"],
               "requests": load["requests"], "loads": loads,
               "slots": eng.peak_slots, "policy": dict(policy, cta_tiles=eng.cta_tiles), "hbm_budget_gb": budget / 1e9,
               "resident_snapshots_gb": store.nbytes / 1e9,
               "latency": "arrival to completion on the device, open-loop Poisson arrivals; p50/p99 at 80% of capacity, "
                          "loads: at 50, 80 and 95%, overall and per grid"}
    finally:
        eng.close()
    return out


def adjoint_leg(args, torch, device, steps=20):
    """
    Differentiation workload: 256 x 256 x 64 polar-vortex film, loss sum_q (log10 I - log10 I_target)^2
    with I_target from the unperturbed field, evaluated at P + N(0, 0.05), u + N(0, 0.001 nm).
    Times forward + loss + backward (the hand-written adjoint recomputes the forward) in float32 and
    compares its gradients with the float64 adjoint of the same kernels.
    """
    from qpop_diffraction_b200 import Plan, autograd, crystal_from, workloads
    shape = (256, 256, 64)
    dev = torch.device("cuda", device)
    params, inputs = workloads.gpu_snapshot("vortex", shape, seed=5, device=f"cuda:{device}")
    crystal = crystal_from(params, workloads.config2_crystal(2, (1, 0, 3)))
    n = params.n
    g = torch.Generator(device=dev)
    g.manual_seed(6)
    dP = torch.randn(3 * n, generator=g, device=dev) * 0.05
    dU = torch.randn(3 * n, generator=g, device=dev) * 0.001
    out = {}
    grads = {}
    for precision in ("fp32", "fp64"):
        with Plan(shape, (params.dx, params.dy, params.dz), params.nPhase, 3, precision=precision, device=device) as plan:
            plan.set_crystal(crystal)
            dt = plan.torch_dtype
            base = dict(inputs, P=inputs["P"].to(dt), U=inputs["U"].to(dt))
            target = plan.run_device(base).clone() if precision == "fp32" else grads["target"]
            grads["target"] = target
            P0 = (inputs["P"].reshape(-1) + dP).to(dt).view((3,) + shape)
            U0 = (inputs["U"].reshape(-1) + dU).to(dt).view((3,) + shape)

            def step():
                P = P0.clone().requires_grad_(True)
                U = U0.clone().requires_grad_(True)
                I = autograd.intensity(plan, P, U, phase=base["phase"], weight=base["weight"])
                loss = ((torch.log10(I) - torch.log10(target)) ** 2).sum()
                loss.backward()
                return loss, P.grad, U.grad

            for _ in range(3):
                step()
            k = steps if precision == "fp32" else 3
            plan.enable_timing(True)
            torch.cuda.synchronize(dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(k):
                loss, gP, gU = step()
            b.record()
            torch.cuda.synchronize(dev)
            plan.device_status()
            st = plan.stage_times()
            plan.enable_timing(False)
            grads[precision] = (gP.double(), gU.double())
            out[precision] = {"ms_per_step": a.elapsed_time(b) / k, "steps": k, "loss": loss.item(),
                              "adjoint_ms": sum(st[kk][0] for kk in st if kk.startswith("adj")) / k,
                              "kernels_ms": {kk: v[0] / k for kk, v in st.items()}}
    (p32, u32), (p64, u64) = grads["fp32"], grads["fp64"]
    rel = lambda x, y: ((x - y).abs().max() / y.abs().max()).item()
    cos = lambda x, y: ((x * y).sum() / (x.norm() * y.norm())).item()
    out.update({"grid": list(shape), "cells": n, "texture": "vortex (seed 5), G=103",
                "fp32_vs_fp64_grad": {"dP_max_rel": rel(p32, p64), "dU_max_rel": rel(u32, u64),
                                      "dP_cos": cos(p32, p64), "dU_cos": cos(u32, u64)},
                "step": "forward + log10 loss + backward (hand-written adjoint, forward recomputed per pass)"})
    return out


def main():
    args = parse()
    from qpop_diffraction_b200 import replicas
    rank, world, local = replicas.rank_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    from qpop_diffraction_b200 import Plan, crystal_from, workloads

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.config == 3:
        run_config3(args, torch, dev, rank, world)
        return
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    shape = tuple(args.grid)
    params, oPhase, oStruc, u, region = workloads.config2_snapshot(seed=2 + rank, shape=shape)
    n = params.n
    spacing = (params.dx, params.dy, params.dz)
    crystals = [crystal_from(params, workloads.config2_crystal(2, h)) for h in REFLECTIONS]
    g1, g2 = atom_groups(crystals[0].R)

    def plans_for(precision, schedule):
        ps = []
        for c in crystals:
            p = Plan(shape, spacing, 2, 3, precision=precision, schedule=schedule, device=local)
            p.set_crystal(c)
            ps.append(p)
        return ps

    host = {k: torch.from_numpy(a) for k, a in (("oPhase", oPhase), ("oStruc", oStruc), ("u", u), ("region", region))}
    d64 = {k: t.to(dev) for k, t in host.items()}

    # ---------------- value: device-resident inputs ----------------
    plans = plans_for("fp32", "fused")
    packed = plans[0].pack(d64["oPhase"], d64["oStruc"], d64["u"], d64["region"])
    out = torch.empty(shape, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(ps, inputs, i):
        ps[i % 2].run_device(inputs, out)

    for i in range(args.warmup):
        step(plans, packed, i)
    torch.cuda.synchronize(dev)
    for p in plans:
        p.stage_times()
        p.enable_timing(True)
    launches0 = sum(p.launches for p in plans)
    smi_id = getattr(torch.cuda.get_device_properties(dev), "uuid", None)
    smi_id = f"GPU-{smi_id}" if smi_id is not None else str(local)
    with Clocks(smi_id) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            step(plans, packed, i)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = sum(p.launches for p in plans) - launches0
    stage = {}
    for p in plans:
        for k, (t, c) in p.stage_times().items():
            s = stage.setdefault(k, [0.0, 0])
            s[0] += t
            s[1] += c
        p.enable_timing(False)
    ms = replicas.slowest(ms, dev)
    value = replicas.throughput(args.steps * n, ms * 1e-3, world) / 1e9
    I32 = plans[0].run_device(packed).clone()      # G = 002, for the float32-vs-float64 accuracy
    I32_host = I32.cpu().numpy()
    I32_103 = plans[1].run_device(packed).cpu().numpy()

    hbm, hbm_src = peaks()
    weight = packed["weight"] is not None
    kb = kernel_bytes(n, g1, g2, weight)
    per_kernel = {}
    for k, (t, c) in stage.items():
        avg = t / c
        per_kernel[k] = {"launches": c, "avg_ms": avg, "bytes_per_launch": kb.get(k),
                         "gbs": kb[k] / (avg * 1e-3) / 1e9 if k in kb else None}
    dom = max(per_kernel, key=lambda k: stage[k][0])
    traffic = profiled_traffic()
    roof = {"bound": "hbm", "kernel": dom, "achieved": per_kernel[dom]["gbs"], "peak": hbm, "unit": "GB/s",
            "frac": per_kernel[dom]["gbs"] / hbm, "peak_source": f"hbm_gbs of {hbm_src}",
            "traffic": traffic[dom] * n if dom in traffic else None,
            "traffic_source": "committed constant: ncu dram__bytes_read.sum + dram__bytes_write.sum per cell of this "
                              "kernel in profiles/ (a smaller capture of the same kernel), times the cells of one launch"}
    model_bytes = n * 5 * (25 + 144)
    model = {"bytes_per_cell": 5 * (25 + 144), "achieved_gbs": model_bytes / (ms / args.steps * 1e-3) / 1e9,
             "frac": model_bytes / (ms / args.steps * 1e-3) / 1e9 / hbm}

    # ---------------- e2e: the C-ABI call with host buffers ----------------
    ke = args.e2e_steps if args.e2e_steps is not None else min(args.steps, 20)
    e2e = None
    if ke > 0:
        pinned = {k: t.pin_memory() for k, t in host.items()}
        pin_np = {k: t.numpy() for k, t in pinned.items()}
        I_host = torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
        plans[0].run_host(pin_np["oPhase"], pin_np["oStruc"], pin_np["u"], pin_np["region"], out=I_host)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for i in range(ke):
            plans[i % 2].run_host(pin_np["oPhase"], pin_np["oStruc"], pin_np["u"], pin_np["region"], out=I_host)
        e2e_s = replicas.slowest(time.perf_counter() - t0, dev)
        h2d = sum(a.nbytes for a in pin_np.values())
        e2e = {"value": replicas.throughput(ke * n, e2e_s, world) / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": I_host.nbytes, "steps": ke, "ms_per_step": e2e_s / ke * 1e3,
               "call": "qpd_run_host (float64 host arrays, pinned)",
               "route": "host workers pack 80% of the 2M-cell chunks to 25 B/cell in a pinned ring while the rest "
                        "cross as float64 and are packed on the GPU; h2d_bytes_per_step counts the float64 inputs"}
    for p in plans:
        p.close()
    del packed

    # ---------------- float64: the same kernels, fused and plain ----------------
    fp64 = None
    accuracy = None
    if not args.no_fp64:
        fp64 = {}
        for schedule, k in (("fused", min(args.steps, 10)), ("plain", min(args.steps, 3))):
            ps = plans_for("fp64", schedule)
            pk = ps[0].pack(d64["oPhase"], d64["oStruc"], d64["u"], d64["region"])
            for i in range(2):
                step(ps, pk, i)
            torch.cuda.synchronize(dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for i in range(k):
                step(ps, pk, i)
            b.record(stream)
            torch.cuda.synchronize(dev)
            t = a.elapsed_time(b) / k
            fp64[schedule] = {"value": n / (t * 1e-3) / 1e9, "ms_per_step": t, "steps": k}
            if schedule == "plain":
                I64 = ps[0].run_device(pk)
                accuracy = {"vs_fp64_plain": dict(intensity_errors(I32_host, I64.cpu().numpy()),
                                                  against="float64 plain schedule of the same kernels (the "
                                                          "reference's per-atom loop), G=002, full grid")}
                del I64
            for p in ps:
                p.close()
            del pk
        for v in fp64.values():
            v["fp32_speedup"] = v["ms_per_step"] / (ms / args.steps)

    del I32
    # ---------------- differentiation: forward + backward at 256 x 256 x 64 ----------------
    adjoint = None
    if not args.no_adjoint:
        torch.cuda.empty_cache()
        adjoint = adjoint_leg(args, torch, local)

    # ---------------- serving: Poisson mix of grids over resident snapshots ----------------
    serving = None
    if not args.no_serving:
        del d64
        torch.cuda.empty_cache()
        serving = serving_leg(args, torch, local)

    # ---------------- float32 against the float64 oracle, per workload ----------------
    if rank == 0 and world == 1 and not args.no_accuracy:
        torch.cuda.empty_cache()
        accuracy = accuracy or {}
        accuracy["per_workload"] = accuracy_leg(torch, dev, (params, (oPhase, oStruc, u, region), I32_103))
    del I32_103

    # ---------------- 4000 x 4000 x 68 on one GPU ----------------
    config3 = None
    if world == 1 and not args.no_config3:
        torch.cuda.empty_cache()
        config3 = config3_leg(args, torch, dev, rank, world, e2e=False)  # e2e from host arrays: bench.py --config 3

    # ---------------- CPU baseline: the reference itself on the full grid ----------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from qpop_diffraction_b200.diffraction import q_axes
        diffraction = reference_diffraction()
        kind = "reference"
        if diffraction is None:  # no install and no checkout: the oracle port, the same algorithm restated
            from oracle import diffraction_oracle as oracle
            diffraction, kind = oracle.diffraction, "port"
        atoms = workloads.config2_crystal(2, REFLECTIONS[0])
        t = time.perf_counter()
        Iref, qx, qy, qz = diffraction(params, atoms, oPhase, oStruc, u, region)
        dt = time.perf_counter() - t
        who = ("the reference's own diffraction() (baseline/_ref, unmodified, NumPy as installed)" if kind == "reference"
               else "the oracle port of the reference's diffraction() (NumPy)")
        cpu = {"value": n / dt / 1e9, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
               "sample": f"{who} on the full {'x'.join(map(str, shape))} config-2 grid, G=002, one run of "
                         f"{dt:.1f} s; host {host_cpu()}"}
        ours = q_axes(params, crystals[0].qC)
        accuracy = accuracy or {}
        accuracy["vs_reference"] = dict(intensity_errors(I32_host, Iref),
                                        against=f"{who}, G=002, full grid (float64)",
                                        q_axes_bit_exact=all(np.array_equal(a, b) for a, b in zip(ours, (qx, qy, qz))))
        del Iref

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded config-2 snapshot)",
            "config": {"workload": f"two-phase polar-vortex film {'x'.join(map(str, shape))}, 5 atoms, 2 phases, "
                                   f"G=002,103 alternating", "grid": list(shape), "cells": n, "atoms": 5, "phases": 2,
                       "precision": "fp32 fields, fp64 phase reduction, fp64 intensity", "schedule": "fused",
                       "l2": "no flush: every step reads and writes about 4 GB, far above the 126 MB L2",
                       "parallelism": f"replicas x{world}"},
            "roofline": roof, "model_roofline": model, "kernels": per_kernel, "gpu_launches": launches,
            "e2e": e2e, "fp64": fp64, "accuracy": accuracy, "adjoint": adjoint, "serving": serving, "config3": config3,
            "cpu_baseline": cpu, "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
