"""
Drop-in for the reference's standard-build compute call.

``diffraction(params, atoms, oPhase, oStruc, u, region) -> (I, qx, qy, qz)`` has the
signature, argument meaning and return values of src/python/diffraction.py:62-113:
float64 host arrays in, the fftshifted float64 intensity (nx, ny, nz) and its 1-D q
axes (nm^-1) out.  The per-cell work runs in libqpopdiff.so on the GPU; G, qC and
the q axes are host float64 exactly as the reference computes them, so the axes
are bit-identical.

``install()`` puts it behind the reference CLI: ``cli.py`` imports the name
``diffraction`` into its own namespace (src/python/cli.py:51), so the binding
there is the one to replace.

Precision and schedule default to ``QPOP_B200_PRECISION`` (fp32 | fp64, default
fp32) and ``QPOP_B200_SCHEDULE`` (fused | plain, default fused), read at call time.
"""

from __future__ import annotations

import math
import os
import sys

import numpy as np

from .plan import Plan, crystal_from, reciprocal_centre as _reciprocal_centre

_plans = {}


def reciprocal_centre(params, atoms):
    """(G, qC) in nm^-1 (src/python/diffraction.py:36-48)."""
    return _reciprocal_centre(atoms.aC, atoms.q00, params.strainAvg)


def wavevectors(params):
    """FFT wavevectors along x, y, z in nm^-1, in FFT order (src/python/diffraction.py:51-54)."""
    shape = (params.nx, params.ny, params.nz)
    return [2 * math.pi * np.fft.fftfreq(m, d) for m, d in zip(shape, (params.dx, params.dy, params.dz))]


def q_axes(params, qC):
    """1-D q axes in nm^-1 of the fftshifted intensity (src/python/diffraction.py:57-59)."""
    return tuple(np.fft.fftshift(kd) + qC[d] for d, kd in enumerate(wavevectors(params)))


def get_plan(shape, spacing, nPhase, nStruc, precision, schedule, device=0):
    """A cached Plan for this grid (workspace kept on the device between calls)."""
    key = (tuple(shape), tuple(spacing), nPhase, nStruc, precision, schedule, device)
    plan = _plans.get(key)
    if plan is None:
        plan = _plans[key] = Plan(shape, spacing, nPhase, nStruc, precision=precision, schedule=schedule,
                                  device=device)
    return plan


def release():
    """Free the device workspace of every cached plan."""
    for plan in _plans.values():
        plan.close()
    _plans.clear()


def diffraction(params, atoms, oPhase, oStruc, u, region, *, precision=None, schedule=None, device=0):
    """
    Args (as src/python/diffraction.py:62-74):
        params: SizeContext after setup() (grid in nm, strainAvg)
        atoms:  AtomList after setup() (aC, q00, xAtom, fAtom; su in nm per C/m^2)
        oPhase: (nPhase * n,) phase fractions
        oStruc: (nStruc * n,) order parameters (P in C/m^2)
        u:      (3 * n,) displacement in nm
        region: (n,) scattering weight

    Returns:
        (I, qx, qy, qz): intensity (nx, ny, nz), fftshifted, and its 1-D q axes in nm^-1
    """
    precision = precision or os.environ.get("QPOP_B200_PRECISION", "fp32").lower()
    schedule = schedule or os.environ.get("QPOP_B200_SCHEDULE", "fused").lower()
    shape = (int(params.nx), int(params.ny), int(params.nz))
    spacing = (float(params.dx), float(params.dy), float(params.dz))
    crystal = crystal_from(params, atoms)
    plan = get_plan(shape, spacing, int(params.nPhase), int(params.nStruc), precision, schedule, device)
    plan.set_crystal(crystal)
    I = plan.run_host(oPhase, oStruc, u, region)
    return (I,) + q_axes(params, crystal.qC)


def install(cli_module=None):
    """
    Route the reference CLI's compute call through this package: rebinds
    ``qpop_diffraction.cli.diffraction`` (imported by name at src/python/cli.py:51)
    and the package-level export (src/python/__init__.py:9).  Returns the CLI module.
    """
    if cli_module is None:
        import importlib
        cli_module = importlib.import_module("qpop_diffraction.cli")
    cli_module.diffraction = diffraction
    pkg = sys.modules.get(cli_module.__name__.rpartition(".")[0])
    if pkg is not None and hasattr(pkg, "diffraction"):
        pkg.diffraction = diffraction
    return cli_module
