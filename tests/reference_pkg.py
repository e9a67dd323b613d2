"""
The reference's Python package (qpop_diffraction), loaded for tests, fixture scripts and the
reference arm of bench.py: test infrastructure, never imported by qpop_diffraction_b200.

Two places can hold it: the offline install under baseline/_ref (``pip install --target
baseline/_ref`` of the reference, which travels with the repository), or a source checkout: the
directory named by the environment variable QPOP_REFERENCE_ROOT, else a directory ``reference``
beside the repository (its package directory is src/python; the examples are under examples/).  The
package cannot be imported whole without h5py: its ``__init__`` (src/python/__init__.py:10) imports
io_utils, which imports h5py (src/python/io_utils.py:10).  So an empty package object is registered
under the reference's name with the package directory as ``__path__``, and modules are imported
from it one by one; QPOP_DIFFRACTION_DEVICE=cpu selects its NumPy path (src/python/diffraction.py:24-33).
"""

from __future__ import annotations

import importlib
import os
import sys
import types
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
INSTALLED = ROOT / "baseline" / "_ref" / "qpop_diffraction"


def source_root():
    """The reference's source checkout (QPOP_REFERENCE_ROOT, else ../reference beside the repository), or None."""
    env = os.environ.get("QPOP_REFERENCE_ROOT")
    cand = Path(env) if env else ROOT.parent / "reference"
    return cand if (cand / "src" / "python").is_dir() else None


def package_dir():
    """The directory of the reference's qpop_diffraction package, or None when neither place has it."""
    if (INSTALLED / "diffraction.py").exists():
        return INSTALLED
    root = source_root()
    if root is not None and (root / "src" / "python" / "diffraction.py").exists():
        return root / "src" / "python"
    return None


def load(*modules, path=None):
    """
    Import qpop_diffraction.<m> for each name in modules through the package shim (package
    directory `path`, default package_dir()) and return the modules; None when it is unavailable.
    """
    d = Path(path) if path is not None else package_dir()
    if d is None:
        return None
    os.environ["QPOP_DIFFRACTION_DEVICE"] = "cpu"
    pkg = sys.modules.get("qpop_diffraction")
    if pkg is None or list(getattr(pkg, "__path__", [])) != [str(d)]:
        for name in [k for k in sys.modules if k == "qpop_diffraction" or k.startswith("qpop_diffraction.")]:
            del sys.modules[name]
        pkg = types.ModuleType("qpop_diffraction")
        pkg.__path__ = [str(d)]
        sys.modules["qpop_diffraction"] = pkg
    return [importlib.import_module(f"qpop_diffraction.{m}") for m in modules]
