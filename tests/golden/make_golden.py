"""
Generate the golden fixtures of tests/golden/ by running the reference's own
standard-build ``diffraction()`` (src/python/diffraction.py:62-113) on seeded
inputs from ``qpop_diffraction_b200.workloads``.

The reference package cannot be imported whole here: its ``__init__``
(src/python/__init__.py:10) pulls in io_utils, which needs h5py.  So an empty
package object is registered under the reference's name with its source
directory as ``__path__``, and only ``diffraction`` is imported from it, on the
CPU (QPOP_DIFFRACTION_DEVICE=cpu, as src/python/diffraction.py:24-33 reads it).

Run from the repository root, in a container where the reference is mounted:

    python tests/golden/make_golden.py [/path/to/reference]   (default: QPOP_REFERENCE_ROOT, else ../reference)

Each fixture ``<name>.npz`` holds the grid, the crystal, the inputs (float32
values; or, for the larger config-1 case, SHA-256 digests of the regenerated
inputs) and the reference's outputs I, qx, qy, qz.
"""

import hashlib
import os
import sys
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import reference_pkg  # noqa: E402

from qpop_diffraction_b200 import workloads  # noqa: E402

HERE = Path(__file__).resolve().parent


def load_reference(ref_root):
    os.environ["QPOP_DIFFRACTION_DEVICE"] = "cpu"
    pkg = types.ModuleType("qpop_diffraction")
    pkg.__path__ = [str(Path(ref_root) / "src" / "python")]
    sys.modules["qpop_diffraction"] = pkg
    from qpop_diffraction.diffraction import diffraction
    return diffraction


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def cases():
    yield workloads.config1(seed=1), False
    yield workloads.random_case((24, 16, 10), seed=11, nPhase=2, weights="dense", strain=True, hkl=(1, 0, 3)), True
    yield workloads.random_case((15, 13, 7), seed=12, nPhase=1, weights="region", hkl=(1, 1, 1)), True
    yield workloads.random_case((1, 40, 30), seed=13, nPhase=1, weights="onehot", hkl=(0, 1, 2)), True
    yield workloads.random_case((8, 12, 68), seed=14, nPhase=2, weights="onehot", hkl=(0, 0, 2)), True
    yield workloads.random_case((20, 9, 11), seed=15, nPhase=3, weights="dense", strain=True, hkl=(2, 1, 1),
                                nAtom=3), True
    yield workloads.random_case((37, 3, 23), seed=16, nPhase=1, weights="onehot", hkl=(1, 0, 2)), True
    c = workloads.config2(seed=2, shape=(16, 16, 104), hkl=(1, 0, 3))
    c.name = "config2_crop_16x16x104_103"
    yield c, True


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else reference_pkg.source_root()
    if ref_root is None:
        sys.exit("give the reference's source checkout as the argument or in QPOP_REFERENCE_ROOT")
    diffraction = load_reference(ref_root)
    for case, store_inputs in cases():
        I, qx, qy, qz = diffraction(*case.args())
        a = case.atoms
        out = dict(
            name=case.name, seed=case.seed, shape=np.array(case.shape),
            spacing=np.array([case.params.dx, case.params.dy, case.params.dz]),
            nPhase=case.params.nPhase, nStruc=case.params.nStruc, strainAvg=case.params.strainAvg,
            aC=a.aC, q00=a.q00, xAtom=a.xAtom, fAtom=a.fAtom, su=np.stack([a.su1, a.su2, a.su3]),
            I=I, qx=qx, qy=qy, qz=qz,
        )
        for key in ("oPhase", "oStruc", "u", "region"):
            arr = getattr(case, key)
            if store_inputs:
                assert np.array_equal(arr.astype(np.float32).astype(np.float64), arr)
                out[key] = arr.astype(np.float32)
            else:
                out[key + "_sha256"] = digest(arr)
        np.savez_compressed(HERE / f"{case.name}.npz", **out)
        print(f"{case.name}: shape {case.shape}, I max {I.max():.6e}")


if __name__ == "__main__":
    main()
