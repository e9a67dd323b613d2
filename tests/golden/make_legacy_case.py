"""
Golden case from a real FerroDyn example of the reference: the disordered polar vortex
(examples/4_polar_vortex_PbTiO3/disordered, 1 x 400 x 400 cells, float32 gzip+shuffle HDF5 inputs).

The example also ships reference_legacy.h5, the intensity of a legacy-format run
(tests/test_examples.py:40-46 compares against it).  The reference's current diffraction() does
not reproduce it on these inputs: the ratio varies over about six orders of magnitude across the
voxels above 1e-8 of the maximum, so it is recorded here (legacy_ratio_*) but cannot pin parity.
The pin is the reference's own diffraction() result on the same arguments.

This script builds the arguments the reference CLI passes to diffraction() for that example,
restating src/python/cli.py:153-221 with the reference's own SizeContext and AtomList (imported
from the reference through a package shim, as make_golden.py does) and reading the HDF5 inputs
with qpop_diffraction_b200.hdf5.  It stores them, the legacy intensity and the reference's own
diffraction() result in tests/golden/polar_vortex_example.npz.

    python tests/golden/make_legacy_case.py [/path/to/reference]   (default: QPOP_REFERENCE_ROOT, else ../reference)
"""

import sys
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import reference_pkg  # noqa: E402

from qpop_diffraction_b200 import hdf5  # noqa: E402

HERE = Path(__file__).resolve().parent
CASE = Path("examples/4_polar_vortex_PbTiO3/disordered")


def load_reference(ref_root):
    import os
    os.environ["QPOP_DIFFRACTION_DEVICE"] = "cpu"
    pkg = types.ModuleType("qpop_diffraction")
    pkg.__path__ = [str(Path(ref_root) / "src" / "python")]
    sys.modules["qpop_diffraction"] = pkg
    from qpop_diffraction.atom_list import AtomList
    from qpop_diffraction.diffraction import diffraction
    from qpop_diffraction.size_context import SizeContext
    return SizeContext, AtomList, diffraction


def field(path, name):
    """A FerroDyn (nz, ny, nx) dataset in (x, y, z) order, float64 (src/python/io_utils.py:30-40)."""
    return np.asarray(hdf5.read_dataset(path, name), dtype=np.float64).transpose(2, 1, 0)


def main():
    ref_root = Path(sys.argv[1]) if len(sys.argv) > 1 else reference_pkg.source_root()
    if ref_root is None:
        sys.exit("give the reference's source checkout as the argument or in QPOP_REFERENCE_ROOT")
    SizeContext, AtomList, diffraction = load_reference(ref_root)
    case = ref_root / CASE
    params = SizeContext()
    fe_ids = params.read_json(case / "system_setting.json")
    full = (params.nx, params.ny, params.nz)
    dz = params.lz / params.nz
    atoms = AtomList()
    assert atoms.read(str(case / "parameter.atom.in"), params.nPhase, params.nStruc) and atoms.setup()
    P = np.stack([field(case / "data/P_Lattice_0.h5", f"P_Lattice_{c}") for c in "xyz"])
    step = int(hdf5.read_attrs(case / "data/P_Lattice_0.h5")["Timestep"])
    mat = field(case / "data/materialField_0.h5", "materialField").astype(int)
    region_file = field(case / "data/region.h5", "region")
    oPhase = np.stack([mat == m for m in fe_ids]).astype(np.float64)
    region = oPhase.sum(axis=0).ravel() * region_file.ravel()
    dc_table = params.reference_strain(np.diag(atoms.aC), params.temperature(step))
    dc = dc_table[mat]
    uz_ref = ((np.cumsum(dc, axis=2) - 0.5 * dc) * dz).ravel()
    params.apply_slice(None, None, None)
    params.setup()
    n = params.n
    u = np.zeros(3 * n)
    u[2 * n:] += uz_ref
    oStruc = P.ravel()
    I, qx, qy, qz = diffraction(params, atoms, oPhase.ravel(), oStruc, u, region)
    legacy = np.asarray(hdf5.read_dataset(case / "reference_legacy.h5", "intensity"), dtype=np.float64)
    legacy = legacy.transpose(2, 1, 0)
    strong = legacy > 1e-8 * legacy.max()
    ratio = I[strong] / legacy[strong]
    np.savez_compressed(
        HERE / "polar_vortex_example.npz",
        shape=np.array(full), spacing=np.array([params.dx, params.dy, params.dz]), nPhase=params.nPhase,
        nStruc=params.nStruc, strainAvg=params.strainAvg, aC=atoms.aC, q00=atoms.q00, xAtom=atoms.xAtom,
        fAtom=atoms.fAtom, su=np.stack([atoms.su1, atoms.su2, atoms.su3]),
        P=P.astype(np.float32), region=region.astype(np.float32), mat=mat.astype(np.int8), fe_ids=np.array(fe_ids),
        uz_ref=uz_ref, dc=np.asarray(dc_table, dtype=np.float64), ramp_dz=dz, I=I, qx=qx, qy=qy, qz=qz, legacy_strong_voxels=int(strong.sum()),
        legacy_ratio_min=ratio.min(), legacy_ratio_max=ratio.max(),
    )
    print(f"reference diffraction() / reference_legacy.h5 on {strong.sum()} strong voxels: "
          f"{ratio.min():.3e} .. {ratio.max():.3e}")


if __name__ == "__main__":
    main()
