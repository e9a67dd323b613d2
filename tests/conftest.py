"""
Test configuration.

``-m gpu`` tests need a CUDA device and the built libqpopdiff.so; everything else
runs on the CPU (oracle pinning, host logic, the C ABI's exports).
"""

import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libqpopdiff.so")


EXAMPLE = "polar_vortex_example"


def golden_names():
    """Fixtures of seeded synthetic inputs (the FerroDyn example has its own loader)."""
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem != EXAMPLE)


def load_example():
    """
    The reference's disordered polar-vortex example (tests/golden/make_legacy_case.py) as FerroDyn
    fields in file order (nz, ny, nx), the per-material tables, the grid and crystal, and the
    reference's own diffraction() result.
    """
    from qpop_diffraction_b200 import workloads

    z = np.load(GOLDEN / f"{EXAMPLE}.npz", allow_pickle=False)
    shape = tuple(int(s) for s in z["shape"])
    fe = [int(m) for m in z["fe_ids"]]
    return SimpleNamespace(
        shape=shape,
        params=workloads.make_params(shape, z["spacing"], int(z["nPhase"]), z["strainAvg"], int(z["nStruc"])),
        atoms=workloads.make_atoms(z["aC"], z["q00"], z["xAtom"], z["fAtom"], z["su"]),
        P=np.ascontiguousarray(z["P"].transpose(0, 3, 2, 1)),
        mat=np.ascontiguousarray(z["mat"].transpose(2, 1, 0)),
        region=np.ascontiguousarray(z["region"].reshape(shape).transpose(2, 1, 0)),
        dc=z["dc"], ramp_dz=float(z["ramp_dz"]),
        phase_of=np.array([fe.index(m) if m in fe else -1 for m in range(len(z["dc"]))], dtype=np.int32),
        uz_ref=z["uz_ref"], I=z["I"], qx=z["qx"], qy=z["qy"], qz=z["qz"])


def load_golden(name):
    """A golden fixture as (case, expected) with the reference's outputs; inputs regenerated when not stored."""
    from qpop_diffraction_b200 import workloads

    z = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    shape = tuple(int(s) for s in z["shape"])
    params = workloads.make_params(shape, z["spacing"], int(z["nPhase"]), z["strainAvg"], int(z["nStruc"]))
    atoms = workloads.make_atoms(z["aC"], z["q00"], z["xAtom"], z["fAtom"], z["su"])
    if "oStruc" in z:
        arrays = {k: z[k].astype(np.float64) for k in ("oPhase", "oStruc", "u", "region")}
    else:
        import hashlib
        gen = {"config1": workloads.config1}[name](seed=int(z["seed"]))
        arrays = {}
        for k in ("oPhase", "oStruc", "u", "region"):
            a = getattr(gen, k)
            assert hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest() == str(z[k + "_sha256"]), \
                f"{name}: regenerated {k} differs from the fixture's inputs"
            arrays[k] = a
    case = workloads.Case(name, params, atoms, arrays["oPhase"], arrays["oStruc"], arrays["u"], arrays["region"],
                          int(z["seed"]))
    expected = SimpleNamespace(I=z["I"], qx=z["qx"], qy=z["qy"], qz=z["qz"])
    return case, expected


def fp32_errors(I, ref):
    """The float32 contract: max |dI| / I_max, and the max relative error on voxels above 1e-6 I_max."""
    imax = ref.max()
    strong = ref > 1e-6 * imax
    return np.abs(I - ref).max() / imax, (np.abs(I - ref)[strong] / ref[strong]).max()


@pytest.fixture(scope="session")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from qpop_diffraction_b200 import _native
    _native.load()
    return torch
