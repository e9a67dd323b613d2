"""
The HDF5 reader and writer (qpop_diffraction_b200.hdf5), which replace h5py for the reference's
FerroDyn inputs and its result file (src/python/io_utils.py:30-141).
"""

import os
import xml.etree.ElementTree as ET
from pathlib import Path

import numpy as np
import pytest

from conftest import load_example
from qpop_diffraction_b200 import hdf5

import reference_pkg

REFERENCE = reference_pkg.source_root()  # the reference's source checkout (QPOP_REFERENCE_ROOT), if any
EXAMPLE = REFERENCE / "examples/4_polar_vortex_PbTiO3/disordered" if REFERENCE else None


def test_contiguous_and_chunked_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    datasets = {
        "P_Lattice_x": (rng.standard_normal((5, 33, 70)).astype(np.float32), {"chunks": (1, 16, 32), "shuffle": True, "gzip": 4}),
        "materialField": (rng.integers(-1, 4, (5, 33, 70)).astype(np.int8), {"chunks": (2, 33, 70), "gzip": 9}),
        "many_chunks": (rng.standard_normal((3, 300, 7)), {"chunks": (1, 2, 7), "shuffle": True}),  # multi-level B-tree
        "grid": np.array([4000, 4000, 68], dtype=np.int64),
        "scalar_like": np.array([2.5]),
    }
    for i in range(12):  # more names than one default symbol-table node holds
        datasets[f"extra_{i:02d}"] = np.full(3, i, dtype=np.int32)
    path = tmp_path / "t.h5"
    hdf5.write_file(path, datasets, attrs={"Timestep": np.int64(7), "platt_prefix": "P_Lattice", "x": 1.5})
    assert hdf5.list_datasets(path) == sorted(datasets)
    for name, v in datasets.items():
        want = v[0] if isinstance(v, tuple) else v
        got = hdf5.read_dataset(path, name)
        assert got.dtype == want.dtype and np.array_equal(got, want), name
    attrs = hdf5.read_attrs(path)
    assert attrs == {"Timestep": 7, "platt_prefix": "P_Lattice", "x": 1.5}


def test_result_file_and_xdmf(tmp_path):
    """write_diffraction_output's contract (src/python/io_utils.py:95-141): /intensity stored (nz, ny, nx)."""
    rng = np.random.default_rng(1)
    I = rng.random((6, 5, 4)) + 1e-50
    qx, qy, qz = (np.linspace(-1, 1, n) for n in I.shape)
    base = str(tmp_path / "out")
    hdf5.write_diffraction_output(base, I, qx, qy, qz, step=1200)
    raw = hdf5.read_dataset(base + ".h5", "intensity")
    assert raw.shape == (4, 5, 6) and np.array_equal(raw, I.transpose(2, 1, 0))
    got, gx, gy, gz, attrs = hdf5.load_diffraction_output(base + ".h5")
    assert np.array_equal(got, I) and all(np.array_equal(a, b) for a, b in ((gx, qx), (gy, qy), (gz, qz)))
    assert attrs == {"Timestep": 1200, "q_units": "nm^-1"}
    root = ET.parse(base + ".xdmf").getroot()
    topo = root.find("./Domain/Grid/Topology")
    assert topo.get("TopologyType") == "3DRectMesh" and topo.get("Dimensions") == "4 5 6"
    items = [e.text for e in root.iter("DataItem")]
    assert items == ["out.h5:/q_x", "out.h5:/q_y", "out.h5:/q_z", "out.h5:/intensity"]


def test_rejects_what_it_cannot_read(tmp_path):
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not an hdf5 file at all")
    with pytest.raises(hdf5.HDF5Error):
        hdf5.read_dataset(bad, "x")
    good = tmp_path / "good.h5"
    hdf5.write_file(good, {"a": np.zeros(3)})
    with pytest.raises(hdf5.HDF5Error):
        hdf5.read_dataset(good, "missing")


@pytest.mark.skipif(EXAMPLE is None or not EXAMPLE.is_dir(), reason="the reference's examples are not mounted")
def test_reads_the_reference_ferrodyn_example():
    """gzip + shuffle float32 and int8 FerroDyn fields, read as the fixture stored them."""
    ex = load_example()
    for c in range(3):
        assert np.array_equal(hdf5.read_dataset(EXAMPLE / "data/P_Lattice_0.h5", f"P_Lattice_{'xyz'[c]}"), ex.P[c])
    assert np.array_equal(hdf5.read_dataset(EXAMPLE / "data/materialField_0.h5", "materialField"), ex.mat)
    assert np.array_equal(hdf5.read_dataset(EXAMPLE / "data/region.h5", "region"), ex.region)
    assert int(hdf5.read_attrs(EXAMPLE / "data/P_Lattice_0.h5")["Timestep"]) == 0
    legacy = hdf5.read_dataset(EXAMPLE / "reference_legacy.h5", "intensity")
    assert legacy.shape == ex.shape[::-1] and legacy.dtype == np.float64


def test_ferrodyn_style_fields_survive_a_round_trip(tmp_path):
    """Fields written the way FerroDyn stores them (chunked, shuffle + gzip) read back bit-exact."""
    ex = load_example()
    path = tmp_path / "P_Lattice_0.h5"
    opts = {"chunks": (ex.P.shape[1], 100, ex.P.shape[3]), "shuffle": True, "gzip": 6}
    hdf5.write_file(path, {f"P_Lattice_{c}": (ex.P[i], opts) for i, c in enumerate("xyz")}, attrs={"Timestep": np.int64(0)})
    for i, c in enumerate("xyz"):
        assert np.array_equal(hdf5.read_dataset(path, f"P_Lattice_{c}"), ex.P[i])
    assert os.path.getsize(path) < ex.P.nbytes
