"""
The drop-in behind the reference's own CLI module: ``qpop_diffraction_b200.diffraction.install``
rebinds the name ``diffraction`` that src/python/cli.py:51 imports, so the compute call of
``cli.main`` (src/python/cli.py:221) runs on the GPU.  The reference package comes from the
offline install under baseline/_ref or a source checkout (tests/reference_pkg.py).  cli.py imports
h5py at module level; where h5py is absent, an empty stand-in module is registered for the import
only (nothing here opens a file through it).  Where h5py is installed, the result file written by
qpop_diffraction_b200.hdf5 is also read back with it (src/python/io_utils.py:95-141 layout).
"""

import sys
import types

import numpy as np
import pytest

import reference_pkg


@pytest.fixture
def cli(monkeypatch):
    if reference_pkg.package_dir() is None:
        pytest.skip("the reference package is not available (baseline/_ref or a source checkout)")
    try:
        import h5py  # noqa: F401
    except ImportError:
        monkeypatch.setitem(sys.modules, "h5py", types.ModuleType("h5py"))
    (mod,) = reference_pkg.load("cli")
    original = mod.diffraction
    yield mod
    mod.diffraction = original


def test_install_rebinds_the_cli_compute_call(cli):
    import qpop_diffraction_b200
    from qpop_diffraction_b200.diffraction import install

    assert cli.diffraction is not qpop_diffraction_b200.diffraction
    assert install(cli) is cli
    assert cli.diffraction is qpop_diffraction_b200.diffraction
    # the reference's own q-axis helpers stay in place: the drop-in returns the same axes
    assert callable(cli.q_axes) and callable(cli.reciprocal_centre)


@pytest.mark.gpu
def test_cli_compute_call_runs_on_the_gpu(gpu, cli):
    """A golden case through cli.diffraction after install(): the reference's q axes bit for bit and
    the float32 contract against the reference's own intensity stored in the fixture."""
    from conftest import fp32_errors, load_golden
    from qpop_diffraction_b200.diffraction import install

    install(cli)
    case, ref = load_golden("random_24x16x10_dense")
    I, qx, qy, qz = cli.diffraction(*case.args())
    for got, want in zip((qx, qy, qz), (ref.qx, ref.qy, ref.qz)):
        assert np.array_equal(got, want)
    dmax, rel = fp32_errors(I, ref.I)
    assert dmax <= 1e-5 and rel <= 1e-3, (dmax, rel)


def test_result_file_opens_in_h5py(tmp_path):
    h5py = pytest.importorskip("h5py")
    if not hasattr(h5py, "File"):
        pytest.skip("only a stand-in h5py module is present")
    from qpop_diffraction_b200 import hdf5

    rng = np.random.default_rng(3)
    I = rng.random((5, 4, 3))
    q = [np.linspace(-1, 1, n) for n in I.shape]
    base = tmp_path / "out"
    hdf5.write_diffraction_output(str(base), I, *q, 7)
    with h5py.File(f"{base}.h5", "r") as f:
        assert np.array_equal(f["intensity"][...], I.transpose(2, 1, 0))
        for name, axis in zip(("q_x", "q_y", "q_z"), q):
            assert np.array_equal(f[name][...], axis)
        assert int(f.attrs["Timestep"]) == 7
