"""
The single-GPU consumer of <out>_params.h5 (qpop_diffraction_b200.params_runner), the drop-in for
the reference's qpop_diffraction_mgpu program (src/heffte/qpop_diffraction_mgpu.cu).

The parameter file and the FerroDyn fields are written here the way the reference writes them
(src/python/io_utils.py:144-183, chunked shuffle + gzip float32 fields), with this package's HDF5
writer since h5py is absent.  CPU tests cover reading and cropping; the GPU tests run the file and
compare the written /intensity with the oracle on the same fields.
"""

import math

import numpy as np
import pytest

from oracle import diffraction_oracle as oracle
from oracle import fields_oracle
from qpop_diffraction_b200 import hdf5, params_runner, workloads
from qpop_diffraction_b200.plan import reciprocal_centre

L0 = 1e-9


def write_run(tmp, *, full=(20, 18, 40), crop=(2, 17, 1, 16, 8, 31), seed=3, phase_file=False, skeleton=True,
              field_dtype=np.float32, nStruc=3):
    """A FerroDyn-style run directory and the <out>_params.h5 that qpop-diffraction --mgpu would write."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = full
    opts = {"chunks": (max(1, nz // 4), ny, nx), "shuffle": True, "gzip": 4}
    data = tmp / "data"
    data.mkdir(exist_ok=True)
    f = lambda s: rng.standard_normal((nz, ny, nx)).astype(field_dtype) * field_dtype(s)
    P = [f(0.4) for _ in range(3)]
    hdf5.write_file(data / "P_Lattice_1200.h5", {f"P_Lattice_{c}": (P[i], opts) for i, c in enumerate("xyz")},
                    attrs={"Timestep": np.int64(1200)})
    u = [f(1e-11) for _ in range(3)]
    hdf5.write_file(data / "Displacement_1200.h5", {f"Displacement_{c}": (u[i], opts) for i, c in enumerate("xyz")})
    mat = np.where(np.arange(nz)[:, None, None] < 12, 0, 2) * np.ones((1, ny, nx), dtype=np.int8)
    mat[rng.random(mat.shape) < 0.05] = 1
    mat = mat.astype(np.int8)
    hdf5.write_file(data / "materialField_0.h5", {"materialField": (mat, opts)})
    region = rng.random((nz, ny, nx)).astype(np.float32)
    hdf5.write_file(data / "region.h5", {"region": (region, opts)})
    phase = None
    if phase_file:
        a = rng.random((nz, ny, nx)).astype(np.float32)
        phase = [a, (1 - a).astype(np.float32)]
        hdf5.write_file(data / "phase.h5", {f"phase_{p + 1}": (phase[p], opts) for p in range(2)})
    # crystal: two FE phases (materials 0 and 2), material 1 is air
    case = workloads.random_case((4, 4, 4), seed=seed, nPhase=2, weights="onehot", strain=True, hkl=(1, 0, 3))
    atoms = case.atoms
    spacing = np.array([0.4, 0.4, 0.41])
    strain = np.array([0.003, 0.003, 0, 0, 0, 0])
    G, qC = reciprocal_centre(atoms.aC, atoms.q00, strain)
    su = np.stack([atoms.su1, atoms.su2, atoms.su3])[:, :nStruc]
    out = tmp / "diffraction.h5"
    shape = tuple(crop[2 * d + 1] - crop[2 * d] + 1 for d in range(3))
    if skeleton:   # write_diffraction_axes: q axes and attributes, no /intensity
        qx, qy, qz = params_runner.q_axes(shape, spacing, qC)
        hdf5.write_file(out, {"q_x": qx, "q_y": qy, "q_z": qz}, attrs={"Timestep": np.int64(1200), "q_units": "nm^-1"})
    phase_of = np.array([0, -1, 1], dtype=np.int32)
    dc = np.array([-0.0121, 0.0, 0.0187])
    attrs = {"platt_file": str(data / "P_Lattice_1200.h5"), "platt_prefix": "P_Lattice",
             "displacement_file": str(data / "Displacement_1200.h5"),
             "material_file": str(data / "materialField_0.h5"), "region_file": str(data / "region.h5"),
             "output_file": str(out)}
    if phase_file:
        attrs["phase_file"] = str(data / "phase.h5")
    params = tmp / "diffraction_params.h5"
    hdf5.write_file(params, {
        "grid": np.array(full, dtype=np.int64), "crop": np.array(crop, dtype=np.int64),
        "spacing": spacing, "G": G, "qC": qC, "V": np.array([np.linalg.det(atoms.aC)]),
        "R": atoms.xAtom @ atoms.aC, "fAtom_re": np.ascontiguousarray(atoms.fAtom.real),
        "fAtom_im": np.ascontiguousarray(atoms.fAtom.imag), "su": su, "phase_of": phase_of, "dc": dc,
        "u_scale": np.array([1.0 / L0])}, attrs=attrs)
    x0, x1, y0, y1, z0, z1 = crop
    cut = (slice(z0, z1 + 1), slice(y0, y1 + 1), slice(x0, x1 + 1))
    fields = dict(P=np.stack([p[cut] for p in P]), u=np.stack([c[cut] for c in u]), mat=mat[:, cut[1], cut[2]],
                  region=region[cut], phase=None if phase is None else np.stack([a[cut] for a in phase]), z0=z0,
                  dc=dc, phase_of=phase_of, ramp_dz=spacing[2], u_scale=1.0 / L0)
    params_ns = workloads.make_params(shape, spacing, 2, strain)
    return params, out, fields, params_ns, atoms


def expected(fields, params_ns, atoms):
    args = fields_oracle.prepare(fields["P"], fields["mat"], fields["dc"], fields["phase_of"], fields["ramp_dz"],
                                 z0=fields["z0"], u=fields["u"], phase=fields["phase"], region=fields["region"],
                                 u_scale=fields["u_scale"])
    return oracle.diffraction(params_ns, atoms, *args)


def test_read_params_and_crop(tmp_path):
    params, out, fields, params_ns, atoms = write_run(tmp_path, phase_file=True)
    prm = params_runner.read_params(params)
    assert prm.full == (20, 18, 40) and prm.shape == (16, 16, 24) and prm.nPhase == 2 and prm.nAtom == atoms.nAtom
    assert prm.output_file == str(out) and prm.platt_prefix == "P_Lattice"
    assert np.array_equal(prm.fAtom, atoms.fAtom) and prm.u_scale == 1.0 / L0
    f = params_runner.load_fields(prm)
    assert np.array_equal(f.P, fields["P"]) and np.array_equal(f.u, fields["u"])
    assert np.array_equal(f.material, fields["mat"]) and f.material.shape == (40, 16, 16)
    assert np.array_equal(f.phase, fields["phase"]) and np.array_equal(f.region, fields["region"])
    assert f.z0 == 8


def test_q_axes_are_the_reference_expression():
    qC = np.array([0.1, -0.2, 15.3])
    qx, qy, qz = params_runner.q_axes((5, 6, 7), (0.4, 0.4, 0.41), qC)
    assert np.array_equal(qz, np.fft.fftshift(2 * math.pi * np.fft.fftfreq(7, 0.41)) + qC[2])
    assert len(qx) == 5 and len(qy) == 6


@pytest.mark.parametrize("what", ["nstruc", "crop", "float64", "material"])
def test_bad_inputs_are_value_errors(tmp_path, what):
    kw = {"nstruc": dict(nStruc=2), "crop": dict(crop=(2, 20, 1, 16, 8, 31)),
          "float64": dict(field_dtype=np.float64), "material": {}}[what]
    params, *_ = write_run(tmp_path, **kw)
    if what == "material":
        mat = hdf5.read_dataset(tmp_path / "data/materialField_0.h5", "materialField")
        mat[0, 1, 2] = 7                        # layer 0 of a column inside the crop
        hdf5.write_file(tmp_path / "data/materialField_0.h5", {"materialField": mat})
    with pytest.raises(ValueError):
        params_runner.load_fields(params_runner.read_params(params))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,phase_file", [("fp64", False), ("fp32", False), ("fp64", True)])
def test_runs_a_params_file_like_the_native_program(gpu, tmp_path, precision, phase_file):
    params, out, fields, params_ns, atoms = write_run(tmp_path, phase_file=phase_file)
    skeleton_q = [hdf5.read_dataset(out, f"q_{c}") for c in "xyz"]
    I = params_runner.run(params, precision=precision, verbose=False)
    got, qx, qy, qz, attrs = hdf5.load_diffraction_output(out)
    assert np.array_equal(got, I) and attrs["Timestep"] == 1200 and attrs["q_units"] == "nm^-1"
    for a, b in zip((qx, qy, qz), skeleton_q):
        assert np.array_equal(a, b)
    assert (tmp_path / "diffraction.xdmf").exists()
    ref, rqx, rqy, rqz = expected(fields, params_ns, atoms)
    for a, b in zip((qx, qy, qz), (rqx, rqy, rqz)):
        np.testing.assert_allclose(a, b, rtol=1e-15, atol=0)
    if precision == "fp64":
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-12 * ref.max())
    else:
        from conftest import fp32_errors
        dmax, rel = fp32_errors(got, ref)
        assert dmax <= 1e-5 and rel <= 1e-3, (dmax, rel)


@pytest.mark.gpu
def test_without_a_skeleton_the_runner_writes_the_axes(gpu, tmp_path):
    params, out, fields, params_ns, atoms = write_run(tmp_path, skeleton=False)
    params_runner.run(params, precision="fp64", verbose=False)
    got, qx, qy, qz, attrs = hdf5.load_diffraction_output(out)
    ref, rqx, rqy, rqz = expected(fields, params_ns, atoms)
    assert attrs["Timestep"] == 1200
    for a, b in zip((qx, qy, qz), (rqx, rqy, rqz)):
        np.testing.assert_allclose(a, b, rtol=1e-15, atol=0)
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-12 * ref.max())
