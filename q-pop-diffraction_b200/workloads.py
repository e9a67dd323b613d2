"""
Seeded synthetic diffraction inputs with the shapes, sizes and value
distributions of the workloads this library is measured on.

The reference ships no dataset at these sizes (its examples are 2-D and small),
so every input here is generated from a recorded seed with
``numpy.random.default_rng``.  All field values are rounded to float32, so the
float32 and float64 paths see bit-identical inputs.

Every generator returns a :class:`Case` whose members have the exact types the
reference's ``diffraction(params, atoms, oPhase, oStruc, u, region)`` takes
(src/python/diffraction.py:62-74): ``params`` carries the SizeContext fields it
reads, ``atoms`` the AtomList fields (su already in nm per C/m^2, as
AtomList.setup leaves it, src/python/atom_list.py:176-193), and the four arrays
are flat float64 in component-major, (nx, ny, nz) C order.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from types import SimpleNamespace

import numpy as np

# Perovskite ABO3 cell: A at the corner, B at the body centre, O on the three face centres.
PEROVSKITE = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])


@dataclass
class Case:
    name: str
    params: SimpleNamespace
    atoms: SimpleNamespace
    oPhase: np.ndarray
    oStruc: np.ndarray
    u: np.ndarray
    region: np.ndarray
    seed: int

    @property
    def shape(self):
        return (self.params.nx, self.params.ny, self.params.nz)

    def args(self):
        """Positional arguments of diffraction(params, atoms, oPhase, oStruc, u, region)."""
        return self.params, self.atoms, self.oPhase, self.oStruc, self.u, self.region


def make_params(shape, spacing, nPhase, strain_avg=None, nStruc=3):
    """The SizeContext fields diffraction() reads (src/python/size_context.py:161-208)."""
    nx, ny, nz = (int(s) for s in shape)
    return SimpleNamespace(nx=nx, ny=ny, nz=nz, n=nx * ny * nz,
                           dx=float(spacing[0]), dy=float(spacing[1]), dz=float(spacing[2]),
                           nPhase=int(nPhase), nStruc=int(nStruc),
                           strainAvg=np.zeros(6) if strain_avg is None else np.asarray(strain_avg, dtype=np.float64))


def make_atoms(aC, q00, xAtom, fAtom, su):
    """The AtomList fields diffraction() reads; su is (3, nStruc, nPhase, nAtom) in nm per C/m^2."""
    su = np.asarray(su, dtype=np.float64)
    xAtom = np.asarray(xAtom, dtype=np.float64)
    return SimpleNamespace(aC=np.asarray(aC, dtype=np.float64), q00=np.asarray(q00, dtype=np.float64),
                           xAtom=xAtom, nAtom=xAtom.shape[0],
                           fAtom=np.asarray(fAtom, dtype=np.complex128),
                           su1=su[0].copy(), su2=su[1].copy(), su3=su[2].copy())


def q00_for(aC, hkl):
    """The q00 that selects reflection hkl of the lattice aC (nm^-1)."""
    return np.asarray(hkl, dtype=np.float64) @ (2 * math.pi * np.linalg.inv(np.asarray(aC)).T)


def cromer_mann(rng, q_abs, shape):
    """
    Form factors from 4-Gaussian Cromer-Mann sums with seeded coefficients,
    evaluated once at |q| (nm^-1): f = sum_i a_i exp(-b_i s^2) + c, s = |q| / (4 pi)
    in 1/Angstrom, plus a small seeded imaginary (anomalous) part.
    """
    s2 = (q_abs / 10.0 / (4 * math.pi)) ** 2
    a = rng.uniform(0.5, 20.0, size=shape + (4,))
    b = rng.uniform(0.5, 60.0, size=shape + (4,))
    c = rng.uniform(0.0, 5.0, size=shape)
    re = np.sum(a * np.exp(-b * s2), axis=-1) + c
    im = rng.uniform(0.0, 2.0, size=shape)
    return re + 1j * im


def isotropic_shifts(k):
    """su[d, s, p, a] = k[p, a] delta_ds: ionic shift along P, nm per C/m^2."""
    nPhase, nAtom = k.shape
    su = np.zeros((3, 3, nPhase, nAtom))
    for d in range(3):
        su[d, d] = k
    return su


def f32(x):
    """Round to float32 and return float64 (bit-exact float32 values)."""
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def fourier_modes(rng, shape, kmax, amplitude, modes=8):
    """Smooth periodic field: a few random Fourier modes with integer |m| <= kmax, max |value| = amplitude."""
    nx, ny, nz = shape
    i, j, k = np.meshgrid(np.arange(nx) / nx, np.arange(ny) / ny, np.arange(nz) / nz, indexing="ij", sparse=True)
    out = np.zeros(shape)
    for _ in range(modes):
        while True:
            m = rng.integers(-kmax, kmax + 1, size=3)
            if 0 < m @ m <= kmax * kmax:
                break
        out += rng.standard_normal() * np.cos(2 * math.pi * (m[0] * i + m[1] * j + m[2] * k) + rng.uniform(0, 2 * math.pi))
    peak = np.abs(out).max()
    return out * (amplitude / peak) if peak > 0 else out


def config1(seed=1, shape=(64, 64, 32)):
    """
    64x64x32 single-phase tetragonal perovskite, a = 0.39 nm, c = 0.415 nm, one cell per voxel.
    Ionic shift delta_j = k_j P, k_j in U[-0.02, 0.05] nm per C/m^2; Cromer-Mann form factors at |G|.
    P: a1/a2 stripes ((i + j) mod 16 < 8 -> P || x, else || y), |P| = 0.5 C/m^2, plus N(0, 0.02).
    u: random Fourier modes |m| <= 4, amplitude 0.005 nm.  G = (0, 0, 2).
    """
    rng = np.random.default_rng(seed)
    aC = np.diag([0.39, 0.39, 0.415])
    q00 = q00_for(aC, (0, 0, 2))
    nAtom = len(PEROVSKITE)
    fAtom = cromer_mann(rng, np.linalg.norm(q00), (1, nAtom))
    su = isotropic_shifts(rng.uniform(-0.02, 0.05, size=(1, nAtom)))
    atoms = make_atoms(aC, q00, PEROVSKITE, fAtom, su)
    params = make_params(shape, (0.39, 0.39, 0.415), 1)
    nx, ny, nz = shape
    i = np.arange(nx)[:, None, None]
    j = np.arange(ny)[None, :, None]
    a1 = np.broadcast_to(((i + j) % 16) < 8, shape)
    P = np.zeros((3,) + shape)
    P[0] = 0.5 * a1
    P[1] = 0.5 * ~a1
    P += rng.normal(0.0, 0.02, size=P.shape)
    U = np.stack([fourier_modes(rng, shape, 4, 0.005) for _ in range(3)])
    n = params.n
    return Case("config1", params, atoms, np.ones(n), f32(P).ravel(), f32(U).ravel(), np.ones(n), seed)


def config2_crystal(seed=2, hkl=(0, 0, 2)):
    """
    Crystal of the two-phase film: aC = diag(0.39, 0.39, 0.40) nm, perovskite cell; per phase and atom
    Cromer-Mann form factors at |G| and ionic shifts k P with k in U[-0.005, 0.005] (substrate) and
    U[-0.02, 0.05] (film) nm per C/m^2.  Seeded by (seed, hkl): form factors depend on |G|.
    """
    rng = np.random.default_rng([seed] + list(hkl))
    aC = np.diag([0.39, 0.39, 0.40])
    q00 = q00_for(aC, hkl)
    nAtom = len(PEROVSKITE)
    fAtom = cromer_mann(rng, np.linalg.norm(q00), (2, nAtom))
    k = np.stack([rng.uniform(-0.005, 0.005, size=nAtom), rng.uniform(-0.02, 0.05, size=nAtom)])
    return make_atoms(aC, q00, PEROVSKITE, fAtom, isotropic_shifts(k))


def config2_snapshot(seed=2, shape=(512, 512, 104), substrate=24):
    """
    Fields of the two-phase film: SrTiO3-like substrate (phase 1, z < 24) under a PbTiO3-like film
    (phase 2), one-hot phase fractions as a phase_file gives them, region 1.  P in the film is a
    polar-vortex texture rotating in x-z with period 10 cells: psi = sin(2 pi x / 10) sin(2 pi z / 10),
    P = 0.6 (d_z psi, 0, -d_x psi) / |grad psi|, plus N(0, 0.02); the substrate has the noise only.
    u: a substrate-strain gradient growing to 1% at the top of the box, integrated up z at the cell
    centres, plus random Fourier modes of amplitude 0.005 nm.
    Returns (params, oPhase, oStruc, u, region).
    """
    rng = np.random.default_rng(seed)
    params = make_params(shape, (0.39, 0.39, 0.40), 2)
    nx, ny, nz = shape
    z = np.arange(nz)
    film = z >= substrate
    oPhase = np.zeros((2,) + shape, dtype=np.float32)
    oPhase[0, :, :, ~film] = 1.0
    oPhase[1, :, :, film] = 1.0

    x = np.arange(nx)[:, None] * (2 * math.pi / 10)
    zz = z[None, :] * (2 * math.pi / 10)
    dz_psi = np.sin(x) * np.cos(zz)
    dx_psi = np.cos(x) * np.sin(zz)
    norm = np.maximum(np.hypot(dz_psi, dx_psi), 1e-12)
    P = rng.normal(0.0, 0.02, size=(3,) + shape).astype(np.float32)
    P[0] += (0.6 * dz_psi / norm * film[None, :])[:, None, :].astype(np.float32)
    P[2] += (-0.6 * dx_psi / norm * film[None, :])[:, None, :].astype(np.float32)

    strain = 0.01 * z / max(nz - 1, 1)
    uz = (np.cumsum(strain) - 0.5 * strain) * params.dz
    U = np.stack([fourier_modes(rng, shape, 4, 0.005).astype(np.float32) for _ in range(3)])
    U[2] += uz[None, None, :].astype(np.float32)
    return (params, oPhase.astype(np.float64).ravel(), P.astype(np.float64).ravel(), U.astype(np.float64).ravel(),
            np.ones(params.n))


def config2(seed=2, shape=(512, 512, 104), hkl=(0, 0, 2), substrate=24):
    """The two-phase vortex film of config2_snapshot seen at reflection hkl (config2_crystal)."""
    params, oPhase, oStruc, u, region = config2_snapshot(seed, shape, substrate)
    return Case(f"config2_{''.join(map(str, hkl))}", params, config2_crystal(seed, hkl), oPhase, oStruc, u, region,
                seed)


def random_case(shape, seed, nPhase=1, weights="onehot", hkl=(1, 0, 3), strain=False, spacing=None,
                nAtom=None, aC=None):
    """
    A small seeded case for parity tests.

    weights: "onehot" (each cell in one phase or none, region 1), "region" (one-hot phases and a
    fractional region weight with zeros), or "dense" (fractional phase fractions that overlap,
    times a fractional region).  strain: a non-zero strainAvg, so qC differs from G.
    """
    rng = np.random.default_rng(seed)
    aC = np.diag([0.4, 0.39, 0.41]) if aC is None else np.asarray(aC)
    xAtom = PEROVSKITE if nAtom is None else rng.integers(0, 4, size=(nAtom, 3)) / 4.0
    nA = xAtom.shape[0]
    q00 = q00_for(aC, hkl)
    fAtom = cromer_mann(rng, np.linalg.norm(q00), (nPhase, nA))
    su = rng.uniform(-0.03, 0.05, size=(3, 3, nPhase, nA))
    atoms = make_atoms(aC, q00, xAtom, fAtom, su)
    strain_avg = rng.uniform(-0.01, 0.01, size=6) if strain else None
    spacing = np.diag(aC) if spacing is None else spacing
    params = make_params(shape, spacing, nPhase, strain_avg)
    n = params.n
    P = rng.normal(0.0, 0.3, size=(3, n))
    U = np.stack([fourier_modes(rng, shape, 3, 0.01).ravel() for _ in range(3)])
    U[2] += (0.01 * np.arange(shape[2]) * spacing[2])[None, None, :].repeat(shape[0], 0).repeat(shape[1], 1).ravel()
    if weights == "dense":
        oPhase = rng.uniform(0.0, 1.0, size=(nPhase, n))
        region = rng.uniform(0.0, 1.0, size=n) * (rng.uniform(size=n) > 0.1)
    else:
        which = rng.integers(-1, nPhase, size=n)
        oPhase = np.stack([(which == p).astype(np.float64) for p in range(nPhase)])
        region = oPhase.sum(axis=0)
        if weights == "region":
            region = region * rng.uniform(0.2, 1.0, size=n)
    return Case(f"random_{'x'.join(map(str, shape))}_{weights}", params, atoms, f32(oPhase).ravel(), f32(P).ravel(),
                f32(U).ravel(), f32(region), seed)


# ---------------------------------------------------------------------------------------------
# Snapshots generated on the GPU, directly in the packed layout the kernels read (float32 P and
# u planes, int8 phase index): the serving mix and the 4000 x 4000 x 68 grid are too large to
# build in NumPy float64 in reasonable time.  Seeded with torch.Generator on the device.
# ---------------------------------------------------------------------------------------------

TEXTURES = ("vortex", "twin", "twophase")


def gpu_snapshot(kind, shape, seed, device="cuda", substrate=None, n_domains=200, spacing=(0.39, 0.39, 0.40),
                 n_phase=2):
    """
    Packed inputs of a seeded film snapshot on the GPU.  Two phases: substrate (phase 0) for
    z < substrate (default a quarter of the box, at most 24 cells), film (phase 1) above.

    kind "vortex":   polar-vortex array rotating in x-z, period 10 cells, |P| = 0.6, plus N(0, 0.02);
                     u = 1% strain gradient up z + small modes (config 2 texture).
    kind "twin":     in-plane Voronoi tessellation of n_domains cells, 3 variants with P along
                     directions 120 degrees apart starting at [110], |P| = 0.5; u_z from a
                     +-0.5% strain per domain (config 3 texture).
    kind "twophase": a1/a2 stripes with period 16 along [110], |P| = 0.5, on the strained substrate.
    n_phase=1: one phase everywhere (no substrate), as in the 4000 x 4000 x 68 twin film.
    Returns (params, inputs) with inputs = {"P", "U", "phase", "weight": None, "wdense": None}.
    """
    import torch

    nx, ny, nz = (int(s) for s in shape)
    n = nx * ny * nz
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    params = make_params(shape, spacing, n_phase)
    if n_phase == 1:
        substrate = 0
    elif substrate is None:
        substrate = min(24, nz // 4)
    f32 = dict(dtype=torch.float32, device=dev)
    x = torch.arange(nx, **f32).view(nx, 1, 1)
    y = torch.arange(ny, **f32).view(1, ny, 1)
    z = torch.arange(nz, **f32).view(1, 1, nz)
    film = (z >= substrate).expand(nx, ny, nz)
    P = torch.empty((3, nx, ny, nz), **f32)
    P.normal_(0.0, 0.02, generator=g)
    if kind == "vortex":
        k = 2 * math.pi / 10
        dz_psi = torch.sin(k * x) * torch.cos(k * z)
        dx_psi = torch.cos(k * x) * torch.sin(k * z)
        norm = torch.clamp(torch.sqrt(dz_psi ** 2 + dx_psi ** 2), min=1e-12)
        P[0] += torch.where(film, (0.6 * dz_psi / norm).expand(nx, ny, nz), 0.0)
        P[2] += torch.where(film, (-0.6 * dx_psi / norm).expand(nx, ny, nz), 0.0)
        strain = 0.01 * z / max(nz - 1, 1)
    elif kind == "twin":
        seeds = torch.rand((n_domains, 2), generator=g, **f32) * torch.tensor([nx, ny], **f32)
        variant = torch.randint(0, 3, (n_domains,), generator=g, device=dev)
        dstrain = (torch.rand(n_domains, generator=g, **f32) * 2 - 1) * 0.005
        # nearest seed per (x, y) column, in row blocks to bound the temporary
        owner = torch.empty((nx, ny), dtype=torch.long, device=dev)
        xs = torch.arange(nx, **f32)
        ys = torch.arange(ny, **f32)
        step = max(1, (1 << 24) // max(1, ny * n_domains))
        for i0 in range(0, nx, step):
            dx = xs[i0:i0 + step].view(-1, 1, 1) - seeds[:, 0].view(1, 1, -1)
            dy = ys.view(1, -1, 1) - seeds[:, 1].view(1, 1, -1)
            owner[i0:i0 + step] = torch.argmin(dx * dx + dy * dy, dim=2)
        ang = math.pi / 4 + variant[owner].to(torch.float32) * (2 * math.pi / 3)
        filmf = film.to(torch.float32)
        P[0] += (0.5 * torch.cos(ang)).unsqueeze(2) * filmf
        P[1] += (0.5 * torch.sin(ang)).unsqueeze(2) * filmf
        strain = dstrain[owner].unsqueeze(2).expand(nx, ny, nz)
    elif kind == "twophase":
        a1 = (((x + y) % 16) < 8).expand(nx, ny, nz)
        P[0] += torch.where(film & a1, 0.5, 0.0)
        P[1] += torch.where(film & ~a1, 0.5, 0.0)
        strain = 0.004 * (z < substrate).to(torch.float32)
    else:
        raise ValueError(f"unknown texture {kind!r}")
    strain = torch.as_tensor(strain, **f32).expand(nx, ny, nz)
    uz = (torch.cumsum(strain, dim=2) - 0.5 * strain) * params.dz
    U = torch.empty((3, nx, ny, nz), **f32)
    U.normal_(0.0, 0.001, generator=g)
    U[2] += uz
    if n_phase == 1:
        phase = torch.zeros(n, dtype=torch.int8, device=dev)
    else:
        phase = film.to(torch.int8).contiguous().view(-1)
    return params, {"P": P.view(-1), "U": U.view(-1), "phase": phase, "weight": None, "wdense": None}


def config3_crystal(seed=3, hkl=(1, 1, 3)):
    """One-phase perovskite of the 4000 x 4000 x 68 twin film: aC = diag(0.39, 0.39, 0.40) nm,
    Cromer-Mann form factors at |G|, ionic shifts k P with k in U[-0.02, 0.05] nm per C/m^2."""
    rng = np.random.default_rng([seed] + list(hkl))
    aC = np.diag([0.39, 0.39, 0.40])
    q00 = q00_for(aC, hkl)
    nAtom = len(PEROVSKITE)
    fAtom = cromer_mann(rng, np.linalg.norm(q00), (1, nAtom))
    return make_atoms(aC, q00, PEROVSKITE, fAtom, isotropic_shifts(rng.uniform(-0.02, 0.05, size=(1, nAtom))))


def serving_crystal(hkl, seed=2):
    """The two-phase perovskite crystal of the serving mix at reflection hkl (config-2 constants)."""
    return config2_crystal(seed, hkl)
