"""Seeded synthetic scenes: the workloads the step is measured and checked on.

Each builder returns a ``Scene``: the Simulation parameters (MtrParams), the
particle arrays (AoS, include/matter_gpu.h layout) and the plates/objects.
Particles sit on a jittered lattice (``ppc`` sub-points per cell, uniform
jitter of +-0.25 dx), the stand-in for the reference's Poisson-disk sampler
(sampling_particles.hpp:12-123), which needs the absent tph_poisson library.

``scale`` shrinks the block (same dx, same materials) for parity tests.
``perturb`` adds a random velocity field, a random elastic deformation and a
random affine matrix B so that one step exercises every branch of the return
mapping and the boundary conditions.
"""
import math
from dataclasses import dataclass, field

import numpy as np

from .abi import (BC, HardeningLaw, ObjectKind, PlasticModel, PlateType, default_params, make_object,
                  make_plate)


@dataclass
class Scene:
    name: str
    params: object
    x: np.ndarray
    v: np.ndarray = None
    F: np.ndarray = None
    B: np.ndarray = None
    scalars: np.ndarray = None
    plates: list = field(default_factory=list)
    objects: list = field(default_factory=list)
    levelsets: list = field(default_factory=list)  # LevelSetData for ObjectKind.LevelSet objects

    @property
    def Np(self):
        return self.x.shape[0]

    @property
    def dim(self):
        return self.params.dim


@dataclass
class LevelSetData:
    """A dense level set (mtr_set_levelset): phi[i, j, k] at origin + (i, j, k) * spacing."""
    slot: int
    phi: np.ndarray          # float32, shape dims (dims[2] = 1 in 2D)
    origin: tuple
    spacing: float
    normals: np.ndarray = None  # float32 (*dims, 3) or None for the gradient of phi

    @property
    def dims(self):
        return tuple(int(n) for n in self.phi.shape)


def sample_levelset(fn, lo, hi, spacing, dim, slot=0):
    """Samples a signed-distance-like function fn(X) (X: (n, dim) array, negative
    inside) on the lattice covering [lo, hi] at `spacing`."""
    n = [int(math.ceil((hi[a] - lo[a]) / spacing)) + 1 for a in range(dim)]
    axes = [lo[a] + spacing * np.arange(n[a]) for a in range(dim)]
    grid = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, dim)
    phi = np.asarray(fn(grid), dtype=np.float64).astype(np.float32)
    shape = tuple(n) + ((1,) if dim == 2 else ())
    return LevelSetData(slot, phi.reshape(shape), tuple(lo[:dim]) + ((0.0,) if dim == 2 else ()), float(spacing))


def terrain_levelset(obj, dim, lo, hi, spacing, slot=0):
    """phi = y - s(x, z) of a TerrainGauss object: its gradient (-s_x, 1, -s_z)
    points along the analytic terrain normal."""
    prm = list(obj.prm)

    def surf(X):
        ys = np.full(X.shape[0], prm[0])
        for b in range(int(prm[1])):
            xb, zb, hb, sb = prm[2 + 4 * b:6 + 4 * b]
            r2 = (X[:, 0] - xb) ** 2 + ((X[:, 2] - zb) ** 2 if dim == 3 else 0.0)
            ys = ys + hb * np.exp(-r2 / (2 * sb * sb))
        return X[:, 1] - ys

    return sample_levelset(surf, lo, hi, spacing, dim, slot)


def lattice(lo, hi, dx, ppc_axis, rng, jitter=0.25):
    """Jittered lattice: ppc_axis^d sub-points per cell at ((i+0.5)/ppc_axis)*dx."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    d = lo.size
    ncell = np.rint((hi - lo) / dx).astype(np.int64)
    n_axis = ncell * ppc_axis
    h = dx / ppc_axis
    axes = [lo[a] + (np.arange(n_axis[a]) + 0.5) * h for a in range(d)]
    mesh = np.meshgrid(*axes, indexing="ij")
    x = np.stack([m.reshape(-1) for m in mesh], axis=1)
    x += rng.uniform(-jitter * dx, jitter * dx, size=x.shape)
    return x


def _finish(scene, dx, ppc, rho):
    p = scene.params
    p.dx = dx
    p.rho = rho
    p.particle_volume = dx ** p.dim / ppc
    p.particle_mass = rho * p.particle_volume
    return scene


def perturb(scene, seed=7, v_amp=0.5, f_amp=0.02, b_amp=5.0, plastic=True):
    """Random velocities, deformation gradients, affine B and plastic history."""
    rng = np.random.default_rng(seed)
    n, d = scene.Np, scene.dim
    scene.v = rng.uniform(-v_amp, v_amp, size=(n, d))
    F = np.tile(np.eye(d), (n, 1, 1)) + rng.uniform(-f_amp, f_amp, size=(n, d, d))
    scene.F = np.ascontiguousarray(np.transpose(F, (0, 2, 1)))  # store column-major
    scene.B = np.ascontiguousarray(rng.uniform(-b_amp, b_amp, size=(n, d, d)) * scene.params.dx ** 2)
    sc = np.zeros((n, 6))
    if plastic:
        sc[:, 0] = rng.uniform(0, 0.05, n)
        sc[:, 1] = rng.uniform(-0.01, 0.01, n)
        sc[:, 2] = rng.uniform(-0.005, 0.0, n)
        sc[:, 5] = scene.params.M
    scene.scalars = sc
    return scene


def collapse2d(scale=1.0, seed=12345):
    """2D plane-strain granular column collapse (USL, APIC, quadratic B-spline).

    Column 0.2 m x 0.4 m on a SlipFree floor plate with Coulomb mu = 0.5,
    dx = 0.0025 m, 4 particles per cell (51,200 at scale 1), rho 1550, Hencky
    E = 1e6 Pa, nu = 0.3, Drucker-Prager M = tan 30 deg, cohesion 0.
    """
    dx = 0.0025
    W, H = 0.2 * scale, 0.4 * scale
    W, H = max(dx, round(W / dx) * dx), max(dx, round(H / dx) * dx)
    rng = np.random.default_rng(seed)
    x = lattice([0.0, 0.0], [W, H], dx, 2, rng)
    p = default_params(2, 2)
    p.flip_ratio = -2.0  # < -1: APIC (position_update.cpp:17)
    p.plastic_model = PlasticModel.DP
    p.M = math.tan(30.0 * math.pi / 180.0)
    p.q_cohesion = 0.0
    p.E, p.nu = 1e6, 0.3
    p.gravity[1] = -9.81
    p.end_frame, p.fps = 1, 1.0
    sc = Scene("collapse2d_dp_usl_apic_q2", p, x)
    sc.plates = [make_plate(0.0, PlateType.bottom, BC.SlipFree, 0.5)]
    return _finish(sc, dx, 4, 1550.0)


def collapse3d_mui(scale=1.0, seed=2024, musl=True):
    """3D mu(I)-Drucker-Prager column collapse (MUSL, AFLIP, cubic B-spline).

    Box 0.5 x 1.0 x 0.5 m (x, height y, z) on a SlipStick floor with mu = 0.4,
    dx = 0.0125 m, 8 particles per cell (1,024,000 at scale 1), mu_1 = 0.38,
    mu_2 = 0.64, I_0 = 0.279, d = 1 mm, rho_s = 2500, rho = 0.6 rho_s,
    E = 1e7 Pa, nu = 0.3.
    """
    dx = 0.0125
    L = [0.5 * scale, 1.0 * scale, 0.5 * scale]
    L = [max(dx, round(v / dx) * dx) for v in L]
    rng = np.random.default_rng(seed)
    x = lattice([0.0, 0.0, 0.0], L, dx, 2, rng)
    p = default_params(3, 3)
    p.use_musl = 1 if musl else 0
    p.flip_ratio = -0.95  # AFLIP
    p.plastic_model = PlasticModel.DPMui
    p.mu_1, p.mu_2, p.I_ref = 0.38, 0.64, 0.279
    p.grain_diameter, p.rho_s = 1e-3, 2500.0
    p.E, p.nu = 1e7, 0.3
    p.gravity[1] = -9.81
    p.end_frame, p.fps = 1, 1.0
    sc = Scene("collapse3d_mui_musl_aflip_q3", p, x)
    sc.plates = [make_plate(0.0, PlateType.bottom, BC.SlipStick, 0.4)]
    return _finish(sc, dx, 8, 0.6 * 2500.0)


def terrain_bumps(rng, n=3, x_range=(1.2, 2.4), z_range=(0.05, 0.45), h=0.1, sigma=0.15):
    prm = [0.0, float(n)]
    for _ in range(n):
        prm += [rng.uniform(*x_range), rng.uniform(*z_range), h, sigma]
    return prm


def incline3d_mcc(scale=1.0, seed=99, theta_deg=30.0):
    """3D Perzyna-Modified-Cam-Clay flow down a 30 deg incline with Gaussian bumps.

    Gravity is rotated by 30 deg (the reference's own way of tilting a slope,
    tests.cpp:112-116); the terrain is the level set y = sum of 3 Gaussian
    bumps (h = 0.1 m, sigma = 0.15 m, seeded positions) with BC SlipFree,
    mu = 0.45.  Release block 1.0 x 0.3 x 0.5 m (x, height y, z), dx = 0.01 m,
    8 particles per cell (1,200,000 at scale 1).  M = 1.2, beta = 0,
    p0 = 1e4 Pa, E = 5e6 Pa, nu = 0.25, rho = 1000 (the reference default).
    The Perzyna parameter of the reference is a relaxation time
    (plasticity.cpp:545); the 10 Pa.s viscosity is mapped to
    perzyna_visc = 10 Pa.s / p0 = 1e-3 s.
    """
    dx = 0.01
    L = [1.0 * scale, 0.3 * scale, 0.5 * scale]
    L = [max(dx, round(v / dx) * dx) for v in L]
    rng = np.random.default_rng(seed)
    x = lattice([0.0, 0.5 * dx, 0.0], [L[0], 0.5 * dx + L[1], L[2]], dx, 2, rng)
    p = default_params(3, 2)
    th = theta_deg * math.pi / 180.0
    p.gravity[0] = 9.81 * math.sin(th)
    p.gravity[1] = -9.81 * math.cos(th)
    p.plastic_model = PlasticModel.MCCVisc
    p.hardening_law = HardeningLaw.ExpoImpl
    p.M, p.beta, p.p0 = 1.2, 0.0, 1e4
    p.perzyna_exp, p.perzyna_visc = 1.0, 10.0 / 1e4
    p.E, p.nu = 5e6, 0.25
    p.end_frame, p.fps = 1, 1.0
    sc = Scene("incline3d_mccvisc_usl_aflip_q2", p, x)
    bumps = terrain_bumps(rng, x_range=(1.2 * scale + 0.2, 2.4 * scale + 0.2), z_range=(0.1 * scale, 0.4 * scale))
    sc.objects = [make_object(ObjectKind.TerrainGauss, BC.SlipFree, 0.45, bumps)]
    return _finish(sc, dx, 8, 1000.0)


def granular_scene(rng, dim, kind, n_target, material, E, phi_deg=30.0, aspect=2.0):
    """One seeded scene of the ensemble and serving workloads: a column
    collapse on a SlipFree floor (mu 0.5) or a release block on a 30 deg
    incline with two Gaussian bumps (SlipFree, mu 0.45); n_target particles
    (2 x 2 (x 2) jittered per cell, the cell size chosen to match), material
    "dp" (M = tan phi), "mcc" (Perzyna Cam-Clay, M 1.2, p0 1e4 Pa, 1e-3 s) or
    "mui" (mu(I): mu_1 0.38, mu_2 0.64); APIC USL, quadratic splines."""
    ppc = 4 if dim == 2 else 8
    cells = max(8.0, n_target / ppc)
    W = 0.2
    if kind == "collapse":
        nw = max(2, int(round((cells / aspect) ** (1.0 / dim))))
        nh = max(2, int(round(aspect * nw)))
        dx = W / nw
        hi = [nw * dx, nh * dx] + ([nw * dx] if dim == 3 else [])
        lo = [0.0] * dim
    else:
        # block 2:1:1 (x, height, z)
        nh = max(2, int(round((cells / 2.0 ** (dim - 1)) ** (1.0 / dim))))
        dx = W / nh
        hi = [2 * nh * dx, nh * dx] + ([nh * dx] if dim == 3 else [])
        lo = [0.0, 0.5 * dx] + ([0.0] if dim == 3 else [])
        hi[1] += 0.5 * dx
    x = lattice(lo, hi, dx, 2, rng)
    p = default_params(dim, 2)
    p.flip_ratio = -2.0
    p.E, p.nu = E, 0.3
    rho = 1550.0
    if material == "dp":
        p.plastic_model = PlasticModel.DP
        p.M = math.tan(phi_deg * math.pi / 180.0)
    elif material == "mcc":
        p.plastic_model = PlasticModel.MCCVisc
        p.hardening_law = HardeningLaw.ExpoImpl
        p.M, p.beta, p.p0 = 1.2, 0.0, 1e4
        p.perzyna_exp, p.perzyna_visc = 1.0, 1e-3
        rho = 1000.0
    else:
        p.plastic_model = PlasticModel.DPMui
        p.mu_1, p.mu_2, p.I_ref = 0.38, 0.64, 0.279
        p.grain_diameter, p.rho_s = 1e-3, 2500.0
        rho = 1500.0
    p.end_frame, p.fps = 1, 1.0
    sc = Scene(f"{kind}{dim}d_{material}", p, x)
    if kind == "collapse":
        p.gravity[1] = -9.81
        sc.plates = [make_plate(0.0, PlateType.bottom, BC.SlipFree, 0.5)]
    else:
        th = 30.0 * math.pi / 180.0
        p.gravity[0] = 9.81 * math.sin(th)
        p.gravity[1] = -9.81 * math.cos(th)
        L = hi[0]
        bumps = [0.0, 2.0]
        for k in range(2):
            bumps += [L * (1.3 + 0.6 * k) + rng.uniform(0, 0.2 * L), float(rng.uniform(0.2, 0.8)) * (hi[2] if dim == 3
                      else 0.0), 0.3 * (hi[1] - lo[1]), 0.5 * (hi[1] - lo[1])]
        sc.objects = [make_object(ObjectKind.TerrainGauss, BC.SlipFree, 0.45, bumps)]
    return _finish(sc, dx, ppc, rho)


def ensemble(n=256, seed=777, n_min=5_000, n_max=300_000):
    """The batched-ensemble workload: n independent DP column collapses,
    particle counts log-uniform in [n_min, n_max], 3D with probability 1/2,
    aspect ratio uniform in [0.5, 4], friction angle uniform in [20, 40] deg,
    E log-uniform in [1e5, 1e7] Pa (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        npart = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
        dim = 3 if rng.uniform() < 0.5 else 2
        aspect = rng.uniform(0.5, 4.0)
        phi = rng.uniform(20.0, 40.0)
        E = math.exp(rng.uniform(math.log(1e5), math.log(1e7)))
        out.append(granular_scene(rng, dim, "collapse", npart, "dp", E, phi, aspect))
    return out


def serving_request(rng, n_min=10_000, n_max=2_000_000):
    """One request of the serving workload: 2D or 3D, collapse or incline,
    particle count log-uniform in [n_min, n_max], material DP, MCC or mu(I)."""
    npart = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
    dim = 3 if rng.uniform() < 0.5 else 2
    kind = "collapse" if rng.uniform() < 0.5 else "incline"
    material = ("dp", "mcc", "mui")[int(rng.integers(0, 3))]
    E = math.exp(rng.uniform(math.log(1e5), math.log(1e7)))
    return granular_scene(rng, dim, kind, npart, material, E, rng.uniform(20.0, 40.0), rng.uniform(0.5, 4.0))


WORKLOADS = {
    "collapse2d": collapse2d,
    "collapse3d_mui": collapse3d_mui,
    "incline3d_mcc": incline3d_mcc,
}
