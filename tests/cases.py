"""Shared scene variants for the parity tests (oracle pin and GPU parity).

Every case is a small perturbed block (random velocities, deformation
gradients, affine B and plastic history; see scenes.perturb) so that a single
step drives each model through its plastic branches and each boundary
through its friction branches.
"""
import math

import numpy as np

from matter_tests_b200 import scenes
from matter_tests_b200.abi import (BC, ElasticModel, HardeningLaw, ObjectKind, PlasticModel, PlateType,
                                   default_params, make_object, make_plate)

PM, HL = PlasticModel, HardeningLaw

# plasticity models and their parameters (plasticity.cpp:11-665)
MODEL_CASES = {
    "noplast": dict(plastic_model=PM.NoPlasticity),
    "neohookean": dict(plastic_model=PM.NoPlasticity, elastic_model=ElasticModel.NeoHookean),
    "vm": dict(plastic_model=PM.VM, q_max=4e3),
    "dp": dict(plastic_model=PM.DP, M=0.6),
    "dp_cohesion": dict(plastic_model=PM.DP, M=0.6, q_cohesion=800.0),
    "dpsoft": dict(plastic_model=PM.DPSoft, M=0.6, q_cohesion=300.0, xi=2.0),
    "dpsoft_nopradhana": dict(plastic_model=PM.DPSoft, M=0.6, q_cohesion=300.0, use_pradhana=0),
    "vmvisc": dict(plastic_model=PM.VMVisc, q_max=5e3, q_min=2e3, xi=0.0, perzyna_visc=2e-4),
    "vmvisc_newton": dict(plastic_model=PM.VMVisc, q_max=5e3, q_min=2e3, xi=1.5, perzyna_visc=2e-4),
    "vmvisc_capped": dict(plastic_model=PM.VMVisc, q_max=5e3, q_min=2e3, p_min=-2e3),
    "dpvisc": dict(plastic_model=PM.DPVisc, M=0.6, perzyna_visc=2e-4),
    "dpvisc_mibf": dict(plastic_model=PM.DPVisc, M=0.6, use_mibf=1),
    "dpvisc_exp2": dict(plastic_model=PM.DPVisc, M=0.6, perzyna_exp=2.0, perzyna_visc=2e-4),
    "dpvisc_misesq": dict(plastic_model=PM.DPVisc, M=0.6 * math.sqrt(3.0), use_mises_q=1),
    "dpmui": dict(plastic_model=PM.DPMui),
    "dpmui_cohesion": dict(plastic_model=PM.DPMui, q_cohesion=200.0),
    "mcc_nohard": dict(plastic_model=PM.MCC, hardening_law=HL.NoHard, p0=3e3),
    "mcc_expoexpl": dict(plastic_model=PM.MCC, hardening_law=HL.ExpoExpl, p0=3e3, xi=5.0),
    "mcc_sinhexpl": dict(plastic_model=PM.MCC, hardening_law=HL.SinhExpl, p0=3e3, xi=5.0),
    "mcc_expoimpl": dict(plastic_model=PM.MCC, hardening_law=HL.ExpoImpl, p0=3e3, xi=5.0),
    "mcc_sinhimpl": dict(plastic_model=PM.MCC, hardening_law=HL.SinhImpl, p0=3e3, xi=5.0),
    "mcc_beta": dict(plastic_model=PM.MCC, hardening_law=HL.ExpoImpl, p0=3e3, beta=0.3, xi=2.0),
    "mccvisc": dict(plastic_model=PM.MCCVisc, hardening_law=HL.ExpoImpl, M=1.2, p0=3e3, perzyna_visc=2e-4),
    "mccvisc_mibf": dict(plastic_model=PM.MCCVisc, hardening_law=HL.ExpoImpl, M=1.2, p0=3e3, use_mibf=1),
    "mccvisc_exp2": dict(plastic_model=PM.MCCVisc, hardening_law=HL.SinhImpl, M=1.2, p0=3e3,
                         perzyna_exp=2.0, perzyna_visc=2e-4, xi=1.0),
    "mccmui_expoimpl": dict(plastic_model=PM.MCCMui, hardening_law=HL.ExpoImpl, p0=3e3, xi=2.0),
    "mccmui_expoexpl": dict(plastic_model=PM.MCCMui, hardening_law=HL.ExpoExpl, p0=3e3, xi=2.0),
    "mccmui_sinhimpl": dict(plastic_model=PM.MCCMui, hardening_law=HL.SinhImpl, p0=3e3, xi=2.0),
    "snow": dict(plastic_model=PM.Snow),
}

# transfer schemes (position_update.cpp:14-24, musl.cpp)
TRANSFER_CASES = {
    "apic_usl": dict(flip_ratio=-2.0, use_musl=0),
    "aflip_usl": dict(flip_ratio=-0.95, use_musl=0),
    "pureaflip_usl": dict(flip_ratio=-1.0, use_musl=0),
    "picflip_usl": dict(flip_ratio=0.9, use_musl=0),
    "apic_musl": dict(flip_ratio=-2.0, use_musl=1),
    "aflip_musl": dict(flip_ratio=-0.95, use_musl=1),
    "picflip_musl": dict(flip_ratio=0.5, use_musl=1),
}


def block(dim=3, deg=2, n=6, seed=3, E=1e6, rho=1000.0, gravity=(0.3, -9.81, 0.2)):
    """A perturbed n^dim-cell block of side n*dx at the origin."""
    dx = 0.01
    rng = np.random.default_rng(seed)
    lo = [0.0] * dim
    hi = [n * dx] * dim
    x = scenes.lattice(lo, hi, dx, 2, rng)
    p = default_params(dim, deg)
    p.E, p.nu = E, 0.3
    for a in range(dim):
        p.gravity[a] = gravity[a]
    p.end_frame, p.fps = 1, 1.0
    sc = scenes.Scene(f"block{dim}d_q{deg}", p, x)
    scenes._finish(sc, dx, 2 ** dim, rho)
    return scenes.perturb(sc, seed=seed + 1)


def apply(scene, **kw):
    for k, v in kw.items():
        if k in ("gravity", "grid_reference_point"):
            for a, g in enumerate(v):
                getattr(scene.params, k)[a] = g
        else:
            setattr(scene.params, k, v)
    if scene.params.use_mibf and scene.scalars is not None:
        pass
    return scene


def box_plates(scene, bc, friction, moving=False):
    """Six plates cutting into the block so every plate branch is reached."""
    dx = scene.params.dx
    lo = scene.x.min(axis=0)
    hi = scene.x.max(axis=0)
    d = scene.dim
    v = (0.0, 0.0, 0.0)
    kinds = [(PlateType.bottom, lo[1] + 1.2 * dx, (0.0, 0.05, 0.0)),
             (PlateType.top, hi[1] - 1.2 * dx, (0.02, -0.05, 0.0)),
             (PlateType.left, lo[0] + 1.2 * dx, (0.05, 0.01, 0.0)),
             (PlateType.right, hi[0] - 1.2 * dx, (-0.05, 0.0, 0.0))]
    if d == 3:
        kinds += [(PlateType.back, lo[2] + 1.2 * dx, (0.0, 0.0, 0.05)),
                  (PlateType.front, hi[2] - 1.2 * dx, (0.0, 0.0, -0.05))]
    plates = []
    for i, (pt, pos, vel) in enumerate(kinds):
        plates.append(make_plate(pos, pt, bc, friction, v=vel if moving else v,
                                 vmin_factor=2.0 if moving else 1.0, load_factor=0.5 if moving else 0.0,
                                 lower=-1e15 if i % 2 == 0 else lo[0] + 2 * dx))
    scene.plates = plates
    return scene


def periodic(dim=3, deg=2, n=6, musl=0, flip_ratio=-2.0, seed=3):
    """A block filling a periodic box in x (pbc, pbc.cpp): it moves +x at
    1.5 m/s so particles cross x = Lx and re-enter at x = 0, under a light
    gravity, clear of the fixed grid's y (and z) edges."""
    sc = apply(block(dim, deg, n=n, seed=seed, gravity=(0.4, -1.0, 0.0)), plastic_model=PM.DP, M=0.6,
               use_musl=musl, flip_ratio=flip_ratio)
    p = sc.params
    p.pbc = 1
    p.L[0], p.L[1], p.L[2] = n * p.dx, 0.1, 0.08
    sc.x[:, 1] += 0.03
    if dim == 3:
        sc.x[:, 2] += 0.01
    sc.v[:, 0] += 1.5
    sc.plates, sc.objects = [], []
    return sc


def object_cases(dim):
    """Analytic objects (object_*.hpp) placed so they intersect a block at the origin."""
    cases = {
        "bump": [make_object(ObjectKind.Bump, BC.SlipFree, 0.3)],
        "ground": [make_object(ObjectKind.Ground, BC.SlipStick, 0.4, [0.012])],
        "ramp": [make_object(ObjectKind.Ramp, BC.SlipFree, 0.0)],
        "curve": [make_object(ObjectKind.Curve, BC.NoSlip, 0.0)],
        "gate": [make_object(ObjectKind.Gate, BC.SlipFree, 0.5, [0.045])],
        "terrain": [make_object(ObjectKind.TerrainGauss, BC.SlipFree, 0.45,
                                [0.005, 2, 0.03, 0.03, 0.01, 0.02, 0.05, 0.01, 0.015, 0.015])],
        "two_objects": [make_object(ObjectKind.Ground, BC.SlipFree, 0.2, [0.01]),
                        make_object(ObjectKind.Gate, BC.SlipStick, 0.3, [0.05])],
    }
    if dim == 3:
        c = math.cos(0.4)
        s = math.sin(0.4)
        R = [c, s, 0.0, -s, c, 0.0, 0.0, 0.0, 1.0]  # column-major rotation about z
        cases["box"] = [make_object(ObjectKind.BoxRotated, BC.SlipStick, 0.35,
                                    [0.03, 0.0, 0.03, 0.02, 0.015, 0.02] + R)]
        cases["silo"] = [make_object(ObjectKind.Silo, BC.SlipFree, 0.2, [-1.0])]
    else:
        c = math.cos(0.4)
        s = math.sin(0.4)
        cases["box"] = [make_object(ObjectKind.BoxRotated, BC.SlipStick, 0.35,
                                    [0.03, 0.0, 0.0, 0.02, 0.015, 0.0, c, s, -s, c])]
    return cases


def max_rel(a, b):
    """max |a - b| / max |b| (with max |b| floored at tiny)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = max(np.abs(b).max(initial=0.0), 1e-300)
    return float(np.abs(a - b).max(initial=0.0) / s)


def levelset_cases(dim):
    """Dense level-set objects (ObjectKind.LevelSet) intersecting a block at the
    origin: name -> (objects, levelsets)."""
    lo, hi = [-0.05] * dim, [0.1] * dim
    h = 0.004
    c = np.array([0.025, -0.004, 0.025][:dim])

    def sphere(X):
        return np.linalg.norm(X - c, axis=1) - 0.02

    def sphere_normals(ls):
        n = [ls.phi.shape[a] for a in range(dim)]
        axes = [ls.origin[a] + ls.spacing * np.arange(n[a]) for a in range(dim)]
        X = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, dim)
        d = X - c
        d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-30)
        out = np.zeros((X.shape[0], 3), dtype=np.float32)
        out[:, :dim] = d
        return out.reshape(ls.phi.shape + (3,))

    terrain = make_object(ObjectKind.TerrainGauss, BC.SlipFree, 0.45,
                          [0.005, 2, 0.03, 0.03, 0.01, 0.02, 0.05, 0.01, 0.015, 0.015])
    out = {}
    s0 = scenes.sample_levelset(sphere, lo, hi, h, dim, slot=0)
    out["sphere_slipstick"] = ([make_object(ObjectKind.LevelSet, BC.SlipStick, 0.4, [0])], [s0])
    s1 = scenes.sample_levelset(sphere, lo, hi, h, dim, slot=2)
    s1.normals = sphere_normals(s1)
    out["sphere_normals_slipfree"] = ([make_object(ObjectKind.LevelSet, BC.SlipFree, 0.3, [2])], [s1])
    t = scenes.terrain_levelset(terrain, dim, lo, hi, h, slot=1)
    out["terrain_slipfree"] = ([make_object(ObjectKind.LevelSet, BC.SlipFree, 0.45, [1])], [t])
    small = scenes.sample_levelset(sphere, [0.0] * dim, [0.03] * dim, h, dim, slot=3)  # ends inside the block
    out["partial_lattice_noslip_and_ground"] = (
        [make_object(ObjectKind.LevelSet, BC.NoSlip, 0.0, [3]),
         make_object(ObjectKind.Ground, BC.SlipFree, 0.2, [0.008])], [small])
    return out
