"""Parity of the CUDA step (libmatter_gpu.so, through its C ABI) with the oracle.

The oracle is the C restatement pinned bit-for-bit to the reference compiled
from source (test_oracle_pin.py).  The plain FP64 GPU path must match it to
1e-10 relative per field (grid mass, momentum/velocity, flip and every
particle field) after one step; GPU atomics and fused multiply-adds change the
summation order, which moves results by a few ulps, far inside that bound.
The grid axes (arange, tools.hpp:291-296) are compared bit for bit.

The six plastic scalars are held to the same 1e-10 of their field's scale plus
100x the oracle's own spread under a few-ulp perturbation of its input
(gpu_util.oracle_sensitivity): several of them come out of cancellation-prone
closed forms in the reference (the mu(I) quadratic root, plasticity.cpp:388;
viscosity = (mu_i - mu_1) p / gamma_dot, :392), which no implementation can
reproduce more closely than the reference reproduces itself.
"""
import numpy as np
import pytest

from matter_tests_b200 import scenes
from matter_tests_b200.abi import BC

import cases
from gpu_util import compare_states, needs_gpu, oracle_sensitivity, run_gpu, run_oracle

pytestmark = [pytest.mark.gpu, needs_gpu]

REL_ONE_STEP = 1e-10


@pytest.mark.parametrize("deg", [2, 3])
@pytest.mark.parametrize("model", sorted(cases.MODEL_CASES))
def test_models_one_step(model, deg):
    sc = cases.apply(cases.block(3, deg, n=5), **cases.MODEL_CASES[model])
    sc = cases.box_plates(sc, BC.SlipFree, 0.3)
    g, o = run_gpu(sc, 1), run_oracle(sc, 1)
    compare_states(g, o, REL_ONE_STEP, sens=oracle_sensitivity(sc, 1))


@pytest.mark.parametrize("model", ["dp", "dpmui", "mccvisc", "dpsoft", "noplast", "vmvisc_newton"])
def test_models_2d_one_step(model):
    sc = cases.apply(cases.block(2, 2, n=8), **cases.MODEL_CASES[model])
    sc = cases.box_plates(sc, BC.SlipStick, 0.3)
    g, o = run_gpu(sc, 1), run_oracle(sc, 1)
    compare_states(g, o, REL_ONE_STEP, sens=oracle_sensitivity(sc, 1))


@pytest.mark.parametrize("dim,deg", [(2, 2), (2, 3), (3, 2), (3, 3)])
@pytest.mark.parametrize("transfer", sorted(cases.TRANSFER_CASES))
def test_transfers_one_step(transfer, dim, deg):
    sc = cases.apply(cases.block(dim, deg, n=6 if dim == 3 else 10), plastic_model=cases.PM.DP, M=0.6,
                     **cases.TRANSFER_CASES[transfer])
    sc = cases.box_plates(sc, BC.SlipStick, 0.4)
    g, o = run_gpu(sc, 1), run_oracle(sc, 1)
    compare_states(g, o, REL_ONE_STEP, sens=oracle_sensitivity(sc, 1))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("bc", [BC.NoSlip, BC.SlipStick, BC.SlipFree])
@pytest.mark.parametrize("moving", [False, True])
def test_plates(bc, moving, dim):
    sc = cases.apply(cases.block(dim, 2, n=6 if dim == 3 else 10), plastic_model=cases.PM.NoPlasticity)
    sc = cases.box_plates(sc, bc, 0.35, moving=moving)
    g, o = run_gpu(sc, 3), run_oracle(sc, 3)
    compare_states(g, o, 1e-9, sens=oracle_sensitivity(sc, 3))
    for pg, po in zip(g["plates"], o["plates"]):
        assert abs(pg.pos_object - po.pos_object) <= 1e-12 * max(1.0, abs(po.pos_object))
        assert abs(pg.pos_upper - po.pos_upper) <= 1e-9 * max(1.0, abs(po.pos_upper))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("obj", ["bump", "ground", "ramp", "curve", "gate", "terrain", "two_objects", "box", "silo"])
def test_objects(obj, dim):
    oc = cases.object_cases(dim)
    if obj not in oc:
        pytest.skip("3D-only object")
    sc = cases.apply(cases.block(dim, 2, n=5 if dim == 3 else 10), plastic_model=cases.PM.DPVisc, M=0.5, use_mibf=1)
    sc.objects = oc[obj]
    g, o = run_gpu(sc, 2), run_oracle(sc, 2)
    compare_states(g, o, 1e-9, sens=oracle_sensitivity(sc, 2))


@pytest.mark.parametrize("name", ["sphere_slipstick", "sphere_normals_slipfree", "terrain_slipfree",
                                  "partial_lattice_noslip_and_ground"])
@pytest.mark.parametrize("dim", [2, 3])
def test_levelset_objects(name, dim):
    """Dense level-set objects (object_vdb.hpp on a lattice): inside test from
    the trilinear sample of phi, normals from its central-difference gradient
    or from given normals, lattice edges reading the background."""
    sc = cases.apply(cases.block(dim, 2, n=5 if dim == 3 else 10), plastic_model=cases.PM.DPVisc, M=0.5, use_mibf=1)
    sc.objects, sc.levelsets = cases.levelset_cases(dim)[name]
    g, o = run_gpu(sc, 3), run_oracle(sc, 3)
    compare_states(g, o, 1e-9, sens=oracle_sensitivity(sc, 3))


def test_levelset_terrain_follows_the_analytic_terrain():
    """The terrain sampled as phi = y - s(x, z) at 1/8 of dx steers the flow
    like the analytic TerrainGauss object: after 20 steps positions agree to
    0.5% of dx on average and 10% at most (the level set differs from the
    surface by the interpolation of s between samples, which can move a node
    across the surface)."""
    import copy
    base = cases.apply(cases.block(3, 2, n=5), plastic_model=cases.PM.DP, M=0.6)
    terrain = cases.object_cases(3)["terrain"][0]
    a = copy.deepcopy(base)
    a.objects = [terrain]
    b = copy.deepcopy(base)
    b.levelsets = [scenes.terrain_levelset(terrain, 3, [-0.05] * 3, [0.1] * 3, base.params.dx / 8, slot=0)]
    lo = cases.make_object(cases.ObjectKind.LevelSet, terrain.bc, terrain.friction, [0])
    b.objects = [lo]
    ga, gb = run_gpu(a, 20), run_gpu(b, 20)
    err = np.abs(ga["p"]["x"] - gb["p"]["x"])
    assert err.mean() <= 0.005 * base.params.dx and err.max() <= 0.1 * base.params.dx, (err.mean(), err.max())


def test_levelset_slot_must_be_loaded():
    from matter_tests_b200.gpu import GpuSim, MtrFailure
    sc = cases.apply(cases.block(3, 2, n=4), plastic_model=cases.PM.DP, M=0.6)
    g = GpuSim(sc.params)
    g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
    g.set_objects([], [cases.make_object(cases.ObjectKind.LevelSet, BC.SlipFree, 0.2, [1])])
    with pytest.raises(MtrFailure):
        g.step(1)  # slot 1 holds no level set
    with pytest.raises(MtrFailure):
        g.set_objects([], [cases.make_object(cases.ObjectKind.LevelSet, BC.SlipFree, 0.2, [7])])
    g.close()


@pytest.mark.parametrize("builder,scale", [("collapse2d", 0.25), ("collapse3d_mui", 0.12), ("incline3d_mcc", 0.12)])
def test_workloads_ten_steps(builder, scale):
    sc = scenes.WORKLOADS[builder](scale=scale)
    g, o = run_gpu(sc, 10), run_oracle(sc, 10)
    compare_states(g, o, 1e-9, sens=oracle_sensitivity(sc, 10))


def test_graphs_match_direct_launches():
    sc = cases.apply(cases.block(3, 3, n=5), plastic_model=cases.PM.DPMui, use_musl=1)
    a = run_gpu(sc, 37, graphs=True)
    b = run_gpu(sc, 37, graphs=False)
    assert a["c"]["step"] == b["c"]["step"] == 37
    for k in ("x", "v", "F"):
        assert np.abs(a["p"][k] - b["p"][k]).max() <= 1e-12 * max(1.0, np.abs(b["p"][k]).max())


@pytest.mark.parametrize("dim", [2, 3])
def test_sort_keys_bitexact(dim):
    """Cell keys equal the oracle's and the order is a stable sort of them."""
    sc = cases.apply(cases.block(dim, 2, n=7 if dim == 3 else 12), plastic_model=cases.PM.DP, M=0.6)
    for nsteps in (1, 4):
        g, o = run_gpu(sc, nsteps), run_oracle(sc, nsteps)
        keys_in, perm, ids_in = g["sort"]
        # keys of the last step, in the order of that step's input, mapped to particle ids
        k_orig = np.zeros_like(keys_in)
        k_orig[ids_in] = keys_in
        assert np.array_equal(k_orig, o["keys"]), "cell keys differ from the oracle's"
        assert np.array_equal(perm, np.argsort(keys_in, kind="stable")), "not a stable sort"


def test_end_of_simulation_clock():
    sc = cases.apply(cases.block(3, 2, n=3), plastic_model=cases.PM.DP, M=0.6)
    dt_max = 0.5 * sc.params.dx / np.sqrt(sc.params.E / sc.params.rho)
    sc.params.fps = 1.0 / (3.5 * dt_max)
    sc.params.end_frame = 1
    g, o = run_gpu(sc, 10), run_oracle(sc, 10)
    assert g["c"]["step"] == o["c"]["step"] == 4
    assert g["c"]["done"] == 1
    compare_states(g, o, 1e-9, sens=oracle_sensitivity(sc, 10))


def test_grid_regrowth():
    """A block flying apart outgrows the first grid allocation; the step
    aborts before touching state, the grid regrows and the run continues."""
    sc = cases.apply(cases.block(3, 2, n=4), plastic_model=cases.PM.NoPlasticity)
    sc.v = sc.v * 0 + np.array([8.0, 0.0, 0.0]) * np.sign(sc.x[:, :1] - sc.x[:, :1].mean())
    g, o = run_gpu(sc, 60), run_oracle(sc, 60)
    assert g["c"]["step"] == 60
    compare_states(g, o, 1e-8, sens=oracle_sensitivity(sc, 60))


@pytest.mark.parametrize("dim,deg,musl,fr", [(3, 2, 0, -2.0), (3, 3, 1, -0.95), (2, 2, 0, 0.9), (2, 3, 1, -2.0)])
@pytest.mark.parametrize("nsteps", [1, 12])
def test_periodic(dim, deg, musl, fr, nsteps):
    """Periodic boundaries in x: the fixed grid, the periodic copies in P2G and
    the wrap of positions, while particles cross x = Lx."""
    sc = cases.periodic(dim, deg, n=6 if dim == 3 else 10, musl=musl, flip_ratio=fr)
    g, o = run_gpu(sc, nsteps), run_oracle(sc, nsteps)
    compare_states(g, o, REL_ONE_STEP if nsteps == 1 else 1e-9, sens=oracle_sensitivity(sc, nsteps))
    x0 = g["p"]["x"][:, 0]
    assert x0.min() >= 0.0 and x0.max() <= sc.params.L[0]


def test_reupload_into_a_used_context():
    """mtr_upload of a scene with the same particle count into a context that
    already stepped another keeps its buffers and step graphs and refills
    them; the result equals a fresh context's.  Then a scene of the same count
    spread over three times the extent, whose grid no longer fits, and one of
    another count."""
    from matter_tests_b200.gpu import GpuSim
    a = cases.apply(cases.block(3, 3, n=6, seed=3), plastic_model=cases.PM.DPMui, use_musl=1, flip_ratio=-0.95)
    b = cases.apply(cases.block(3, 3, n=6, seed=8), plastic_model=cases.PM.DPMui, use_musl=1, flip_ratio=-0.95)
    b.x = b.x + np.array([0.013, 0.002, -0.007])
    wide = cases.apply(cases.block(3, 3, n=6, seed=9), plastic_model=cases.PM.DPMui, use_musl=1, flip_ratio=-0.95)
    wide.x = wide.x * 3.0
    other = cases.apply(cases.block(3, 3, n=5, seed=4), plastic_model=cases.PM.DPMui, use_musl=1, flip_ratio=-0.95)
    assert a.Np == b.Np == wide.Np != other.Np
    g = GpuSim(a.params)
    for sc in (a, b, wide, other, b):
        g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
        g.set_scene_objects(sc)
        g.step(20)
        got = g.particles()
        assert g.clock()["step"] == 20
        ref = run_gpu(sc, 20, keep_pic_flip=False)
        for k in ("x", "v", "F", "B"):
            scale = max(np.abs(ref["p"][k]).max(), 1e-300)
            assert np.abs(got[k] - ref["p"][k]).max() <= 1e-10 * scale, (sc.name, k)
    g.close()


@pytest.mark.parametrize("pinned", [False, True])
def test_upload_download_round_trip_through_the_copy_staging(pinned):
    """mtr_upload then mtr_download, no step: every field comes back bit for
    bit in FP64.  700,001 particles make every array several staging chunks
    (8 MB) long with a partial last chunk; pageable numpy arrays go through the
    pinned staging, pinned ones are copied directly.  Absent F, B and scalars
    are filled on the device (identity, zeros, zeros), and a download of some
    fields leaves the others out."""
    import torch
    from matter_tests_b200.abi import PREC_FP64, default_params
    from matter_tests_b200.gpu import GpuSim
    n, d = 700_001, 3
    rng = np.random.default_rng(21)

    def arr(shape, lo=None):
        a = rng.normal(size=shape) if lo is None else rng.uniform(lo, lo + 0.5, size=shape)
        if not pinned:
            return a
        t = torch.empty(shape, dtype=torch.float64).pin_memory()
        t.numpy()[...] = a
        return t.numpy()
    x = arr((n, d), lo=0.1)  # a 0.5 m cube: a 50-cell grid per axis
    v, F, B, S = arr((n, d)), arr((n, d, d)), arr((n, d, d)), arr((n, 6))
    p = default_params(d, 2)
    p.dx = 0.01
    p.precision = PREC_FP64
    g = GpuSim(p)
    g.upload(x, v, F, B, S)
    got = g.particles()
    for k, a in (("x", x), ("v", v), ("F", F), ("B", B), ("scalars", S)):
        assert np.array_equal(got[k], a), k
    part = g.particles(fields=("x", "v"))
    assert set(part) == {"x", "v"} and np.array_equal(part["x"], x) and np.array_equal(part["v"], v)
    g.upload(x, v)
    got = g.particles()
    assert np.array_equal(got["F"], np.broadcast_to(np.eye(d), (n, d, d)))
    assert not got["B"].any() and not got["scalars"].any()
    g.close()
