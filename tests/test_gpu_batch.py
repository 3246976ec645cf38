"""Batched stepping (mtr_batch): scenes of different dimension, spline,
precision and transfer scheme advance together, each exactly as it does alone.

Alone and in the batch a scene runs the same step; the only difference is
the order of the floating-point atomic sums, so FP64 states agree to 1e-10
of each field's scale after a few steps and FP32 states to 1e-5 (the
mixed-precision one-step tolerances, grown over the steps)."""
import copy

import numpy as np
import pytest

from matter_tests_b200.abi import BC, PREC_FP64, PREC_MIXED

import cases
from gpu_util import needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]


def scene_set():
    out = []
    a = cases.apply(cases.block(3, 3, n=5), plastic_model=cases.PM.DPMui, use_musl=1, flip_ratio=-0.95)
    out.append(cases.box_plates(a, BC.SlipStick, 0.4))
    b = cases.apply(cases.block(3, 2, n=6, seed=5), plastic_model=cases.PM.DP, M=0.6, flip_ratio=-2.0)
    b.objects = cases.object_cases(3)["two_objects"]
    out.append(b)
    c = cases.apply(cases.block(2, 2, n=10, seed=8), plastic_model=cases.PM.MCCVisc, M=1.2, p0=3e3,
                    perzyna_visc=2e-4)
    out.append(cases.box_plates(c, BC.SlipFree, 0.3))
    d = cases.apply(cases.block(3, 3, n=4, seed=9), plastic_model=cases.PM.DPMui, use_musl=1, flip_ratio=-0.95)
    d.params.precision = PREC_MIXED
    out.append(d)
    e = cases.apply(cases.block(2, 3, n=12, seed=10), plastic_model=cases.PM.DPVisc, M=0.5, use_mibf=1)
    e.params.precision = PREC_MIXED
    out.append(cases.box_plates(e, BC.SlipStick, 0.3))
    return out


def make_sim(sc):
    from matter_tests_b200.gpu import GpuSim
    g = GpuSim(copy.copy(sc.params))
    g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
    g.set_objects(sc.plates, sc.objects)
    return g


def state(g):
    return g.particles(), g.clock(), g.status()


def assert_same(a, b, prec):
    tol = 1e-10 if prec == PREC_FP64 else 1e-5
    pa, ca, sa = a
    pb, cb, sb = b
    assert ca["step"] == cb["step"] and ca["frame"] == cb["frame"], (ca, cb)
    assert abs(ca["time"] - cb["time"]) <= 1e-14 * max(1.0, abs(cb["time"]))
    assert sa[0] == sb[0], (sa, sb)
    for k in ("x", "v", "F", "B"):
        scale = max(np.abs(pb[k]).max(), 1e-300)
        e = np.abs(pa[k] - pb[k]).max() / scale
        assert e <= tol, (k, e)


@pytest.mark.parametrize("nsteps", [1, 13])
def test_each_scene_is_the_same_alone_and_in_the_batch(nsteps):
    from matter_tests_b200.gpu import GpuBatch
    scs = scene_set()
    alone = []
    for sc in scs:
        g = make_sim(sc)
        g.step(nsteps)
        alone.append(state(g))
        g.close()
    sims = [make_sim(sc) for sc in scs]
    batch = GpuBatch(sims)
    batch.step(nsteps)
    for sc, g, ref in zip(scs, sims, alone):
        assert_same(state(g), ref, sc.params.precision)
    batch.close()
    for g in sims:
        g.close()


def test_batch_steps_in_several_calls_and_members_continue_alone():
    from matter_tests_b200.gpu import GpuBatch
    scs = scene_set()[:3]
    alone = []
    for sc in scs:
        g = make_sim(sc)
        g.step(12)
        alone.append(state(g))
        g.close()
    sims = [make_sim(sc) for sc in scs]
    batch = GpuBatch(sims)
    batch.step(3)
    batch.step(5)
    batch.close()
    for g in sims:
        g.step(4)  # after the batch is gone the members step on their own
    for sc, g, ref in zip(scs, sims, alone):
        assert_same(state(g), ref, sc.params.precision)
        g.close()


def test_batch_members_stop_at_their_own_end_and_regrow_their_own_grid():
    from matter_tests_b200.gpu import GpuBatch
    scs = scene_set()[:2]
    # the first scene ends after about six steps (end of its only frame)
    p0 = scs[0].params
    dt_max = p0.cfl_elastic * p0.dx / (p0.E / p0.rho) ** 0.5
    p0.end_frame, p0.fps = 1, 1.0 / (6.5 * dt_max)
    # the second flies apart (a radial velocity of about 50 m/s at the
    # corners; the CFL limit then moves them half a cell per step), so its
    # extent grows several-fold and outgrows the 1.5x headroom of its grid
    c = scs[1].x.mean(axis=0)
    scs[1].v = scs[1].v + 1000.0 * (scs[1].x - c)
    scs[1].plates, scs[1].objects = [], []
    alone = []
    for sc in scs:
        g = make_sim(sc)
        g.step(60)
        alone.append(state(g))
        g.close()
    sims = [make_sim(sc) for sc in scs]
    batch = GpuBatch(sims)
    batch.step(60)
    assert sims[0].clock()["done"] == 1
    assert sims[1].clock()["step"] == 60
    st = batch.stats()  # the regrowths happened inside the batch, and each rebuilt it
    assert st["regrowths"] >= 1 and st["rebuilds"] >= 1 + st["regrowths"] // len(scs)
    assert st["regrow_ms"] >= 0 and st["rebuild_ms"] > 0
    for sc, g, ref in zip(scs, sims, alone):
        assert_same(state(g), ref, sc.params.precision)
    batch.close()
    for g in sims:
        g.close()


def test_periodic_scenes_are_refused():
    from matter_tests_b200.gpu import GpuBatch, MtrFailure
    sims = [make_sim(scene_set()[0]), make_sim(cases.periodic(3, 2))]
    with pytest.raises(MtrFailure):
        GpuBatch(sims)
    for g in sims:
        g.close()


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
def test_footprint_matches_the_upload(prec):
    """mtr_footprint predicts what mtr_upload allocates (within the driver's
    allocation granularity) for a 128,000-particle scene."""
    import torch
    from matter_tests_b200 import scenes
    from matter_tests_b200.gpu import footprint
    sc = scenes.collapse3d_mui(scale=0.5)
    sc.params.precision = prec
    est = footprint(sc.params, sc.x)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    g = make_sim(sc)
    free1, _ = torch.cuda.mem_get_info()
    g.close()
    used = free0 - free1
    assert 0.8 * used <= est <= 1.25 * used + (32 << 20), (est, used)


def test_batch_clocks_match_each_members_clock():
    from matter_tests_b200.gpu import GpuBatch
    scs = scene_set()
    sims = [make_sim(sc) for sc in scs]
    sims[1].set_step_limit(5)
    batch = GpuBatch(sims)
    batch.step(9)
    got = batch.clocks()
    assert len(got) == len(sims)
    for g, ck in zip(sims, got):
        assert ck == g.clock()
    assert got[1]["step"] == 5 and got[0]["step"] == 9
    batch.close()
    for g in sims:
        g.close()


def test_members_join_and_leave_one_batch():
    """mtr_batch_set_members: one batch whose members change between calls
    (scenes join after others have stepped, leave and continue alone), each
    scene ending exactly as when stepped alone for the same number of steps;
    membership changes within the same groups update the step graph in place."""
    from matter_tests_b200.gpu import GpuBatch
    scs = scene_set()
    # a second scene of scene 1's group (3D, quadratic, FP64, USL, Drucker-Prager)
    scs.append(cases.apply(cases.block(3, 2, n=5, seed=21), plastic_model=cases.PM.DP, M=0.6, flip_ratio=-2.0))
    sims = [make_sim(sc) for sc in scs]
    # scene i steps: in the batch for the calls it is a member of, then alone to 36;
    # the first two changes keep the same groups (1 <-> 5, then both)
    plan = [(0, 1, 2), (0, 5, 2), (0, 1, 2, 5), (1, 2, 3, 4, 5), (3, 4), (0, 1, 2, 3, 4, 5)]
    b = GpuBatch([sims[i] for i in plan[0]])
    done = [0] * len(scs)
    for members in plan:
        b.set_members([sims[i] for i in members])
        b.step(6)
        for i in members:
            done[i] += 6
    updates = b.graph_updates()
    b.close()
    for i, g in enumerate(sims):
        g.step(36 - done[i])
    for i, sc in enumerate(scs):
        alone = make_sim(sc)
        alone.step(36)
        assert_same(state(sims[i]), state(alone), sc.params.precision)
        alone.close()
        sims[i].close()
    assert updates >= 2, updates
