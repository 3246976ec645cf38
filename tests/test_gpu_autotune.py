"""Block shapes of the tile kernels (mtr_autotune, mtr_set_tile_threads,
mtr_batch_autotune): every shape gives the step of the default shape, and
tuning leaves the scene exactly as it was.

A shape changes only the order of the floating-point atomic sums in the
shared-memory patches, so FP64 states agree to 1e-10 of each field's scale
after a few steps and FP32 states to 1e-5, the tolerances of the batch tests.
Tuning runs trial steps that stop before the commit: the particle state, the
clock, the plates and the status read back bit-identical afterwards."""
import numpy as np
import pytest

from matter_tests_b200.abi import PREC_FP64, PREC_MIXED, TILE_SLOTS

from gpu_util import needs_gpu
from test_gpu_batch import assert_same, make_sim, scene_set, state

pytestmark = [pytest.mark.gpu, needs_gpu]

SHAPES = [
    {"p2g": 64, "musl": 64, "g2p": 64, "defgrad": 64},
    {"p2g": 256, "musl": 128, "g2p": 128, "defgrad": 256},
    {"p2g": 64, "musl": 96, "g2p": 96, "defgrad": 160},
]
# x split of the scatters' stencil columns per shape: lanes per particle =
# split x (16 in 3D, 4 in 2D)
SPLITS = [(2, 2), (2, 1), (1, 2)]


def lanes_of(dim, split):
    cols = 16 if dim == 3 else 4
    return {"p2g": split[0] * cols, "musl": split[1] * cols}


def exact_state(g):
    p = g.particles()
    return p, g.clock(), g.status(), [bytes(q) for q in g.plates()]


def assert_identical(a, b):
    pa, ca, sa, la = a
    pb, cb, sb, lb = b
    assert ca == cb and sa == sb and la == lb
    for k in ("x", "v", "F", "B", "scalars"):
        assert np.array_equal(pa[k], pb[k]), k


@pytest.mark.parametrize("shape", range(len(SHAPES)))
def test_every_shape_steps_as_the_default(shape):
    for sc in scene_set():
        ref = make_sim(sc)
        ref.step(9)
        want = state(ref)
        ref.close()
        g = make_sim(sc)
        g.tile_threads = SHAPES[shape]
        g.tile_lanes = lanes_of(sc.dim, SPLITS[shape])
        assert g.tile_threads == SHAPES[shape] and g.tile_lanes == lanes_of(sc.dim, SPLITS[shape])
        g.step(9)
        assert_same(state(g), want, sc.params.precision)
        g.close()


def test_autotune_leaves_the_scene_as_it_was_and_steps_the_same():
    for sc in scene_set():
        ref = make_sim(sc)
        ref.step(12)
        want = state(ref)
        ref.close()
        g = make_sim(sc)
        g.step(5)
        before = exact_state(g)
        chosen = g.autotune(reps=2)
        assert set(chosen) == set(TILE_SLOTS)
        assert all(t in (64, 128, 256) for t in chosen.values())
        assert chosen["g2p"] <= 128
        assert g.tile_threads == chosen
        cols = 16 if sc.dim == 3 else 4
        assert all(l in (cols, 2 * cols) for l in g.tile_lanes.values())
        assert_identical(exact_state(g), before)  # trial steps leave no trace
        g.step(7)
        assert_same(state(g), want, sc.params.precision)
        g.close()


def test_autotune_at_the_first_step_and_after_the_end():
    sc = scene_set()[0]
    g = make_sim(sc)
    before = exact_state(g)
    g.autotune(reps=1)  # step 0: the trial steps set up the initial grid as step 0 will
    assert_identical(exact_state(g), before)
    g.set_step_limit(3)
    g.step(10)
    assert g.clock()["step"] == 3
    shapes = g.tile_threads
    assert g.autotune(reps=1) == shapes  # no step left to take: shapes kept
    g.close()


def test_invalid_shapes_are_refused():
    from matter_tests_b200.gpu import MtrFailure
    g = make_sim(scene_set()[1])
    for bad in ({"p2g": 48}, {"p2g": 512}, {"g2p": 256}, {"musl": 256}, {"defgrad": 0}):
        with pytest.raises(MtrFailure):
            g.tile_threads = bad
    assert g.tile_threads == {k: 128 for k in TILE_SLOTS}
    for bad in ({"p2g": 8}, {"musl": 64}, {"p2g": 4}):  # 3D: 16 or 32
        with pytest.raises(MtrFailure):
            g.tile_lanes = bad
    assert g.tile_lanes == {"p2g": 16, "musl": 16}
    g.close()


def test_batch_autotune_and_per_group_shapes():
    from matter_tests_b200.gpu import GpuBatch
    scs = scene_set()
    alone = []
    for sc in scs:
        g = make_sim(sc)
        g.step(4)
        alone.append(state(g))
        g.close()
    sims = [make_sim(sc) for sc in scs]
    before = [exact_state(g) for g in sims]
    batch = GpuBatch(sims)
    groups = batch.autotune(reps=2)
    assert sum(gr["members"] for gr in groups) == len(scs)
    for gr in groups:
        assert all(t in (64, 128, 256) for t in gr["tile_threads"].values())
        assert gr["fp32"] in (False, True) and gr["dim"] in (2, 3)
    for g, b in zip(sims, before):
        assert_identical(exact_state(g), b)
    batch.set_tile_threads(0, SHAPES[1])
    lanes = lanes_of(batch.groups()[0]["dim"], (2, 2))
    batch.set_tile_lanes(0, lanes)
    assert batch.groups()[0]["tile_threads"] == SHAPES[1] and batch.groups()[0]["tile_lanes"] == lanes
    batch.step(4)
    for sc, g, ref in zip(scs, sims, alone):
        assert_same(state(g), ref, sc.params.precision)
    batch.close()
    for g in sims:
        g.close()


def test_batch_groups_start_with_their_first_members_shapes():
    from matter_tests_b200.gpu import GpuBatch
    sc = scene_set()[2]
    sims = [make_sim(sc), make_sim(sc)]
    sims[0].tile_threads = SHAPES[0]
    sims[0].tile_lanes = lanes_of(sc.dim, (2, 1))
    batch = GpuBatch(sims)
    gr = batch.groups()
    assert len(gr) == 1 and gr[0]["members"] == 2 and gr[0]["tile_threads"] == SHAPES[0]
    assert gr[0]["tile_lanes"] == lanes_of(sc.dim, (2, 1))
    assert gr[0]["fp32"] == (sc.params.precision == PREC_MIXED)
    assert sc.params.precision in (PREC_FP64, PREC_MIXED)
    batch.close()
    for g in sims:
        g.close()


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED])
def test_tuned_shapes_are_not_slower_than_the_defaults(prec):
    """On the 1M-particle 3D collapse after 20 steps, the shapes mtr_autotune
    picks (3 interleaved repetitions, median, noise margin) against the
    default shapes on the same scene: both timed interleaved, 5 rounds of 4
    profiled steps each (CUDA events per kernel), the median over rounds of
    the tile kernels' summed time.  A 3% allowance covers timing noise."""
    import copy
    from matter_tests_b200 import scenes
    from matter_tests_b200.gpu import GpuSim
    sc = scenes.collapse3d_mui(scale=1.0)
    p = copy.copy(sc.params)
    p.precision = prec
    g = GpuSim(p)
    g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
    g.set_objects(sc.plates, sc.objects)
    g.step(20)
    default = (g.tile_threads, g.tile_lanes)
    g.autotune(3)
    tuned = (g.tile_threads, g.tile_lanes)
    kernels = ("k_p2g", "k_g2p_musl", "k_defgrad")
    times = {"default": [], "tuned": []}
    for _ in range(5):
        for name, (tt, ln) in (("default", default), ("tuned", tuned)):
            g.tile_threads = tt
            g.tile_lanes = ln
            g.profile(1)
            times[name].append(sum(t for k, t in g.profile(4) if k in kernels))
    g.close()
    med = {k: float(np.median(v)) for k, v in times.items()}
    print(prec, default, tuned, med)
    assert med["tuned"] <= 1.03 * med["default"], (tuned, med)


def test_batch_retunes_when_its_grids_double():
    """With re-tuning on (mtr_batch_set_retune), a batch whose scenes fly
    apart (their grids grow past twice their size at the tune) is tuned again
    inside mtr_batch_step; the re-tunes, like the first tune, leave every
    scene as it is when stepped alone.  Without it the same batch is tuned
    only once."""
    import cases
    from matter_tests_b200.gpu import GpuBatch
    scs = []
    for seed in (3, 5):
        # a soft block bursting outwards: its grid grows from ~2.5k nodes to
        # ~50k over 48 steps (the oracle's remesh), four doublings
        sc = cases.apply(cases.block(3, 2, n=4, seed=seed, E=1e3), plastic_model=cases.PM.NoPlasticity)
        d = sc.x - sc.x.mean(0)
        sc.v = 4.0 * d / np.linalg.norm(d, axis=1, keepdims=True)
        scs.append(sc)
    off = [make_sim(sc) for sc in scs]
    b = GpuBatch(off)
    b.autotune(1)
    b.step(48)
    assert b.retunes() == 0
    b.close()
    for g in off:
        g.close()
    sims = [make_sim(sc) for sc in scs]
    b = GpuBatch(sims)
    b.autotune(1)
    b.set_retune(1)
    b.step(48)
    n = b.retunes()
    b.close()
    assert n >= 1, n
    for sc, g in zip(scs, sims):
        alone = make_sim(sc)
        alone.step(48)
        assert_same(state(g), state(alone), sc.params.precision)
        alone.close()
        g.close()
