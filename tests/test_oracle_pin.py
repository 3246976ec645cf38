"""Pins the C restatement (oracle/mpm_oracle.c) to the reference itself.

The reference's own src/simulation/*.cpp are compiled from source by
oracle/Makefile (3D and 2D, quadratic and cubic splines; Eigen replaced by the
project-written subset in oracle/shim; 2D from a copy of src/ whose tools.hpp
leaves THREEDIM undefined) and run on the same seeded scene as the
restatement.  Both evaluate the same expressions in the same order, so the
particle state, grid and clock must agree bit for bit after several steps.
The restatement then serves as the checker for the CUDA path.
"""
import numpy as np
import pytest

from matter_tests_b200 import scenes
from matter_tests_b200.abi import BC
from oracle.checkers import Oracle, Reference, reference_available

import cases

DIMS = [3, 2]


def _need(dim, deg):
    if not reference_available(dim, deg):
        pytest.skip(f"reference build {dim}D q{deg} (oracle/_ref) unavailable")


def _block(dim, deg):
    return cases.block(dim, deg, n=5 if dim == 3 else 8)


def _run_both(sc, nsteps):
    res = []
    for cls in (Oracle, Reference):
        c = cls(sc.params)
        c.set_particles(sc.x, sc.v, sc.F, sc.B, sc.scalars)
        c.set_objects(sc.plates, sc.objects)
        n = c.step(nsteps)
        res.append(dict(n=n, p=c.particles(), g=c.grid(), c=c.clock(),
                        plates=[(q.pos_object, q.pos_lower, q.pos_upper, tuple(q.v_object)) for q in c.plates()]))
        c.close()
    return res


def _assert_identical(o, r):
    assert o["n"] == r["n"]
    for k in ("time", "dt", "step", "frame", "done", "exit"):
        assert o["c"][k] == r["c"][k], k
    for k in ("x", "v", "F", "B", "scalars", "pic", "flip"):
        assert np.array_equal(o["p"][k], r["p"][k], equal_nan=True), (k, np.nanmax(np.abs(o["p"][k] - r["p"][k])))
    assert o["g"]["dims"] == r["g"]["dims"]
    for k in ("x", "y", "z", "mass", "v", "flip"):
        assert np.array_equal(o["g"][k], r["g"][k], equal_nan=True), k
    assert o["plates"] == r["plates"]


@pytest.mark.parametrize("dim", DIMS)
@pytest.mark.parametrize("deg", [2, 3])
@pytest.mark.parametrize("model", sorted(cases.MODEL_CASES))
def test_models_bitexact(model, deg, dim):
    _need(dim, deg)
    sc = cases.apply(_block(dim, deg), **cases.MODEL_CASES[model])
    sc = cases.box_plates(sc, BC.SlipFree, 0.3)
    o, r = _run_both(sc, 3)
    _assert_identical(o, r)


@pytest.mark.parametrize("dim", DIMS)
@pytest.mark.parametrize("deg", [2, 3])
@pytest.mark.parametrize("transfer", sorted(cases.TRANSFER_CASES))
def test_transfers_bitexact(transfer, deg, dim):
    _need(dim, deg)
    sc = cases.apply(_block(dim, deg), plastic_model=cases.PM.DP, M=0.6, **cases.TRANSFER_CASES[transfer])
    sc = cases.box_plates(sc, BC.SlipStick, 0.4)
    o, r = _run_both(sc, 3)
    _assert_identical(o, r)


@pytest.mark.parametrize("dim", DIMS)
@pytest.mark.parametrize("bc", [BC.NoSlip, BC.SlipStick, BC.SlipFree])
@pytest.mark.parametrize("moving", [False, True])
def test_plates_bitexact(bc, moving, dim):
    _need(dim, 2)
    sc = cases.apply(_block(dim, 2), plastic_model=cases.PM.NoPlasticity)
    sc = cases.box_plates(sc, bc, 0.35, moving=moving)
    o, r = _run_both(sc, 4)
    _assert_identical(o, r)


@pytest.mark.parametrize("dim,obj", [(d, o) for d in DIMS for o in sorted(cases.object_cases(d))])
def test_objects_bitexact(dim, obj):
    _need(dim, 2)
    sc = cases.apply(_block(dim, 2), plastic_model=cases.PM.DPVisc, M=0.5, use_mibf=1)
    sc.objects = cases.object_cases(dim)[obj]
    o, r = _run_both(sc, 3)
    _assert_identical(o, r)


@pytest.mark.parametrize("builder,scale,nsteps", [("collapse3d_mui", 0.12, 5), ("incline3d_mcc", 0.12, 5),
                                                  ("collapse2d", 0.25, 20)])
def test_workloads_bitexact(builder, scale, nsteps):
    sc = scenes.WORKLOADS[builder](scale=scale)
    _need(sc.params.dim, sc.params.spline_deg)
    o, r = _run_both(sc, nsteps)
    _assert_identical(o, r)


@pytest.mark.parametrize("dim", DIMS)
def test_grid_reference_point_and_gravity_ramp(dim):
    _need(dim, 3)
    sc = cases.apply(cases.block(dim, 3, n=4 if dim == 3 else 7), plastic_model=cases.PM.DPMui, gravity_special=1,
                     gravity_time=1e-3, grid_reference_point=(0.0, -0.02, 0.0))
    sc.plates = [scenes.make_plate(-0.005, cases.PlateType.bottom, BC.SlipFree, 0.2)]
    o, r = _run_both(sc, 4)
    _assert_identical(o, r)


@pytest.mark.parametrize("dim", DIMS)
def test_end_of_simulation_clock(dim):
    """simulate() stops at final_time with a clipped last dt (update_dt.cpp:34-35)."""
    _need(dim, 2)
    sc = cases.apply(cases.block(dim, 2, n=3 if dim == 3 else 5), plastic_model=cases.PM.DP, M=0.6)
    dt_max = 0.5 * sc.params.dx / np.sqrt(sc.params.E / sc.params.rho)
    sc.params.fps = 1.0 / (3.5 * dt_max)
    sc.params.end_frame = 1
    o, r = _run_both(sc, 10)
    _assert_identical(o, r)
    assert o["n"] == 4 and o["c"]["done"] == 1


@pytest.mark.parametrize("dim", DIMS)
@pytest.mark.parametrize("deg,musl,fr", [(2, 0, -2.0), (3, 1, -0.95), (2, 0, 0.9)])
def test_periodic_bitexact(deg, musl, fr, dim):
    """Periodic boundaries (remeshFixed(4), PBCAddParticles(4) and the wrap in
    positionUpdate) over 12 steps in which particles cross x = Lx."""
    _need(dim, deg)
    sc = cases.periodic(dim, deg, musl=musl, flip_ratio=fr)
    o, r = _run_both(sc, 12)
    _assert_identical(o, r)
    assert o["p"]["x"][:, 0].min() >= 0.0 and o["p"]["x"][:, 0].max() <= sc.params.L[0]
