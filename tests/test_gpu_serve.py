"""The serving loop (matter_tests_b200.serve): requests that arrive while
others run are admitted within the memory budget, join the running batch and
leave it when done, and each result is the same as the request run alone.

Alone and in the mix a request runs the same mixed-precision step; only the
order of the FP32 atomic sums differs, so positions agree to 1e-6 of their
scale and velocities to 1e-4 of theirs after the requested steps."""
import copy

import numpy as np
import pytest

from matter_tests_b200 import scenes
from matter_tests_b200.abi import PREC_MIXED

from gpu_util import needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]


def small_request(rng):
    return scenes.serving_request(rng, n_min=3_000, n_max=40_000)


def alone(req):
    from matter_tests_b200.gpu import GpuSim
    p = copy.copy(req.scene.params)
    p.precision = PREC_MIXED
    g = GpuSim(p)
    sc = req.scene
    g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
    g.set_objects(sc.plates, sc.objects)
    g.step(req.steps)
    out = g.particles()
    ck = g.clock()
    g.close()
    return out, ck


@pytest.mark.parametrize("budget_factor,frame_ms", [(1e3, None), (1.0, None), (1e3, 1.0)])
def test_requests_in_the_mix_match_alone(budget_factor, frame_ms):
    """frame_ms = 1: ticks of 1 to 8 steps, sized by the step-time model."""
    from matter_tests_b200.serve import Server, poisson_requests
    reqs = poisson_requests(6, rate=400.0, seed=11, steps=24, builder=small_request)
    from matter_tests_b200.gpu import footprint
    big = max(footprint(_mixed(r.scene.params), r.scene.x) for r in reqs)
    srv = Server(budget_bytes=int(big * budget_factor), tick_steps=8, frame_ms=frame_ms)
    done = srv.run(reqs)
    assert len(done) == len(reqs)
    assert srv.peak_bytes <= srv.budget  # admission never exceeds the budget
    if budget_factor > 1:
        assert srv.peak_members >= 2  # requests overlap on the GPU
    for r in done:
        ref, ck = alone(r)
        assert r.result["clock"]["step"] == ck["step"] == r.steps
        assert r.result["status"][0] == 0
        ex = np.abs(r.result["x"] - ref["x"]).max() / np.abs(ref["x"]).max()
        ev = np.abs(r.result["v"] - ref["v"]).max() / max(np.abs(ref["v"]).max(), 1e-300)
        assert ex <= 1e-6 and ev <= 1e-4, (r.rid, r.scene.name, ex, ev)
    rep = srv.report(done)
    assert rep["requests"] == len(reqs) and rep["throughput"] > 0


def _mixed(p):
    q = copy.copy(p)
    q.precision = PREC_MIXED
    return q
