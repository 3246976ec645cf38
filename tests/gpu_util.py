"""Helpers for the GPU tests: run a scene on the CUDA path and on the oracle."""
import numpy as np
import pytest

from oracle.checkers import Oracle


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


needs_gpu = pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")


def run_gpu(scene, nsteps, keep_pic_flip=True, graphs=True):
    from matter_tests_b200.gpu import GpuSim
    g = GpuSim(scene.params)
    g.upload(scene.x, scene.v, scene.F, scene.B, scene.scalars)
    g.set_scene_objects(scene)
    if keep_pic_flip:
        g.keep_pic_flip(True)
    if not graphs:
        g.use_graphs(False)
    rc = g.step(nsteps, check=False)
    out = dict(rc=rc, p=g.particles(pic_flip=keep_pic_flip), g=g.grid(), c=g.clock(), status=g.status(),
               plates=g.plates(), sort=g.sort_state())
    g.close()
    return out


def run_oracle(scene, nsteps):
    o = Oracle(scene.params)
    o.set_particles(scene.x, scene.v, scene.F, scene.B, scene.scalars)
    for ls in getattr(scene, "levelsets", ()):
        o.set_levelset(ls)
    o.set_objects(scene.plates, scene.objects)
    n = o.step(nsteps)
    out = dict(n=n, p=o.particles(), g=o.grid(), c=o.clock(), keys=o.keys(), plates=o.plates())
    o.close()
    return out


def run_reference(scene, nsteps, threads=None):
    """The reference compiled from its own sources (oracle/_ref), with OpenMP
    threads; same result layout as run_oracle (keys excepted)."""
    import os
    from oracle.checkers import Reference
    if threads is None:
        try:
            threads = len(os.sched_getaffinity(0))
        except Exception:
            threads = os.cpu_count() or 1
        threads = max(1, min(threads, 32))
    r = Reference(scene.params, n_threads=threads)
    r.set_particles(scene.x, scene.v, scene.F, scene.B, scene.scalars)
    r.set_objects(scene.plates, scene.objects)
    n = r.step(nsteps)
    out = dict(n=n, p=r.particles(), g=r.grid(), c=r.clock(), plates=r.plates())
    r.close()
    return out


def oracle_sensitivity(scene, nsteps, ulps=4.0, seed=11, runner=None):
    """How far the reference's own algorithm moves, per field, when the initial
    positions, velocities and affine matrices are perturbed by a few ulps (the
    size of the reordering error of GPU atomics).  Fields the reference computes
    through cancellation-prone closed forms (the mu(I) quadratic root at
    plasticity.cpp:388, tip projections, viscosity = (mu_i - mu_1) p / gamma)
    cannot be reproduced more closely than this by any implementation."""
    import copy
    rng = np.random.default_rng(seed)
    sc = copy.copy(scene)
    eps = ulps * np.finfo(np.float64).eps
    sc.x = scene.x * (1.0 + eps * rng.choice([-1.0, 1.0], size=scene.x.shape))
    v = np.zeros_like(scene.x) if scene.v is None else scene.v
    sc.v = v * (1.0 + eps * rng.choice([-1.0, 1.0], size=v.shape))
    if scene.B is not None:
        sc.B = scene.B * (1.0 + eps * rng.choice([-1.0, 1.0], size=scene.B.shape))
    run = runner or run_oracle
    a, b = run(scene, nsteps), run(sc, nsteps)
    from matter_tests_b200.abi import SCALARS
    out = {k: np.abs(a["p"]["scalars"][:, i] - b["p"]["scalars"][:, i]).max() for i, k in enumerate(SCALARS)}
    for k in ("x", "v", "F", "B", "pic", "flip"):
        out[k] = np.abs(a["p"][k] - b["p"][k]).max()
    if tuple(a["g"]["dims"]) == tuple(b["g"]["dims"]):
        for k in ("mass", "v", "flip"):
            out["grid " + k] = np.abs(a["g"][k] - b["g"][k]).max()
    return out


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max(initial=0.0)
    diff = np.abs(a - b).max(initial=0.0)
    if scale == 0.0:
        return diff
    return diff / scale


def assert_close(name, a, b, rel, report=None, allowance=0.0):
    e = rel_err(a, b)
    if allowance:
        scale = np.abs(np.asarray(b, dtype=np.float64)).max(initial=0.0)
        e = max(0.0, np.abs(np.asarray(a) - np.asarray(b)).max(initial=0.0) - allowance) / (scale or 1.0)
    ok = bool(np.all(np.isfinite(a) == np.isfinite(b))) and e <= rel
    if report is not None:
        report.append((name, e, rel, ok))
        return e
    assert np.all(np.isfinite(a) == np.isfinite(b)), f"{name}: finiteness differs"
    assert e <= rel, f"{name}: relative error {e:.3e} > {rel:.1e}"
    return e


def compare_states(gpu, orc, rel=1e-10, fields=("x", "v", "F", "B", "pic", "flip"), grid=True, sens=None,
                   sens_factor=100.0):
    """Every field must agree to `rel` of its scale plus, when `sens` is given,
    sens_factor times the oracle's own spread under a few-ulp input
    perturbation (oracle_sensitivity).  One-step tests use rel = 1e-10, where
    that spread is ~1e-15 for the state fields; over several steps friction
    and yield thresholds make some grid nodes and plastic scalars
    discontinuous in their inputs, and the allowance measures exactly that."""
    errs = {}
    assert gpu["c"]["step"] == orc["c"]["step"], (gpu["c"], orc["c"])
    assert gpu["c"]["frame"] == orc["c"]["frame"]
    # the oracle reports the reference's exit flag apart from the end of time
    assert gpu["c"]["done"] == int(orc["c"]["done"] or orc["c"]["exit"])
    rep = []
    errs["time"] = assert_close("time", gpu["c"]["time"], orc["c"]["time"], rel, rep)
    errs["dt"] = assert_close("dt", gpu["c"]["dt"], orc["c"]["dt"], rel, rep)
    allow = (lambda k: sens_factor * sens.get(k, 0.0)) if sens is not None else (lambda k: 0.0)
    for k in fields:
        if k in gpu["p"]:
            errs[k] = assert_close(k, gpu["p"][k], orc["p"][k], rel, rep, allow(k))
    from matter_tests_b200.abi import SCALARS
    for i, k in enumerate(SCALARS):
        a, b = gpu["p"]["scalars"][:, i], orc["p"]["scalars"][:, i]
        scale = np.abs(b).max(initial=0.0)
        tol = rel * scale + (sens_factor * sens[k] if sens is not None else 0.0)
        diff = np.abs(a - b).max(initial=0.0)
        ok = bool(np.all(np.isfinite(a) == np.isfinite(b))) and diff <= tol
        rep.append((k + " (abs)", diff, tol, ok))
        errs[k] = diff / scale if scale > 0 else diff
    if grid:
        assert tuple(gpu["g"]["dims"]) == tuple(orc["g"]["dims"])
        for k in ("x", "y", "z"):
            assert np.array_equal(gpu["g"][k], orc["g"][k]), f"grid axis {k} not bit-identical"
        errs["grid_mass"] = assert_close("grid mass", gpu["g"]["mass"], orc["g"]["mass"], rel, rep, allow("grid mass"))
        errs["grid_v"] = assert_close("grid v", gpu["g"]["v"], orc["g"]["v"], rel, rep, allow("grid v"))
        errs["grid_flip"] = assert_close("grid flip", gpu["g"]["flip"], orc["g"]["flip"], rel, rep, allow("grid flip"))
    bad = [r for r in rep if not r[3]]
    assert not bad, "parity failures: " + "; ".join(f"{n}: {e:.3e} > {t:.1e}" for n, e, t, _ in bad) + \
        " | all: " + ", ".join(f"{n}={e:.1e}" for n, e, _, _ in rep)
    return errs
