"""Frame output (mtr_frame_begin / mtr_frame_wait): the rows of the particle
file (save_data.cpp:7-171), built on the GPU behind the steps and copied out
while the context keeps stepping.

Checked against the state downloaded at the same step: positions, velocities
and the plastic scalars bit for bit; p, q and Je against numpy from the
downloaded F (Hencky: tau = U diag(2 mu ln s + lambda sum ln s) U^T;
Neo-Hookean: tau = mu (F F^T - I) + lambda ln J I), to 1e-9 of the stress
scale in FP64 and 1e-5 with the FP32 stress of the mixed path."""
import numpy as np
import pytest

import cases
from matter_tests_b200.abi import BC, ElasticModel, PREC_FP64, PREC_MIXED

from gpu_util import needs_gpu
from test_gpu_batch import make_sim

pytestmark = [pytest.mark.gpu, needs_gpu]


def frame_scenes():
    out = []
    a = cases.apply(cases.block(3, 3, n=5), plastic_model=cases.PM.DPMui, use_musl=1, flip_ratio=-0.95)
    out.append(cases.box_plates(a, BC.SlipStick, 0.4))
    b = cases.apply(cases.block(2, 2, n=8, seed=5), plastic_model=cases.PM.DP, M=0.6, flip_ratio=-2.0)
    out.append(cases.box_plates(b, BC.SlipFree, 0.3))
    c = cases.apply(cases.block(3, 2, n=5, seed=6), plastic_model=cases.PM.MCCVisc, M=1.2, p0=3e3,
                    perzyna_visc=2e-4, use_mibf=1)
    out.append(cases.box_plates(c, BC.SlipStick, 0.3))
    d = cases.apply(cases.block(3, 2, n=5, seed=7), plastic_model=cases.PM.NoPlasticity,
                    elastic_model=ElasticModel.NeoHookean)
    out.append(cases.box_plates(d, BC.NoSlip, 0.0))
    e = cases.apply(cases.block(3, 3, n=5, seed=8), plastic_model=cases.PM.DPMui, use_musl=1, flip_ratio=-0.95)
    e.params.precision = PREC_MIXED
    out.append(cases.box_plates(e, BC.SlipStick, 0.4))
    return out


def expected_names(p):
    d = p.dim
    names = ["x", "y", "z"][:d] + ["vx", "vy", "vz"][:d] + ["p", "q", "Je"]
    pm = p.plastic_model
    if pm != cases.PM.NoPlasticity:
        names += ["eps_pl_vol", "eps_pl_dev", "delta_gamma"]
        mui = pm in (cases.PM.DPMui, cases.PM.MCCMui)
        if (pm in (cases.PM.DPVisc, cases.PM.MCCVisc) and p.use_mibf) or mui:
            names.append("muI")
        if mui:
            names.append("viscosity")
    return names


def stress(p, F):
    mu = p.E / (2 * (1 + p.nu))
    lam = p.nu * p.E / ((1 + p.nu) * (1 - 2 * p.nu))
    d = F.shape[-1]
    if p.elastic_model == ElasticModel.NeoHookean:
        J = np.linalg.det(F)
        tau = mu * (F @ np.swapaxes(F, 1, 2) - np.eye(d)) + (lam * np.log(J))[:, None, None] * np.eye(d)
    else:
        U, s, _ = np.linalg.svd(F)
        ls = np.log(s)
        e = 2 * mu * ls + lam * ls.sum(axis=1, keepdims=True)
        tau = np.einsum("nij,nj,nkj->nik", U, e, U)
    pr = -np.trace(tau, axis1=1, axis2=2) / d
    dev = tau + pr[:, None, None] * np.eye(d)
    c = 1.5 if p.use_mises_q else 0.5
    q = np.sqrt(c * (dev * dev).sum(axis=(1, 2)))
    return pr, q, np.linalg.det(F)


@pytest.mark.parametrize("k", range(5))
def test_frame_rows_match_the_state_of_their_step(k):
    sc = frame_scenes()[k]
    p = sc.params
    g = make_sim(sc)
    g.step(4)
    want = g.particles()
    g.frame_begin()
    g.step(3)  # the snapshot is taken behind step 4; these steps run while it is copied
    rows, names, ck = g.frame_wait()
    assert names == expected_names(p)
    assert ck["step"] == 4 and g.clock()["step"] == 7
    d = p.dim
    col = {n: rows[:, i] for i, n in enumerate(names)}
    assert rows.shape == (sc.Np, len(names))
    assert np.array_equal(rows[:, :d], want["x"])
    assert np.array_equal(rows[:, d:2 * d], want["v"])
    sc_idx = {"eps_pl_vol": 1, "eps_pl_dev": 0, "delta_gamma": 3, "viscosity": 4, "muI": 5}
    for n, i in sc_idx.items():
        if n in col:
            assert np.array_equal(col[n], want["scalars"][:, i]), n
    pr, q, je = stress(p, want["F"])
    tol = 1e-9 if p.precision == PREC_FP64 else 1e-5
    scale = max(np.abs(pr).max(), np.abs(q).max(), 1e-300)
    assert np.abs(col["p"] - pr).max() <= tol * scale
    assert np.abs(col["q"] - q).max() <= tol * scale
    assert np.abs(col["Je"] - je).max() <= 1e-12
    g.close()


def test_frame_wait_without_a_snapshot_is_refused():
    from matter_tests_b200.gpu import MtrFailure
    g = make_sim(frame_scenes()[1])
    g.step(2)
    with pytest.raises(MtrFailure):
        g.frame_wait()
    g.frame_begin()
    g.frame_begin()  # a second snapshot waits for the first copy, then replaces it
    rows, names, ck = g.frame_wait()
    assert ck["step"] == 2 and rows.shape[0] == g.Np
    with pytest.raises(MtrFailure):
        g.frame_wait()  # already collected
    g.close()


def test_grid_friction_with_mibf():
    sc = frame_scenes()[2]
    g = make_sim(sc)
    g.step(2)
    grid = g.grid()
    fr = g.grid_friction()
    assert fr.shape == grid["mass"].shape
    m = grid["mass"] > 0
    assert np.all(np.isfinite(fr[m])) and fr[m].min() > 0
    g.close()
    g2 = make_sim(frame_scenes()[1])
    g2.step(1)
    from matter_tests_b200.gpu import MtrFailure
    with pytest.raises(MtrFailure):
        g2.grid_friction()  # no MIBF: no grid friction
    g2.close()
