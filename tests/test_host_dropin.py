"""The C++ drop-in Simulation (matter_tests_b200/host): setup files written
for the reference build against it unchanged, its objects describe themselves
to the device as the Python scenes do, its sampler keeps the Poisson-disk
distance, it fails loudly without a GPU, and on a GPU its advanceStep() and
simulate() reproduce the oracle and pass the reference's own known-answer
tests (tests/tests.cpp, built by oracle/Makefile's kat target)."""
import math
import os
import subprocess

import numpy as np
import pytest

from matter_tests_b200 import abi
from matter_tests_b200.abi import BC, ObjectKind, PlasticModel, PlateType
from gpu_util import compare_states, gpu_available, oracle_sensitivity, run_oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "matter_tests_b200", "host")
SETUPS = os.path.join(ROOT, "tests", "host_setups")
LIB = os.path.join(ROOT, "matter_tests_b200", "libmatter_gpu.so")
KAT = os.path.join(ROOT, "oracle", "_ref", "kat", "kat")
# copies of the reference's setup and test files, staged by oracle/Makefile (`stage`)
SETUP_COPIES = os.path.join(ROOT, "oracle", "_ref", "setups")


def build_setup(src, out_dir, dim=3, deg=2):
    """Builds one setup file with the host Makefile; returns the binary."""
    if not os.path.exists(LIB):
        from matter_tests_b200 import build
        build.build()
    out = os.path.join(str(out_dir), f"{os.path.splitext(os.path.basename(src))[0]}_{dim}d_q{deg}")
    r = subprocess.run(["make", "-s", "-C", HOST, f"SETUP={src}", f"OUT={out}", f"DIM={dim}", f"DEG={deg}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


# ---------------------------------------------------------------- CPU tests

@pytest.mark.parametrize("dim,deg", [(3, 2), (3, 3), (2, 2), (2, 3)])
def test_host_builds_for_every_dimension_and_spline(tmp_path, dim, deg):
    assert os.path.exists(build_setup(os.path.join(SETUPS, "host_parity.cpp"), tmp_path, dim, deg))


@pytest.mark.skipif(not os.path.isdir(SETUP_COPIES), reason="staged reference setup files not present")
@pytest.mark.parametrize("setup", ["src/mpm.cpp", "examples/collapse.cpp", "examples/cube_rotating.cpp",
                                   "tests/tests.cpp"])
def test_reference_setup_files_compile_unchanged(tmp_path, setup):
    """The reference's own setup and test files compile, as they are, against
    the host headers (fed on standard input from a directory whose quoted
    includes resolve to the host tree)."""
    if setup.startswith("tests/"):
        work = tmp_path / "tests"
        work.mkdir()
        os.symlink(HOST, tmp_path / "src")
        extra = ["-I", os.path.join(ROOT, "tests", "host_shim")]
    else:
        work = HOST
        extra = []
    with open(os.path.join(SETUP_COPIES, setup)) as f:
        r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-fsyntax-only", "-w", "-I", HOST, "-I",
                            os.path.join(ROOT, "include"), *extra, "-x", "c++", "-"], stdin=f, cwd=str(work),
                           capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.fixture(scope="module")
def describe_output(tmp_path_factory):
    d = tmp_path_factory.mktemp("describe")
    outs = {}
    for dim in (3, 2):
        exe = build_setup(os.path.join(SETUPS, "host_describe.cpp"), d, dim, 2)
        pts = os.path.join(str(d), f"pts{dim}.bin")
        r = subprocess.run([exe, "0.01" if dim == 3 else "0.004", pts], capture_output=True, text=True, check=True)
        lines = [l for l in r.stdout.splitlines() if l and l[0].isdigit()]
        outs[dim] = ([np.array([float(t) for t in l.split()]) for l in lines], np.fromfile(pts))
    return outs


def test_object_descriptors_match_the_python_scene_builders(describe_output):
    objs3, _ = describe_output[3]
    objs2, _ = describe_output[2]
    R = np.array([[0.8, -0.6, 0.0], [0.6, 0.8, 0.0], [0.0, 0.0, 1.0]])
    want3 = [
        abi.make_object(ObjectKind.Bump, BC.SlipFree, 0.1),
        abi.make_object(ObjectKind.Ground, BC.SlipStick, 0.2, [-0.25]),
        abi.make_object(ObjectKind.Ramp, BC.NoSlip, 0.3),
        abi.make_object(ObjectKind.Curve, BC.SlipFree, 0.4),
        abi.make_object(ObjectKind.Gate, BC.SlipStick, 0.5, [0.03]),
        abi.make_object(ObjectKind.Silo, BC.SlipFree, 0.6, [0.07]),
        abi.make_object(ObjectKind.BoxRotated, BC.NoSlip, 0.7, [1, 2, 3, 0.1, 0.2, 0.3, *R.T.reshape(-1)]),
        abi.make_object(ObjectKind.TerrainGauss, BC.SlipFree, 0.45, [-0.5, 2, 0.1, 0.2, 0.3, 0.4, 1.1, 1.2, 1.3, 1.4]),
    ]
    flat = lambda o: np.array([o.kind, o.bc, o.friction, *list(o.prm)])
    assert len(objs3) == len(want3)
    for got, w in zip(objs3, want3):
        np.testing.assert_array_equal(got, flat(w))
    # 2D: no silo and no rotated box
    want2 = [w for w in want3 if w.kind not in (ObjectKind.Silo, ObjectKind.BoxRotated)]
    assert len(objs2) == len(want2)
    for got, w in zip(objs2, want2):
        np.testing.assert_array_equal(got, flat(w))


@pytest.mark.parametrize("dim", [3, 2])
def test_sampler_keeps_the_disk_radius_and_sets_dx(describe_output, dim):
    from scipy.spatial import cKDTree
    _, raw = describe_output[dim]
    n, dx, vol = int(raw[0]), raw[1], raw[2]
    x = raw[3:].reshape(n, dim)
    r = 0.01 if dim == 3 else 0.004
    box = np.array([0.3, 0.2, 0.1][:dim])
    assert np.all(x >= 0) and np.all(x <= box)
    dist, _ = cKDTree(x).query(x, k=2)
    assert dist[:, 1].min() >= r * (1 - 1e-12)
    # maximal packing: no empty ball of radius 2r inside the box (Bridson's cover)
    probe = np.random.default_rng(0).uniform(2 * r, box - 2 * r, size=(2000, dim))
    assert cKDTree(x).query(probe)[0].max() < 2 * r
    ppc = 8 if dim == 3 else 6
    np.testing.assert_allclose(dx, (ppc / n * np.prod(box)) ** (1.0 / dim), rtol=1e-14)
    np.testing.assert_allclose(vol, dx ** dim / ppc, rtol=1e-14)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU failure")
def test_host_fails_loudly_without_a_gpu(tmp_path):
    exe = build_setup(os.path.join(SETUPS, "host_parity.cpp"), tmp_path)
    r = subprocess.run([exe, "steps", "1", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 1
    assert "no CUDA device" in r.stdout + r.stderr
    assert not (tmp_path / "final.bin").exists()


# ---------------------------------------------------------------- GPU tests

def read_state(path, dim, with_clock):
    raw = np.fromfile(path)
    n = int(raw[0])
    o = 1
    out = {}
    for k, w in (("x", dim), ("v", dim), ("F", dim * dim), ("B", dim * dim), ("scalars", 6)):
        out[k] = raw[o:o + n * w].reshape((n, dim, dim) if w == dim * dim else (n, w))
        o += n * w
    if with_clock:
        out["time"], out["step"] = raw[o], int(raw[o + 1])
    return out


def parity_scene(init, dim, deg, end_frame):
    """The scene host_parity.cpp sets up, restated through the Python ABI."""
    from matter_tests_b200.scenes import Scene
    p = abi.default_params(dim, deg)
    p.end_frame, p.fps, p.cfl, p.flip_ratio, p.use_musl = end_frame, 400.0, 0.5, -0.95, 1
    p.gravity[0], p.gravity[1] = 2.0, -9.81
    p.plastic_model, p.use_pradhana = PlasticModel.DPVisc, 1
    p.M, p.q_cohesion = math.tan(30.0 * math.pi / 180.0), 50.0
    p.perzyna_exp, p.perzyna_visc = 1.0, 0.01
    p.E, p.nu, p.rho = 1e6, 0.3, 1500.0
    p.dx = 0.02
    p.particle_volume = math.pow(p.dx, dim) / math.pow(2, dim)
    p.particle_mass = p.rho * p.particle_volume
    for a in range(3):
        p.grid_reference_point[a] = 0.0 if a < dim else 2e10
    plates = [abi.make_plate(0.0, PlateType.bottom, BC.SlipStick, 0.35),
              abi.make_plate(0.01, PlateType.left, BC.SlipFree, 0.2),
              abi.make_plate(0.3, PlateType.right, BC.NoSlip)]
    objects = [abi.make_object(ObjectKind.Bump, BC.SlipFree, 0.3)]
    if dim == 3:
        c, s = math.cos(0.3), math.sin(0.3)
        objects.append(abi.make_object(ObjectKind.BoxRotated, BC.SlipStick, 0.25,
                                       [0.2, 0.16, 0.06, 0.03, 0.02, 0.2, c, s, 0, -s, c, 0, 0, 0, 1]))
    return Scene("host_parity", p, init["x"].copy(), init["v"].copy(), init["F"].copy(), init["B"].copy(),
                 init["scalars"].copy(), plates, objects)


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("mode,n", [("steps", 3), ("frames", 2)])
@pytest.mark.parametrize("dim,deg", [(3, 2), (2, 3)])
def test_host_simulation_matches_the_oracle(tmp_path, mode, n, dim, deg):
    exe = build_setup(os.path.join(SETUPS, "host_parity.cpp"), tmp_path, dim, deg)
    r = subprocess.run([exe, mode, str(n), str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    init = read_state(tmp_path / "init.bin", dim, False)
    fin = read_state(tmp_path / "final.bin", dim, True)
    sc = parity_scene(init, dim, deg, end_frame=n if mode == "frames" else 1000)
    nsteps = n if mode == "steps" else 1 << 20
    o = run_oracle(sc, nsteps)
    assert o["c"]["step"] == fin["step"]
    if mode == "frames":
        assert o["c"]["frame"] == n and o["c"]["done"]
    assert abs(fin["time"] - o["c"]["time"]) <= 1e-12 * o["c"]["time"]
    gpu = {"p": {k: fin[k] for k in ("x", "v", "F", "B", "scalars")},
           "c": {"step": fin["step"], "frame": o["c"]["frame"], "done": int(o["c"]["done"] or o["c"]["exit"]),
                 "time": fin["time"], "dt": o["c"]["dt"]}}
    sens = oracle_sensitivity(sc, o["c"]["step"])
    compare_states(gpu, o, 1e-9, fields=("x", "v", "F", "B"), grid=False, sens=sens)


def read_ply(path):
    """(property names, rows) of a binary little-endian PLY file of doubles."""
    with open(path, "rb") as f:
        names, n = [], 0
        assert f.readline() == b"ply\n"
        assert f.readline() == b"format binary_little_endian 1.0\n"
        for line in iter(f.readline, b"end_header\n"):
            t = line.decode().split()
            if t[0] == "element":
                assert t[1] == "vertex"
                n = int(t[2])
            elif t[0] == "property":
                assert t[1] == "double"
                names.append(t[2])
        rows = np.frombuffer(f.read(), dtype="<f8")
    return names, rows.reshape(n, len(names))


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("dim,deg", [(3, 2), (2, 3)])
def test_saved_frames_have_the_reference_columns_and_the_run_state(tmp_path, dim, deg):
    """simulate() with save_sim: the particle file of every frame (written from
    a GPU snapshot while the next frame steps) and the grid file carry the
    reference's properties in its order (save_data.cpp:7-255); the first file
    holds the initial state and the last one the final state."""
    exe = build_setup(os.path.join(SETUPS, "host_parity.cpp"), tmp_path, dim, deg)
    n = 3
    r = subprocess.run([exe, "saved", str(n), str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    init = read_state(tmp_path / "init.bin", dim, False)
    fin = read_state(tmp_path / "final.bin", dim, True)
    run = tmp_path / "run"
    xyz, vel = ["x", "y", "z"][:dim], ["vx", "vy", "vz"][:dim]
    want = xyz + vel + ["p", "q", "Je", "eps_pl_vol", "eps_pl_dev", "delta_gamma"]  # DPVisc without MIBF
    for f in range(n + 1):
        names, rows = read_ply(run / f"particles_f{f}.ply")
        assert names == want, names
        assert rows.shape[0] == init["x"].shape[0]
    _, first = read_ply(run / "particles_f0.ply")
    assert np.array_equal(first[:, :dim], init["x"]) and np.array_equal(first[:, dim:2 * dim], init["v"])
    _, last = read_ply(run / f"particles_f{n}.ply")
    assert np.array_equal(last[:, :dim], fin["x"]) and np.array_equal(last[:, dim:2 * dim], fin["v"])
    assert np.array_equal(last[:, 2 * dim + 3], fin["scalars"][:, 1])  # eps_pl_vol
    assert np.array_equal(last[:, 2 * dim + 4], fin["scalars"][:, 0])  # eps_pl_dev
    je = np.linalg.det(fin["F"])
    assert np.abs(last[:, 2 * dim + 2] - je).max() <= 1e-12
    gnames, grows = read_ply(run / f"grid_f{n}.ply")
    assert gnames == xyz + vel + ["mass"]
    assert grows[:, 2 * dim].sum() > 0
    assert (run / "last_written.txt").read_text().strip() == str(n)


@pytest.mark.parametrize("dim", [3, 2])
def test_user_object_setup_builds(tmp_path, dim):
    assert os.path.exists(build_setup(os.path.join(SETUPS, "host_baked.cpp"), tmp_path, dim, 2))


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("dim", [3, 2])
def test_user_object_is_baked_and_steers_like_the_builtin(tmp_path, dim):
    """A user subclass of ObjectGeneral (inside()/normal() only) is baked into a
    dense level set at dx/4 and steers a falling block like the built-in
    analytic object it delegates to: final positions within 2% of dx on
    average and 0.5 dx at most."""
    exe = build_setup(os.path.join(SETUPS, "host_baked.cpp"), tmp_path, dim, 2)
    out = {}
    for mode in ("builtin", "user"):
        path = tmp_path / f"{mode}.bin"
        r = subprocess.run([exe, mode, str(path)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        raw = np.fromfile(path)
        out[mode] = raw[1:].reshape(int(raw[0]), dim)
    err = np.abs(out["user"] - out["builtin"])
    assert err.mean() <= 0.02 * 0.01 and err.max() <= 0.5 * 0.01, (err.mean(), err.max())


KATS = ["BoundaryTest.AnalyticSlipFree", "BoundaryTest.AnalyticSlipStick", "CoulombFrictionTest.PlateSlipFree",
        "CoulombFrictionTest.PlateSlipStick", "CoulombFrictionTest.GeneralSlipFree",
        "CoulombFrictionTest.GeneralSlipStick", "BoundaryTest.MIBF", "ElasticityTest.BulkModulus",
        "EnergyTest.Rotation", "CollapseTest.DruckerPragerOne", "CollapseTest.DruckerPragerTwo"]


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
@pytest.mark.skipif(not os.path.exists(KAT), reason="oracle/_ref/kat/kat not built (needs the reference tree)")
@pytest.mark.parametrize("name", KATS)
def test_reference_known_answer_tests_on_the_gpu(name, tmp_path):
    """Each TEST of the reference's tests/tests.cpp, run through the host
    Simulation on the GPU, meets the reference's own tolerance."""
    r = subprocess.run([KAT, f"--gtest_filter={name}"], capture_output=True, text=True, timeout=1500,
                       cwd=str(tmp_path))
    tail = "\n".join(l for l in r.stdout.splitlines() if "diff" in l or "Failure" in l or "|" in l or "[" in l)
    assert r.returncode == 0 and f"[       OK ] {name}" in r.stdout, tail[-3000:] + r.stderr[-2000:]
