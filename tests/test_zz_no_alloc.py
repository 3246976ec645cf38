"""mtr_p2g_noalloc: the particle-to-grid transfer for callers that cannot
allocate device memory where they call it (code under CUDA-graph capture,
solvers inside a framework that owns all device memory through its own pool,
real-time loops).  It keeps its sort, tile and accumulator scratch in one fixed
device array, so these tests check that

* it reproduces both the grid the regular step (mtr_step through mtr_ctx)
  deposits and the oracle's P2G on the same grid, on two calls in a row whose
  particle counts and grids differ (the second call must not see the first
  call's sort keys, tile ranges or accumulators);
* it works at exactly its documented capacity (2^18 particles, 2^17 nodes);
* particles outside the grid are dropped without disturbing the others, and
  the call's status word says so (and the next clean call's does not);
* it refuses requests larger than the array.

This file is collected last on purpose: a failure here stops a -x run only
after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from matter_tests_b200 import abi
from matter_tests_b200.gpu import GpuSim, load_library
from oracle.checkers import p2g_grid

import cases
from gpu_util import needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

REL = 1e-10
MTR_ERR_TOO_LARGE = -8
MTR_STATUS_STENCIL_OOB = 0x0002
MAX_PARTICLES = 1 << 18
MAX_NODES = 1 << 17


def _scene(dim, deg, n, seed):
    sc = cases.block(dim, deg, n=n, seed=seed, gravity=(0.0, 0.0, 0.0))
    sc.F = None          # F = I: zero stress, so the step's grid velocity is the P2G velocity
    sc.scalars = None
    sc.params.flip_ratio = -2.0  # APIC: the B term is part of the transfer
    sc.plates, sc.objects = [], []
    return sc


def _step_grid(sc):
    g = GpuSim(sc.params)
    g.upload(sc.x, sc.v, None, sc.B, None)
    g.set_objects([], [])
    g.step(1)
    grid = g.grid()
    g.close()
    return grid


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class _Call:
    """Device copies of one scene's inputs and a grid, and one call of the entry point."""

    def __init__(self, params, x, v, B, gx, gy, gz, dims):
        import torch
        self.dev = torch.device("cuda", 0)
        self.params = params
        d = params.dim
        n = x.shape[0]
        self.n, self.d = n, d
        self.x = torch.tensor(np.ascontiguousarray(x.T), device=self.dev)
        self.v = torch.tensor(np.ascontiguousarray(v.T), device=self.dev)
        b_rm = B.reshape(n, d, d).transpose(0, 2, 1).reshape(n, d * d)  # host layout is column-major
        self.B = torch.tensor(np.ascontiguousarray(b_rm.T), device=self.dev)
        self.gx = torch.tensor(gx, device=self.dev)
        self.gy = torch.tensor(gy, device=self.dev)
        self.gz = torch.tensor(gz if d == 3 else np.zeros(1), device=self.dev)
        self.dims = (C.c_uint32 * 3)(*[int(a) for a in dims])
        self.G = int(dims[0]) * int(dims[1]) * (int(dims[2]) if d == 3 else 1)
        self.mass = torch.empty(self.G, dtype=torch.float64, device=self.dev)
        self.vel = torch.empty(d * self.G, dtype=torch.float64, device=self.dev)
        self.status = torch.empty(1, dtype=torch.int32, device=self.dev)

    def run(self, lib):
        import torch
        self.mass.fill_(-1.0)
        self.vel.fill_(-1.0)
        self.status.fill_(-1)
        stream = C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        rc = lib.mtr_p2g_noalloc(C.byref(self.params), _ptr(self.x), _ptr(self.v), _ptr(self.B), self.n,
                                 _ptr(self.gx), _ptr(self.gy), _ptr(self.gz), self.dims, _ptr(self.mass),
                                 _ptr(self.vel), _ptr(self.status), stream)
        torch.cuda.synchronize(self.dev)
        m = self.mass.cpu().numpy()
        vv = self.vel.cpu().numpy().reshape(self.d, self.G).T
        return rc, m, vv, int(self.status.cpu().numpy()[0]) & 0xffffffff


def _close(got_m, got_v, ref_m, ref_v, what):
    scale_m = np.abs(ref_m).max()
    scale_v = max(np.abs(ref_v).max(), 1e-300)
    assert np.abs(got_m - ref_m).max() <= REL * scale_m, (what, "mass", np.abs(got_m - ref_m).max() / scale_m)
    assert np.abs(got_v - ref_v).max() <= REL * scale_v, (what, "velocity", np.abs(got_v - ref_v).max() / scale_v)


@pytest.mark.parametrize("dim,deg", [(3, 3), (3, 2), (2, 2), (2, 3)])
def test_noalloc_matches_the_step_and_the_oracle_on_two_calls(dim, deg):
    """First call: a larger block; second call: a smaller block with other
    particles on a smaller grid.  Each is checked against the regular step's
    grid and the oracle's P2G on that grid."""
    lib = load_library()
    big = _scene(dim, deg, n=8 if dim == 3 else 14, seed=3)
    small = _scene(dim, deg, n=5 if dim == 3 else 9, seed=17)
    for call, sc in enumerate((big, small)):
        ref = _step_grid(sc)
        om, ov, left = p2g_grid(sc.params, sc.x, sc.v, sc.B, ref["x"], ref["y"], ref["z"], ref["dims"])
        assert left == 0
        _close(om, ov, ref["mass"], ref["v"], "oracle vs step")
        c = _Call(sc.params, sc.x, sc.v, sc.B, ref["x"], ref["y"], ref["z"], ref["dims"])
        rc, m, vv, status = c.run(lib)
        assert rc == abi.MTR_OK, (call, rc)
        assert status == 0, (call, hex(status))
        _close(m, vv, ref["mass"], ref["v"], f"call {call} vs step")
        _close(m, vv, om, ov, f"call {call} vs oracle")
    assert small.Np < big.Np


def _uniform_grid(dims, dx, origin):
    return [origin[a] + dx * np.arange(dims[a], dtype=np.float64) for a in range(3)]


def test_noalloc_at_its_capacity():
    """Exactly MTR_NOALLOC_MAX_PARTICLES particles on a grid of exactly
    MTR_NOALLOC_MAX_NODES nodes (64 x 64 x 32), against the oracle; mass sums
    to the particles' mass."""
    lib = load_library()
    dims = (64, 64, 32)
    assert dims[0] * dims[1] * dims[2] == MAX_NODES
    p = abi.default_params(3, 2)
    p.dx, p.particle_mass, p.flip_ratio = 0.01, 2.5e-4, -2.0
    rng = np.random.default_rng(5)
    org = (-0.2, 0.1, 0.05)
    gx, gy, gz = _uniform_grid(dims, p.dx, org)
    # cells 1 .. N-4 on every axis: every stencil inside the grid
    lo = np.array(org) + p.dx * 1.0
    hi = np.array(org) + p.dx * (np.array(dims) - 3.0)
    x = lo + (hi - lo) * rng.random((MAX_PARTICLES, 3))
    v = rng.normal(size=(MAX_PARTICLES, 3))
    B = 5.0 * rng.normal(size=(MAX_PARTICLES, 9))
    om, ov, left = p2g_grid(p, x, v, B, gx, gy, gz, dims)
    assert left == 0
    c = _Call(p, x, v, B, gx, gy, gz, dims)
    rc, m, vv, status = c.run(lib)
    assert rc == abi.MTR_OK and status == 0, (rc, hex(status))
    _close(m, vv, om, ov, "capacity vs oracle")
    assert abs(m.sum() - MAX_PARTICLES * p.particle_mass) <= 1e-10 * MAX_PARTICLES * p.particle_mass


def test_noalloc_drops_out_of_grid_particles_and_reports_them():
    """Particles far outside the grid (beyond its last tile, at negative
    cells, non-finite) and one whose stencil passes the last node are dropped;
    the rest deposit as if they were absent, and the status word carries
    MTR_STATUS_STENCIL_OOB.  A following clean call reports 0."""
    lib = load_library()
    sc = _scene(3, 2, n=8, seed=3)
    ref = _step_grid(sc)
    dims = ref["dims"]
    gx, gy, gz = ref["x"], ref["y"], ref["z"]
    dx = sc.params.dx
    bad = np.array([
        [gx[0] + 1e3, gy[0] + 0.5 * dx, gz[0] + 0.5 * dx],     # far beyond the grid on x
        [gx[0] - 40 * dx, gy[3], gz[3]],                       # negative cell
        [np.nan, gy[3], gz[3]],                                 # not finite
        [gx[-1] - 0.5 * dx, gy[3] + 0.2 * dx, gz[3] + 0.2 * dx],  # in the grid, stencil past the last node
        [gx[2] + 0.3 * dx, gy[2] + 0.4 * dx, gz[2] + 0.6 * dx],   # a kept one among them
    ])
    x = np.concatenate([sc.x[:100], bad, sc.x[100:]])
    rng = np.random.default_rng(9)
    v = np.concatenate([sc.v[:100], rng.normal(size=(len(bad), 3)), sc.v[100:]])
    Bb = rng.normal(size=(len(bad), 9))
    B = np.concatenate([sc.B.reshape(-1, 9)[:100], Bb, sc.B.reshape(-1, 9)[100:]])
    om, ov, left = p2g_grid(sc.params, x, v, B, gx, gy, gz, dims)
    assert left == 4
    c = _Call(sc.params, x, v, B, gx, gy, gz, dims)
    rc, m, vv, status = c.run(lib)
    assert rc == abi.MTR_OK
    assert status & MTR_STATUS_STENCIL_OOB, hex(status)
    _close(m, vv, om, ov, "with dropped particles vs oracle")
    c2 = _Call(sc.params, sc.x, sc.v, sc.B, gx, gy, gz, dims)
    rc, m, vv, status = c2.run(lib)
    assert rc == abi.MTR_OK and status == 0, (rc, hex(status))
    _close(m, vv, ref["mass"], ref["v"], "clean call after a dropping one")


def test_noalloc_rejects_requests_beyond_its_capacity():
    import torch
    lib = load_library()
    p = abi.default_params(3, 2)
    p.dx, p.particle_mass = 0.01, 1e-3
    dev = torch.device("cuda", 0)
    t = torch.zeros(16, dtype=torch.float64, device=dev)
    ok = (C.c_uint32 * 3)(8, 8, 8)
    big = (C.c_uint32 * 3)(128, 128, 128)
    stream = C.c_void_p(0)
    assert lib.mtr_p2g_noalloc(C.byref(p), _ptr(t), _ptr(t), _ptr(t), MAX_PARTICLES + 1, _ptr(t), _ptr(t), _ptr(t),
                               ok, _ptr(t), _ptr(t), None, stream) == MTR_ERR_TOO_LARGE
    assert lib.mtr_p2g_noalloc(C.byref(p), _ptr(t), _ptr(t), _ptr(t), 4, _ptr(t), _ptr(t), _ptr(t), big,
                               _ptr(t), _ptr(t), None, stream) == MTR_ERR_TOO_LARGE
