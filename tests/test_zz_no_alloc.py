"""mtr_p2g_noalloc: the particle-to-grid transfer for callers that cannot
allocate device memory where they call it (code under CUDA-graph capture,
solvers inside a framework that owns all device memory through its own pool,
real-time loops).  It keeps its sort, tile and accumulator scratch in one fixed
device array, so these tests check that it reproduces the grid the regular
step (mtr_step through mtr_ctx) deposits, on two calls in a row (the second
call must not see the first call's leftovers), and that it refuses requests
larger than the array.

This file is collected last on purpose: a failure here stops a -x run only
after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from matter_tests_b200 import abi
from matter_tests_b200.gpu import GpuSim, load_library

import cases
from gpu_util import needs_gpu

pytestmark = [pytest.mark.gpu, needs_gpu]

REL = 1e-10


def _scene(dim, deg):
    sc = cases.block(dim, deg, n=8 if dim == 3 else 14, gravity=(0.0, 0.0, 0.0))
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


@pytest.mark.parametrize("dim,deg", [(3, 3), (3, 2), (2, 2)])
def test_noalloc_matches_the_step_on_two_calls(dim, deg):
    import torch
    sc = _scene(dim, deg)
    ref = _step_grid(sc)
    lib = load_library()
    dev = torch.device("cuda", 0)
    n, d = sc.Np, dim
    x = torch.tensor(np.ascontiguousarray(sc.x.T), device=dev)
    v = torch.tensor(np.ascontiguousarray(sc.v.T), device=dev)
    b_rm = sc.B.reshape(n, d, d).transpose(0, 2, 1).reshape(n, d * d)  # host layout is column-major
    B = torch.tensor(np.ascontiguousarray(b_rm.T), device=dev)
    gx = torch.tensor(ref["x"], device=dev)
    gy = torch.tensor(ref["y"], device=dev)
    gz = torch.tensor(ref["z"], device=dev)
    dims = (C.c_uint32 * 3)(*ref["dims"])
    G = int(np.prod(ref["dims"]))
    mass = torch.empty(G, dtype=torch.float64, device=dev)
    vel = torch.empty(d * G, dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for call in range(2):
        mass.fill_(-1.0)
        vel.fill_(-1.0)
        rc = lib.mtr_p2g_noalloc(C.byref(sc.params), _ptr(x), _ptr(v), _ptr(B), n, _ptr(gx), _ptr(gy), _ptr(gz),
                                 dims, _ptr(mass), _ptr(vel), stream)
        assert rc == abi.MTR_OK, (call, rc)
        torch.cuda.synchronize(dev)
        m = mass.cpu().numpy()
        vv = vel.cpu().numpy().reshape(d, G).T
        scale_m = np.abs(ref["mass"]).max()
        scale_v = np.abs(ref["v"]).max()
        assert np.abs(m - ref["mass"]).max() <= REL * scale_m, (call, "mass")
        assert np.abs(vv - ref["v"]).max() <= REL * scale_v, (call, "velocity")


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
    too_many = abi_max_particles() + 1
    assert lib.mtr_p2g_noalloc(C.byref(p), _ptr(t), _ptr(t), _ptr(t), too_many, _ptr(t), _ptr(t), _ptr(t), ok,
                               _ptr(t), _ptr(t), stream) == MTR_ERR_TOO_LARGE
    assert lib.mtr_p2g_noalloc(C.byref(p), _ptr(t), _ptr(t), _ptr(t), 4, _ptr(t), _ptr(t), _ptr(t), big,
                               _ptr(t), _ptr(t), stream) == MTR_ERR_TOO_LARGE


MTR_ERR_TOO_LARGE = -8


def abi_max_particles():
    return 1 << 18
