"""ctypes binding of libmatter_gpu.so (include/matter_gpu.h).

This is the only way Python reaches the CUDA step.  There is no fallback: if
the library is missing or no CUDA device is visible, calls raise.
"""
import ctypes as C
import os

import numpy as np

from .abi import (MtrClock, MtrGroupInfo, MtrObject, MtrParams, MtrPlate, ERROR_NAMES, MTR_OK, SCALARS, SCATTER_SLOTS,
                  TILE_SLOTS)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmatter_gpu.so")

_P = C.POINTER(C.c_double)
_U = C.POINTER(C.c_uint32)

# every entry point declared in include/matter_gpu.h
EXPORTS = (
    "mtr_ctx_create", "mtr_upload", "mtr_set_objects", "mtr_step", "mtr_run", "mtr_run_frame", "mtr_download",
    "mtr_download_pic_flip", "mtr_get_grid", "mtr_get_sort", "mtr_get_plates", "mtr_get_clock",
    "mtr_status", "mtr_clear_status", "mtr_sync", "mtr_stream", "mtr_launch_count", "mtr_keep_pic_flip",
    "mtr_use_graphs", "mtr_profile", "mtr_active_nodes", "mtr_balance", "mtr_set_step_limit",
    "mtr_batch_create", "mtr_batch_step", "mtr_batch_launch_count", "mtr_batch_stream", "mtr_batch_destroy",
    "mtr_footprint", "mtr_ctx_destroy", "mtr_last_error", "mtr_p2g_noalloc",
    "mtr_autotune", "mtr_set_tile_threads", "mtr_get_tile_threads", "mtr_batch_autotune", "mtr_batch_groups",
    "mtr_batch_get_group", "mtr_batch_set_tile_threads", "mtr_frame_columns", "mtr_frame_begin",
    "mtr_frame_wait", "mtr_get_grid_friction", "mtr_set_levelset", "mtr_set_tile_lanes", "mtr_get_tile_lanes",
    "mtr_batch_set_tile_lanes", "mtr_batch_clocks", "mtr_batch_stats", "mtr_batch_set_members",
    "mtr_batch_graph_updates", "mtr_batch_set_retune", "mtr_batch_retunes",
)

_lib = None


class MtrFailure(RuntimeError):
    def __init__(self, fn, rc, msg):
        super().__init__(f"{fn} returned {ERROR_NAMES.get(rc, rc)}: {msg}")
        self.rc = rc


def load_library(path=LIB_PATH):
    """Loads and types the library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m matter_tests_b200.build`")
    lib = C.CDLL(path)
    lib.mtr_ctx_create.argtypes = [C.POINTER(MtrParams), C.c_int, C.POINTER(C.c_void_p)]
    lib.mtr_upload.argtypes = [C.c_void_p, _P, _P, _P, _P, _P, C.c_uint32]
    lib.mtr_set_objects.argtypes = [C.c_void_p, C.POINTER(MtrPlate), C.c_int, C.POINTER(MtrObject), C.c_int]
    lib.mtr_step.argtypes = [C.c_void_p, C.c_int]
    lib.mtr_run.argtypes = [C.c_void_p]
    lib.mtr_run_frame.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.mtr_download.argtypes = [C.c_void_p, _P, _P, _P, _P, _P]
    lib.mtr_download_pic_flip.argtypes = [C.c_void_p, _P, _P]
    lib.mtr_get_grid.argtypes = [C.c_void_p, _U, _P, _P, _P, _P, _P, _P]
    lib.mtr_get_sort.argtypes = [C.c_void_p, _U, _U, _U]
    lib.mtr_get_plates.argtypes = [C.c_void_p, C.POINTER(MtrPlate), C.c_int]
    lib.mtr_get_clock.argtypes = [C.c_void_p, C.POINTER(MtrClock)]
    lib.mtr_status.argtypes = [C.c_void_p, _U, _U]
    lib.mtr_clear_status.argtypes = [C.c_void_p]
    lib.mtr_sync.argtypes = [C.c_void_p, C.c_double]
    lib.mtr_stream.argtypes = [C.c_void_p]
    lib.mtr_stream.restype = C.c_void_p
    lib.mtr_launch_count.argtypes = [C.c_void_p]
    lib.mtr_launch_count.restype = C.c_int64
    lib.mtr_keep_pic_flip.argtypes = [C.c_void_p, C.c_int]
    lib.mtr_use_graphs.argtypes = [C.c_void_p, C.c_int]
    lib.mtr_profile.argtypes = [C.c_void_p, C.c_int, _P, C.POINTER(C.c_char_p), C.c_int, C.POINTER(C.c_int)]
    lib.mtr_active_nodes.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    lib.mtr_balance.argtypes = [C.c_void_p, _P, _P, _P, _P]
    lib.mtr_set_step_limit.argtypes = [C.c_void_p, C.c_uint32]
    lib.mtr_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
    lib.mtr_batch_set_members.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int]
    lib.mtr_batch_graph_updates.argtypes = [C.c_void_p]
    lib.mtr_batch_set_retune.argtypes = [C.c_void_p, C.c_int]
    lib.mtr_batch_retunes.argtypes = [C.c_void_p]
    lib.mtr_batch_step.argtypes = [C.c_void_p, C.c_int]
    lib.mtr_batch_launch_count.argtypes = [C.c_void_p]
    lib.mtr_batch_launch_count.restype = C.c_int64
    lib.mtr_batch_stream.argtypes = [C.c_void_p]
    lib.mtr_batch_stream.restype = C.c_void_p
    lib.mtr_batch_destroy.argtypes = [C.c_void_p]
    lib.mtr_batch_destroy.restype = None
    lib.mtr_footprint.argtypes = [C.POINTER(MtrParams), C.c_uint32, _P, C.POINTER(C.c_uint64)]
    lib.mtr_p2g_noalloc.argtypes = [C.POINTER(MtrParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32), C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]
    _I4 = C.POINTER(C.c_int)
    lib.mtr_autotune.argtypes = [C.c_void_p, C.c_int, _I4]
    lib.mtr_set_tile_threads.argtypes = [C.c_void_p, _I4]
    lib.mtr_get_tile_threads.argtypes = [C.c_void_p, _I4]
    lib.mtr_batch_autotune.argtypes = [C.c_void_p, C.c_int]
    lib.mtr_batch_groups.argtypes = [C.c_void_p]
    lib.mtr_batch_get_group.argtypes = [C.c_void_p, C.c_int, C.POINTER(MtrGroupInfo)]
    lib.mtr_batch_set_tile_threads.argtypes = [C.c_void_p, C.c_int, _I4]
    lib.mtr_set_tile_lanes.argtypes = [C.c_void_p, _I4]
    lib.mtr_get_tile_lanes.argtypes = [C.c_void_p, _I4]
    lib.mtr_batch_set_tile_lanes.argtypes = [C.c_void_p, C.c_int, _I4]
    lib.mtr_batch_clocks.argtypes = [C.c_void_p, C.POINTER(MtrClock), C.c_int]
    lib.mtr_batch_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64), _P, C.POINTER(C.c_int64), _P]
    lib.mtr_frame_columns.argtypes = [C.c_void_p, C.POINTER(C.c_char_p), C.c_int]
    lib.mtr_frame_begin.argtypes = [C.c_void_p]
    lib.mtr_frame_wait.argtypes = [C.c_void_p, C.c_double, C.POINTER(_P), C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_int), C.POINTER(MtrClock)]
    lib.mtr_get_grid_friction.argtypes = [C.c_void_p, _P]
    _F = C.POINTER(C.c_float)
    lib.mtr_set_levelset.argtypes = [C.c_void_p, C.c_int, _F, _F, _U, _P, C.c_double]
    lib.mtr_ctx_destroy.argtypes = [C.c_void_p]
    lib.mtr_ctx_destroy.restype = None
    lib.mtr_last_error.restype = C.c_char_p
    _lib = lib
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _set_levelset(fn, h, ls):
    """Calls an mtr_set_levelset-shaped entry point with a scenes.LevelSetData."""
    phi = np.ascontiguousarray(ls.phi, dtype=np.float32).reshape(-1)
    nrm = None if ls.normals is None else np.ascontiguousarray(ls.normals, dtype=np.float32).reshape(-1)
    dims = (C.c_uint32 * 3)(*(list(ls.dims) + [1] * (3 - len(ls.dims))))
    org = np.zeros(3)
    org[:len(ls.origin)] = ls.origin
    F = C.POINTER(C.c_float)
    return fn(h, int(ls.slot), phi.ctypes.data_as(F), None if nrm is None else nrm.ctypes.data_as(F), dims,
              _ptr(org), float(ls.spacing))


def _check(lib, fn, rc):
    if rc != MTR_OK:
        raise MtrFailure(fn, rc, lib.mtr_last_error().decode())
    return rc


class GpuSim:
    """One simulation context on one GPU (mtr_ctx)."""

    def __init__(self, params, device=0):
        self.lib = load_library()
        self.params = params
        self.dim = params.dim
        h = C.c_void_p()
        _check(self.lib, "mtr_ctx_create", self.lib.mtr_ctx_create(C.byref(params), device, C.byref(h)))
        self.h = h
        self.Np = 0
        self.nplates = 0

    # -- set-up ---------------------------------------------------------
    def upload(self, x, v=None, F=None, B=None, scalars=None):
        d = self.dim
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        n = x.size // d
        arrs = []
        for a, w in ((v, d), (F, d * d), (B, d * d), (scalars, 6)):
            if a is None:
                arrs.append(None)
            else:
                a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                assert a.size == n * w
                arrs.append(a)
        _check(self.lib, "mtr_upload", self.lib.mtr_upload(self.h, _ptr(x), *(_ptr(a) for a in arrs), n))
        self.Np = n

    def set_objects(self, plates=(), objects=()):
        self.nplates = len(plates)
        pa = (MtrPlate * max(1, len(plates)))(*plates)
        oa = (MtrObject * max(1, len(objects)))(*objects)
        _check(self.lib, "mtr_set_objects", self.lib.mtr_set_objects(self.h, pa, len(plates), oa, len(objects)))

    def set_levelset(self, ls):
        """Uploads a scenes.LevelSetData to its slot (mtr_set_levelset)."""
        _check(self.lib, "mtr_set_levelset", _set_levelset(self.lib.mtr_set_levelset, self.h, ls))

    def set_scene_objects(self, scene):
        """The scene's level sets, plates and objects."""
        for ls in getattr(scene, "levelsets", ()):
            self.set_levelset(ls)
        self.set_objects(scene.plates, scene.objects)

    def set_step_limit(self, last_step):
        """No step past step number last_step (mtr_set_step_limit)."""
        _check(self.lib, "mtr_set_step_limit", self.lib.mtr_set_step_limit(self.h, int(last_step)))

    def keep_pic_flip(self, on=True):
        _check(self.lib, "mtr_keep_pic_flip", self.lib.mtr_keep_pic_flip(self.h, 1 if on else 0))

    def use_graphs(self, on=True):
        _check(self.lib, "mtr_use_graphs", self.lib.mtr_use_graphs(self.h, 1 if on else 0))

    # -- block shapes of the tile kernels ---------------------------------
    def autotune(self, reps=3):
        """Times trial steps with 64, 128 and 256 threads per tile block and
        keeps the fastest per kernel (mtr_autotune); returns {slot: threads}."""
        t = (C.c_int * 4)()
        _check(self.lib, "mtr_autotune", self.lib.mtr_autotune(self.h, int(reps), t))
        return dict(zip(TILE_SLOTS, list(t)))

    @property
    def tile_threads(self):
        t = (C.c_int * 4)()
        _check(self.lib, "mtr_get_tile_threads", self.lib.mtr_get_tile_threads(self.h, t))
        return dict(zip(TILE_SLOTS, list(t)))

    @tile_threads.setter
    def tile_threads(self, shapes):
        cur = self.tile_threads
        cur.update(shapes)
        t = (C.c_int * 4)(*[cur[k] for k in TILE_SLOTS])
        _check(self.lib, "mtr_set_tile_threads", self.lib.mtr_set_tile_threads(self.h, t))

    @property
    def tile_lanes(self):
        """Lanes per particle of the P2G and MUSL scatters (mtr_get_tile_lanes)."""
        t = (C.c_int * 2)()
        _check(self.lib, "mtr_get_tile_lanes", self.lib.mtr_get_tile_lanes(self.h, t))
        return dict(zip(SCATTER_SLOTS, list(t)))

    @tile_lanes.setter
    def tile_lanes(self, lanes):
        cur = self.tile_lanes
        cur.update(lanes)
        t = (C.c_int * 2)(*[cur[k] for k in SCATTER_SLOTS])
        _check(self.lib, "mtr_set_tile_lanes", self.lib.mtr_set_tile_lanes(self.h, t))

    # -- stepping -------------------------------------------------------
    def step(self, n=1, check=True):
        rc = self.lib.mtr_step(self.h, n)
        if check:
            _check(self.lib, "mtr_step", rc)
        return rc

    def run(self, check=True):
        rc = self.lib.mtr_run(self.h)
        if check:
            _check(self.lib, "mtr_run", rc)
        return rc

    def sync(self, timeout=600.0):
        _check(self.lib, "mtr_sync", self.lib.mtr_sync(self.h, timeout))

    @property
    def stream(self):
        return self.lib.mtr_stream(self.h)

    def launch_count(self):
        return self.lib.mtr_launch_count(self.h)

    def profile(self, nsteps=5, max_slots=64):
        """Mean device ms per launch slot of a step: [(name, ms), ...]."""
        ms = np.zeros(max_slots)
        names = (C.c_char_p * max_slots)()
        n = C.c_int()
        _check(self.lib, "mtr_profile", self.lib.mtr_profile(self.h, nsteps, _ptr(ms), names, max_slots, C.byref(n)))
        return [(names[i].decode(), float(ms[i])) for i in range(min(n.value, max_slots))]

    def active_nodes(self):
        a, t = C.c_uint64(), C.c_uint64()
        _check(self.lib, "mtr_active_nodes", self.lib.mtr_active_nodes(self.h, C.byref(a), C.byref(t)))
        return a.value, t.value

    def balance(self):
        """FP64 mass and momentum balance of the last step (mtr_balance)."""
        gm, pm = C.c_double(), C.c_double()
        gp, pp = np.zeros(self.dim), np.zeros(self.dim)
        _check(self.lib, "mtr_balance", self.lib.mtr_balance(self.h, C.byref(gm), _ptr(gp), C.byref(pm), _ptr(pp)))
        return {"grid_mass": gm.value, "grid_momentum": gp, "particle_mass": pm.value, "particle_momentum": pp}

    # -- read-back ------------------------------------------------------
    def particles(self, pic_flip=False, fields=("x", "v", "F", "B", "scalars")):
        """The particle state in the caller's order; `fields` names the arrays
        to read back (the others are not copied and are absent)."""
        d, n = self.dim, self.Np
        size = {"x": n * d, "v": n * d, "F": n * d * d, "B": n * d * d, "scalars": n * 6}
        out = {k: np.zeros(size[k]) for k in fields}
        _check(self.lib, "mtr_download", self.lib.mtr_download(
            self.h, *(_ptr(out.get(k)) for k in ("x", "v", "F", "B", "scalars"))))
        if pic_flip:
            out["pic"], out["flip"] = np.zeros(n * d), np.zeros(n * d)
            _check(self.lib, "mtr_download_pic_flip",
                   self.lib.mtr_download_pic_flip(self.h, _ptr(out["pic"]), _ptr(out["flip"])))
            out["pic"] = out["pic"].reshape(n, d)
            out["flip"] = out["flip"].reshape(n, d)
        shape = {"x": (n, d), "v": (n, d), "F": (n, d, d), "B": (n, d, d), "scalars": (n, 6)}
        for k in fields:
            out[k] = out[k].reshape(shape[k])
        return out

    def grid(self):
        d = self.dim
        dims = (C.c_uint32 * 3)()
        _check(self.lib, "mtr_get_grid", self.lib.mtr_get_grid(self.h, dims, None, None, None, None, None, None))
        nx, ny, nz = dims[0], dims[1], dims[2]
        G = nx * ny * nz
        gx, gy, gz = np.zeros(nx), np.zeros(ny), np.zeros(max(nz, 1))
        m, v, fl = np.zeros(G), np.zeros(G * d), np.zeros(G * d)
        _check(self.lib, "mtr_get_grid", self.lib.mtr_get_grid(self.h, dims, _ptr(gx), _ptr(gy), _ptr(gz), _ptr(m),
                                                               _ptr(v), _ptr(fl)))
        return {"dims": (nx, ny, nz), "x": gx, "y": gy, "z": gz, "mass": m, "v": v.reshape(G, d),
                "flip": fl.reshape(G, d)}

    # -- frame output -----------------------------------------------------
    def frame_columns(self):
        names = (C.c_char_p * 32)()
        n = self.lib.mtr_frame_columns(self.h, names, 32)
        if n < 0:
            _check(self.lib, "mtr_frame_columns", n)
        return [names[i].decode() for i in range(n)]

    def frame_begin(self):
        """Snapshot of the particle file's rows behind the issued steps (mtr_frame_begin)."""
        _check(self.lib, "mtr_frame_begin", self.lib.mtr_frame_begin(self.h))

    def frame_wait(self, timeout=600.0):
        """(rows [Np, ncols] copied out of the pinned buffer, column names, clock)."""
        rows, n, nc, ck = _P(), C.c_uint32(), C.c_int(), MtrClock()
        _check(self.lib, "mtr_frame_wait", self.lib.mtr_frame_wait(self.h, timeout, C.byref(rows), C.byref(n),
                                                                   C.byref(nc), C.byref(ck)))
        a = np.ctypeslib.as_array(rows, shape=(n.value * nc.value,)).reshape(n.value, nc.value).copy()
        return a, self.frame_columns(), {"time": ck.time, "dt": ck.dt, "step": ck.step, "frame": ck.frame,
                                         "done": ck.done}

    def grid_friction(self):
        G = int(np.prod(self.grid()["dims"]))
        out = np.zeros(G)
        _check(self.lib, "mtr_get_grid_friction", self.lib.mtr_get_grid_friction(self.h, _ptr(out)))
        return out

    def sort_state(self):
        n = self.Np
        keys, perm, ids = (np.zeros(n, dtype=np.uint32) for _ in range(3))
        _check(self.lib, "mtr_get_sort", self.lib.mtr_get_sort(
            self.h, keys.ctypes.data_as(_U), perm.ctypes.data_as(_U), ids.ctypes.data_as(_U)))
        return keys, perm, ids

    def clock(self):
        ck = MtrClock()
        _check(self.lib, "mtr_get_clock", self.lib.mtr_get_clock(self.h, C.byref(ck)))
        return {"time": ck.time, "dt": ck.dt, "step": ck.step, "frame": ck.frame, "done": ck.done}

    def status(self):
        f, b = C.c_uint32(), C.c_uint32()
        _check(self.lib, "mtr_status", self.lib.mtr_status(self.h, C.byref(f), C.byref(b)))
        return f.value, b.value

    def clear_status(self):
        _check(self.lib, "mtr_clear_status", self.lib.mtr_clear_status(self.h))

    def plates(self):
        arr = (MtrPlate * max(1, self.nplates))()
        _check(self.lib, "mtr_get_plates", self.lib.mtr_get_plates(self.h, arr, self.nplates))
        return list(arr)[: self.nplates]

    def close(self):
        if getattr(self, "h", None):
            self.lib.mtr_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scalars_dict(sc):
    return {k: sc[:, i] for i, k in enumerate(SCALARS)}


class GpuBatch:
    """Several GpuSim contexts on one GPU stepped together (mtr_batch)."""

    def __init__(self, sims):
        self.lib = load_library()
        self.sims = list(sims)
        arr = (C.c_void_p * len(self.sims))(*[s.h.value if isinstance(s.h, C.c_void_p) else s.h for s in self.sims])
        h = C.c_void_p()
        _check(self.lib, "mtr_batch_create", self.lib.mtr_batch_create(arr, len(self.sims), C.byref(h)))
        self.h = h

    def step(self, n=1):
        _check(self.lib, "mtr_batch_step", self.lib.mtr_batch_step(self.h, n))

    def set_members(self, sims):
        """Replaces the members (mtr_batch_set_members): the batch keeps its
        stream, the group shapes and its step graph, updated in place."""
        sims = list(sims)
        arr = (C.c_void_p * len(sims))(*[s.h.value if isinstance(s.h, C.c_void_p) else s.h for s in sims])
        _check(self.lib, "mtr_batch_set_members", self.lib.mtr_batch_set_members(self.h, arr, len(sims)))
        self.sims = sims

    def graph_updates(self):
        """Rebuilds that updated the instantiated step graph in place."""
        return self.lib.mtr_batch_graph_updates(self.h)

    def set_retune(self, reps):
        """With reps > 0, step() tunes the batch again (reps repetitions) when a
        group's grids have doubled since its last tune; 0 turns it off."""
        _check(self.lib, "mtr_batch_set_retune", self.lib.mtr_batch_set_retune(self.h, int(reps)))

    def retunes(self):
        """Re-tunes step() ran because a group's grid had doubled since its last tune."""
        return self.lib.mtr_batch_retunes(self.h)

    @property
    def stream(self):
        return self.lib.mtr_batch_stream(self.h)

    def launch_count(self):
        return self.lib.mtr_batch_launch_count(self.h)

    def stats(self):
        """Grid regrowths and batch rebuilds of step() so far, with their wall ms (mtr_batch_stats)."""
        rg, rb = C.c_int64(), C.c_int64()
        rgm, rbm = C.c_double(), C.c_double()
        _check(self.lib, "mtr_batch_stats", self.lib.mtr_batch_stats(self.h, C.byref(rg), C.byref(rgm), C.byref(rb),
                                                                     C.byref(rbm)))
        return {"regrowths": rg.value, "regrow_ms": rgm.value, "rebuilds": rb.value, "rebuild_ms": rbm.value}

    def clocks(self):
        """Each member's clock after the last step() (mtr_batch_clocks, no device round trip)."""
        arr = (MtrClock * len(self.sims))()
        n = self.lib.mtr_batch_clocks(self.h, arr, len(self.sims))
        if n < 0:
            _check(self.lib, "mtr_batch_clocks", n)
        return [{"time": c.time, "dt": c.dt, "step": c.step, "frame": c.frame, "done": c.done} for c in arr[:n]]

    def autotune(self, reps=3):
        """mtr_batch_autotune; returns groups()."""
        _check(self.lib, "mtr_batch_autotune", self.lib.mtr_batch_autotune(self.h, int(reps)))
        return self.groups()

    def groups(self):
        """Each group's key, member count and tile-kernel block shapes."""
        out = []
        for g in range(self.lib.mtr_batch_groups(self.h)):
            info = MtrGroupInfo()
            _check(self.lib, "mtr_batch_get_group", self.lib.mtr_batch_get_group(self.h, g, C.byref(info)))
            out.append({"dim": info.dim, "spline_deg": info.spline_deg, "fp32": bool(info.fp32),
                        "musl": bool(info.musl), "plastic_model_kernel": info.plastic_model_kernel,
                        "members": info.members, "tile_threads": dict(zip(TILE_SLOTS, list(info.tile_threads))),
                        "tile_lanes": dict(zip(SCATTER_SLOTS, list(info.tile_lanes)))})
        return out

    def set_tile_threads(self, group, shapes):
        cur = self.groups()[group]["tile_threads"]
        cur.update(shapes)
        t = (C.c_int * 4)(*[cur[k] for k in TILE_SLOTS])
        _check(self.lib, "mtr_batch_set_tile_threads", self.lib.mtr_batch_set_tile_threads(self.h, group, t))

    def set_tile_lanes(self, group, lanes):
        cur = self.groups()[group]["tile_lanes"]
        cur.update(lanes)
        t = (C.c_int * 2)(*[cur[k] for k in SCATTER_SLOTS])
        _check(self.lib, "mtr_batch_set_tile_lanes", self.lib.mtr_batch_set_tile_lanes(self.h, group, t))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mtr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(params, x):
    """Device bytes mtr_upload allocates for particles at x (mtr_footprint)."""
    lib = load_library()
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    out = C.c_uint64()
    _check(lib, "mtr_footprint", lib.mtr_footprint(C.byref(params), x.size // params.dim, _ptr(x), C.byref(out)))
    return out.value
