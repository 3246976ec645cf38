"""ctypes front end of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm import this module.  Two checkers share one interface:

* ``Oracle``    — oracle/liboracle.so, the C restatement (mpm_oracle.c), any
                  dim (2|3) and spline degree (2|3);
* ``Reference`` — oracle/_ref/libref_{2,3}d_q{2,3}.so, the reference's own
                  src/simulation/*.cpp compiled by oracle/Makefile (2D from a
                  copy whose tools.hpp leaves THREEDIM undefined).

Arrays are numpy float64, AoS per particle exactly as include/matter_gpu.h
describes (vectors dim-wide, matrices column-major dim*dim, six scalars).
"""
import ctypes as C
import os

import numpy as np

from matter_tests_b200.abi import MtrParams, MtrPlate, MtrObject

HERE = os.path.dirname(os.path.abspath(__file__))
_P = C.POINTER(C.c_double)
_U = C.POINTER(C.c_uint32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _f64(a, n):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    assert a.size == n, (a.size, n)
    return a


class _Checker:
    prefix = None

    def _bind(self, lib):
        pf = self.prefix
        self.lib = lib
        getattr(lib, pf + "set_particles").argtypes = [C.c_void_p, C.c_uint32, _P, _P, _P, _P, _P]
        getattr(lib, pf + "set_objects").argtypes = [C.c_void_p, C.POINTER(MtrPlate), C.c_int,
                                                     C.POINTER(MtrObject), C.c_int]
        getattr(lib, pf + "step").argtypes = [C.c_void_p, C.c_int]
        getattr(lib, pf + "get_particles").argtypes = [C.c_void_p, _P, _P, _P, _P, _P, _P, _P]
        getattr(lib, pf + "get_grid").argtypes = [C.c_void_p, _U, _P, _P, _P, _P, _P, _P]
        getattr(lib, pf + "get_clock").argtypes = [C.c_void_p, _P]
        getattr(lib, pf + "get_plates").argtypes = [C.c_void_p, C.POINTER(MtrPlate), C.c_int]
        getattr(lib, pf + "destroy").argtypes = [C.c_void_p]

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def set_particles(self, x, v=None, F=None, B=None, scalars=None):
        d = self.dim
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        n = x.size // d
        self.Np = n
        v, F, B, scalars = _f64(v, n * d), _f64(F, n * d * d), _f64(B, n * d * d), _f64(scalars, n * 6)
        self._keep = (x, v, F, B, scalars)
        rc = self._f("set_particles")(self.h, n, _ptr(x), _ptr(v), _ptr(F), _ptr(B), _ptr(scalars))
        assert rc == 0

    def set_objects(self, plates=(), objects=()):
        self.nplates = len(plates)
        pa = (MtrPlate * max(1, len(plates)))(*plates)
        oa = (MtrObject * max(1, len(objects)))(*objects)
        rc = self._f("set_objects")(self.h, pa, len(plates), oa, len(objects))
        assert rc == 0

    def step(self, n=1):
        return self._f("step")(self.h, n)

    def particles(self):
        d, n = self.dim, self.Np
        out = {k: np.zeros(n * s) for k, s in
               (("x", d), ("v", d), ("F", d * d), ("B", d * d), ("scalars", 6), ("pic", d), ("flip", d))}
        self._f("get_particles")(self.h, *(_ptr(out[k]) for k in ("x", "v", "F", "B", "scalars", "pic", "flip")))
        out["x"] = out["x"].reshape(n, d)
        out["v"] = out["v"].reshape(n, d)
        out["pic"] = out["pic"].reshape(n, d)
        out["flip"] = out["flip"].reshape(n, d)
        out["F"] = out["F"].reshape(n, d, d)
        out["B"] = out["B"].reshape(n, d, d)
        out["scalars"] = out["scalars"].reshape(n, 6)
        return out

    def grid(self):
        d = self.dim
        dims = (C.c_uint32 * 3)()
        self._f("get_grid")(self.h, dims, None, None, None, None, None, None)
        nx, ny, nz = dims[0], dims[1], dims[2]
        G = nx * ny * nz
        gx, gy, gz = np.zeros(nx), np.zeros(ny), np.zeros(max(nz, 1))
        m, v, fl = np.zeros(G), np.zeros(G * d), np.zeros(G * d)
        self._f("get_grid")(self.h, dims, _ptr(gx), _ptr(gy), _ptr(gz), _ptr(m), _ptr(v), _ptr(fl))
        return {"dims": (nx, ny, nz), "x": gx, "y": gy, "z": gz, "mass": m,
                "v": v.reshape(G, d), "flip": fl.reshape(G, d)}

    def clock(self):
        out = np.zeros(8)
        self._f("get_clock")(self.h, _ptr(out))
        return {"time": out[0], "dt": out[1], "step": int(out[2]), "frame": int(out[3]),
                "done": int(out[4]), "exit": int(out[5]), "status": int(out[6]),
                "plastic_count": int(out[7])}

    def plates(self):
        arr = (MtrPlate * max(1, self.nplates))()
        self._f("get_plates")(self.h, arr, self.nplates)
        return list(arr)[: self.nplates]

    def close(self):
        if getattr(self, "h", None):
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_oracle_lib = None


def _load_oracle():
    global _oracle_lib
    if _oracle_lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is missing; run `make -C oracle oracle`")
        lib = C.CDLL(path)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(MtrParams)]
        lib.orc_sizeof_params.restype = C.c_size_t
        lib.orc_sizeof_plate.restype = C.c_size_t
        lib.orc_sizeof_object.restype = C.c_size_t
        assert lib.orc_sizeof_params() == C.sizeof(MtrParams)
        assert lib.orc_sizeof_plate() == C.sizeof(MtrPlate)
        assert lib.orc_sizeof_object() == C.sizeof(MtrObject)
        lib.orc_svd.argtypes = [C.c_int, _P, _P, _P, _P]
        lib.orc_get_keys.argtypes = [C.c_void_p, _U]
        lib.orc_get_constants.argtypes = [C.c_void_p, _P]
        _oracle_lib = lib
    return _oracle_lib


class Oracle(_Checker):
    """The C restatement (mpm_oracle.c)."""
    prefix = "orc_"

    def __init__(self, params):
        lib = _load_oracle()
        self._bind(lib)
        self.dim = params.dim
        self.params = params
        self.h = lib.orc_create(C.byref(params))
        if not self.h:
            raise ValueError("oracle rejected the parameters")

    def set_levelset(self, ls):
        """A scenes.LevelSetData into its slot (orc_set_levelset)."""
        from matter_tests_b200.gpu import _set_levelset
        self.lib.orc_set_levelset.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                              _U, _P, C.c_double]
        self._ls_keep = getattr(self, "_ls_keep", []) + [ls]
        assert _set_levelset(self.lib.orc_set_levelset, self.h, ls) == 0

    def keys(self):
        k = np.zeros(self.Np, dtype=np.uint32)
        self.lib.orc_get_keys(self.h, k.ctypes.data_as(_U))
        return k

    def constants(self):
        out = np.zeros(10)
        self.lib.orc_get_constants(self.h, _ptr(out))
        names = ("lambda", "mu", "K", "wave_speed", "dt_max", "apicDinverse", "e_mu_prefac",
                 "f_mu_prefac", "d_prefac", "fac_Q")
        return dict(zip(names, out))


def svd(A):
    """Oracle SVD of one dim x dim matrix (numpy, row-major in and out)."""
    lib = _load_oracle()
    d = A.shape[0]
    a = np.ascontiguousarray(A.T, dtype=np.float64).reshape(-1)
    U, S, V = np.zeros(d * d), np.zeros(d), np.zeros(d * d)
    lib.orc_svd(d, _ptr(a), _ptr(U), _ptr(S), _ptr(V))
    return U.reshape(d, d).T, S, V.reshape(d, d).T


def p2g_grid(params, x, v, B, gx, gy, gz, dims):
    """Oracle P2G of particles onto a given uniform grid (orc_p2g_grid): the
    checker of mtr_p2g_noalloc.  x, v (Np, dim); B per particle column-major
    dim*dim like set_particles, or None; returns (mass[G], v[G, dim],
    particles left out)."""
    lib = _load_oracle()
    lib.orc_p2g_grid.restype = C.c_uint32
    lib.orc_p2g_grid.argtypes = [C.POINTER(MtrParams), C.c_uint32, _P, _P, _P, _P, _P, _P, _U, _P, _P]
    d = params.dim
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, d)
    n = x.shape[0]
    v = np.ascontiguousarray(v, dtype=np.float64).reshape(n, d)
    Bc = _f64(B, n * d * d)
    gx = np.ascontiguousarray(gx, dtype=np.float64)
    gy = np.ascontiguousarray(gy, dtype=np.float64)
    gz = np.ascontiguousarray(gz if gz is not None and d == 3 else np.zeros(1), dtype=np.float64)
    dd = (C.c_uint32 * 3)(*[int(a) for a in dims])
    G = int(dims[0]) * int(dims[1]) * (int(dims[2]) if d == 3 else 1)
    m, gv = np.zeros(G), np.zeros(G * d)
    left = lib.orc_p2g_grid(C.byref(params), n, _ptr(x), _ptr(v), _ptr(Bc), _ptr(gx), _ptr(gy), _ptr(gz), dd,
                            _ptr(m), _ptr(gv))
    return m, gv.reshape(G, d), int(left)


_ref_libs = {}


def _ref_path(dim, deg):
    return os.path.join(HERE, "_ref", f"libref_{dim}d_q{deg}.so")


def reference_available(dim, deg):
    return os.path.exists(_ref_path(dim, deg))


class Reference(_Checker):
    """The reference's own Simulation, compiled from its sources."""
    prefix = "ref_"

    def __init__(self, params, n_threads=1):
        if not reference_available(params.dim, params.spline_deg):
            raise RuntimeError("reference build for dim=%d deg=%d is not available"
                               % (params.dim, params.spline_deg))
        key = (params.dim, params.spline_deg)
        if key not in _ref_libs:
            lib = C.CDLL(_ref_path(*key))
            lib.ref_create.restype = C.c_void_p
            lib.ref_create.argtypes = [C.POINTER(MtrParams), C.c_int]
            _ref_libs[key] = lib
        lib = _ref_libs[key]
        self._bind(lib)
        self.dim = params.dim
        self.params = params
        self.h = lib.ref_create(C.byref(params), n_threads)
        if not self.h:
            raise ValueError("reference harness rejected the parameters")
