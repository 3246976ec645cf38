"""ctypes mirror of include/matter_gpu.h (structs, enums, error codes).

The numbering of every enum is that of the reference's tools.hpp:53-57, so a
value read from a reference setup maps one to one.
"""
import ctypes as C

# ---- error codes ----------------------------------------------------------
MTR_OK = 0
MTR_ERR_INVALID = -1
MTR_ERR_CUDA = -2
MTR_ERR_OOM = -3
MTR_ERR_DEVICE_STATUS = -4
MTR_ERR_TIMEOUT = -5
MTR_ERR_NO_DEVICE = -6
MTR_ERR_STATE = -7
ERROR_NAMES = {
    MTR_OK: "MTR_OK", MTR_ERR_INVALID: "MTR_ERR_INVALID", MTR_ERR_CUDA: "MTR_ERR_CUDA",
    MTR_ERR_OOM: "MTR_ERR_OOM", MTR_ERR_DEVICE_STATUS: "MTR_ERR_DEVICE_STATUS",
    MTR_ERR_TIMEOUT: "MTR_ERR_TIMEOUT", MTR_ERR_NO_DEVICE: "MTR_ERR_NO_DEVICE",
    MTR_ERR_STATE: "MTR_ERR_STATE",
}

# ---- status flags ---------------------------------------------------------
STATUS_GRID_OVERFLOW = 0x0001
STATUS_STENCIL_OOB = 0x0002
STATUS_BAD_BC = 0x0004
STATUS_RMA_NOCONV = 0x0008
STATUS_RMA_NOSTEP = 0x0010
STATUS_NEG_DGAMMA = 0x0020
STATUS_NONFINITE = 0x0040
STATUS_BAD_MODEL = 0x0080
STATUS_RESID_DIFF = 0x0100


class PlateType:  # tools.hpp:53
    top, bottom, left, right, front, back = range(6)


class ElasticModel:  # tools.hpp:54
    Hencky, NeoHookean = range(2)


class PlasticModel:  # tools.hpp:55
    (NoPlasticity, VM, DP, DPSoft, MCC, VMVisc, DPVisc, MCCVisc, DPMui, MCCMui,
     Snow) = range(11)


class HardeningLaw:  # tools.hpp:56
    NoHard, ExpoExpl, ExpoImpl, SinhExpl, SinhImpl = range(5)


class BC:  # tools.hpp:57
    NoSlip, SlipStick, SlipFree = range(3)


class ObjectKind:
    Bump, Ground, Ramp, Curve, Gate, Silo, BoxRotated, TerrainGauss, LevelSet = range(9)


MAX_LEVELSETS = 4


PREC_FP64 = 0
PREC_MIXED = 1

SCALARS = ("eps_pl_dev", "eps_pl_vol", "eps_pl_vol_pradhana", "delta_gamma", "viscosity", "muI")


class MtrParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("spline_deg", C.c_int32), ("precision", C.c_int32),
        ("elastic_model", C.c_int32), ("plastic_model", C.c_int32), ("hardening_law", C.c_int32),
        ("use_pradhana", C.c_int32), ("use_mises_q", C.c_int32), ("use_mibf", C.c_int32),
        ("use_musl", C.c_int32), ("gravity_special", C.c_int32), ("pbc", C.c_int32),
        ("end_frame", C.c_uint32), ("change_particle_positions", C.c_int32),
        ("fps", C.c_double), ("cfl", C.c_double), ("cfl_elastic", C.c_double),
        ("flip_ratio", C.c_double), ("rho", C.c_double), ("gravity_time", C.c_double),
        ("gravity", C.c_double * 3), ("grid_reference_point", C.c_double * 3),
        ("dx", C.c_double), ("particle_mass", C.c_double), ("particle_volume", C.c_double),
        ("E", C.c_double), ("nu", C.c_double), ("stress_tolerance", C.c_double), ("xi", C.c_double),
        ("q_max", C.c_double), ("q_min", C.c_double), ("p_min", C.c_double),
        ("M", C.c_double), ("q_cohesion", C.c_double),
        ("perzyna_exp", C.c_double), ("perzyna_visc", C.c_double),
        ("beta", C.c_double), ("p0", C.c_double),
        ("rho_s", C.c_double), ("grain_diameter", C.c_double), ("I_ref", C.c_double),
        ("mu_1", C.c_double), ("mu_2", C.c_double),
        ("L", C.c_double * 3),
    ]


class MtrPlate(C.Structure):
    _fields_ = [
        ("plate_type", C.c_int32), ("bc", C.c_int32), ("friction", C.c_double),
        ("pos_object", C.c_double), ("pos_lower", C.c_double), ("pos_upper", C.c_double),
        ("v_object", C.c_double * 3), ("v_object_original", C.c_double * 3),
        ("vmin_factor", C.c_double), ("load_factor", C.c_double),
    ]


class MtrObject(C.Structure):
    _fields_ = [("kind", C.c_int32), ("bc", C.c_int32), ("friction", C.c_double),
                ("prm", C.c_double * 24)]


class MtrClock(C.Structure):
    _fields_ = [("time", C.c_double), ("dt", C.c_double), ("step", C.c_uint32),
                ("frame", C.c_uint32), ("done", C.c_int32), ("reserved", C.c_int32)]


class MtrGroupInfo(C.Structure):
    _fields_ = [("dim", C.c_int32), ("spline_deg", C.c_int32), ("fp32", C.c_int32), ("musl", C.c_int32),
                ("plastic_model_kernel", C.c_int32), ("members", C.c_int32), ("tile_threads", C.c_int32 * 4),
                ("tile_lanes", C.c_int32 * 2)]


# slots of the tile-kernel block shapes (MTR_TILE_*); the first two are the
# scatters, which also have a lanes-per-particle choice
TILE_SLOTS = ("p2g", "musl", "g2p", "defgrad")
SCATTER_SLOTS = TILE_SLOTS[:2]


def default_params(dim=3, spline_deg=2):
    """Defaults of Simulation's public fields (simulation.hpp:36-106)."""
    import math
    p = MtrParams()
    p.dim, p.spline_deg, p.precision = dim, spline_deg, PREC_FP64
    p.elastic_model, p.plastic_model = ElasticModel.Hencky, PlasticModel.NoPlasticity
    p.hardening_law = HardeningLaw.ExpoImpl
    p.use_pradhana, p.use_mises_q, p.use_mibf, p.use_musl = 1, 0, 0, 0
    p.gravity_special, p.pbc, p.end_frame, p.change_particle_positions = 0, 0, 1, 0
    p.fps, p.cfl, p.cfl_elastic, p.flip_ratio, p.rho, p.gravity_time = 1.0, 0.5, 0.5, -0.95, 1000.0, 0.0
    for a in range(3):
        p.gravity[a] = 0.0
        p.grid_reference_point[a] = 2e10
    p.E, p.nu, p.stress_tolerance, p.xi = 1e6, 0.3, 1e-5, 0.0
    p.q_max, p.q_min, p.p_min = 100.0, 100.0, -1e20
    p.M, p.q_cohesion, p.perzyna_exp, p.perzyna_visc = 1.0, 0.0, 1.0, 0.0
    p.beta, p.p0 = 0.0, 1000.0
    p.rho_s, p.grain_diameter, p.I_ref = 2500.0, 1e-3, 0.279
    p.mu_1 = math.tan(20.9 * math.pi / 180.0)
    p.mu_2 = math.tan(32.8 * math.pi / 180.0)
    for a in range(3):
        p.L[a] = 1.0  # Lx = Ly = Lz = 1 (simulation.hpp:60-66)
    return p


def make_plate(pos, plate_type, bc=BC.NoSlip, friction=0.0, lower=-1e15, upper=1e15,
               v=(0.0, 0.0, 0.0), vmin_factor=1.0, load_factor=0.0):
    """ObjectPlate's constructor arguments (object_plate.hpp:13-24)."""
    q = MtrPlate()
    q.plate_type, q.bc, q.friction = plate_type, bc, friction
    q.pos_object, q.pos_lower, q.pos_upper = pos, lower, upper
    for a in range(3):
        q.v_object[a] = v[a] if a < len(v) else 0.0
        q.v_object_original[a] = q.v_object[a]
    q.vmin_factor, q.load_factor = vmin_factor, load_factor
    return q


def make_object(kind, bc=BC.NoSlip, friction=0.0, prm=()):
    o = MtrObject()
    o.kind, o.bc, o.friction = kind, bc, friction
    for i, v in enumerate(prm):
        o.prm[i] = v
    return o
