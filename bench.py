#!/usr/bin/env python
"""Throughput of the explicit MPM time step on B200, in particle-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference]
                    [--workload collapse3d_mui|collapse2d|incline3d_mcc] [--scale S]

Workload (default): the 3D mu(I)-Drucker-Prager column collapse, MUSL, AFLIP,
cubic B-splines, 1,024,000 particles (box 0.5 x 1.0 x 0.5 m, dx 0.0125 m,
8 particles per cell), seeded synthetic jittered-lattice particles.  A step is
one Simulation::advanceStep of the whole scene.  Both forms of the step run
on the same scene: plain FP64 and mixed precision.

value     plain FP64 particle-steps/s (the reference's arithmetic) over K
          steps timed with CUDA events on the context's stream, state
          resident in HBM (particle state larger than the 126 MB L2 on both
          paths, so every step streams it from HBM; no L2 flush is needed).
mixed     the same figures for the mixed-precision step (FP32 state and
          transfers, FP64 positions, SVD, return mapping and balances), its
          speed-up over FP64 and its state error against the FP64 state after
          the same W + K steps.
configs   the three single-scene workloads at full size and full length
          (2D DP collapse 2000 steps, 3D mu(I) collapse 1000, 3D Cam-Clay
          incline 3000), each in both precisions: device-timed throughput,
          per-kernel times, and the mixed state's position, velocity and
          Kirchhoff-stress error against the FP64 state at the last step.
e2e       the FP64 metric through the C ABI with host buffers: mtr_upload from
          pinned host memory + mtr_step(K) + mtr_download, wall clock, into a
          context that already holds a scene of that size (its buffers and
          step graphs are refilled, not reallocated); the split into upload,
          steps and download, and the first upload into a fresh context.
roofline  the step's most expensive kernel: algorithmic bytes per launch
          (compulsory particle and grid traffic) / its mean CUDA-event
          duration, against the measured HBM copy bandwidth; traffic = that
          kernel's DRAM bytes per launch from the committed ncu capture when
          the capture was taken of the current kernel sources.
cpu_baseline  the reference's own OpenMP step (src/simulation/*.cpp compiled
          from source, oracle/_ref) on a bounded sample of the same workload.
--impl reference  times that reference build alone, on rank 0.
N > 1     independent replicas, one per GPU (the step does not shard); value is
          the sum over ranks of particles*steps / the slowest rank's time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="collapse3d_mui")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=5)
    ap.add_argument("--ensemble-size", type=int, default=256, help="scenes of the batched ensemble")
    ap.add_argument("--ensemble-steps", type=int, default=500, help="timed steps of the batched ensemble")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble measurement")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="forms of the step to time (one form only: for profiler captures)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the full-length runs of the three single-scene workloads")
    ap.add_argument("--serve-requests", type=int, default=60, help="requests of the serving measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving measurement")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default tile-kernel block shapes (128 threads) instead of tuning them")
    ap.add_argument("--tune-reps", type=int, default=3, help="rounds of trial steps per candidate block shape")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value, local):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", local) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid=None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.25)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        busy = [v for v in sm if v > 600] or sm
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for name, val in zip(names, r[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": busy[len(busy) // 2] if busy else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


# DRAM bytes (read + write) per launch of the dominant kernels, from ncu
# captures (dram__bytes_read.sum + dram__bytes_write.sum), stored with the
# hash of the device code they were captured on (the .cuh files of csrc,
# which hold every step kernel); a figure whose hash does not match the code
# being run is reported as stale (traffic null).
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_traffic.json")


def kernel_source_hash():
    import hashlib
    h = hashlib.sha256()
    csrc = os.path.join(ROOT, "matter_tests_b200", "csrc")
    for f in sorted(os.listdir(csrc)):
        if f.endswith(".cuh"):
            with open(os.path.join(csrc, f), "rb") as fh:
                h.update(f.encode() + b"\0" + fh.read())
    return h.hexdigest()[:16]


def capture_entry(workload, scale, kernel, precision):
    """(entry, None) of the ncu capture of this kernel taken on the current
    kernel sources, or (None, why not)."""
    try:
        with open(TRAFFIC_FILE) as f:
            tab = json.load(f)
    except Exception:
        return None, "no capture file"
    for e in tab.get("captures", []):
        if (e.get("workload") == workload and float(e.get("scale", 1.0)) == scale and e.get("kernel") == kernel
                and e.get("precision") == precision):
            if e.get("source_hash", tab.get("source_hash")) != kernel_source_hash():
                return None, "capture predates the current kernel sources"
            return e, None
    return None, "no capture of this kernel"


def measured_traffic(workload, scale, kernel, precision):
    """(bytes per launch, source) of the ncu capture for this kernel, or (None, why)."""
    e, why = capture_entry(workload, scale, kernel, precision)
    if e is None:
        return None, why
    return float(e["dram_bytes_per_launch"]), "ncu capture (profiles/dram_traffic.json): " + e.get("note", "")


def measured_pipes(workload, scale, kernel, precision):
    """Pipe utilisation and top stalls of the same capture (what bounds a
    kernel that is far from the HBM roofline), or None."""
    e, _ = capture_entry(workload, scale, kernel, precision)
    return None if e is None else e.get("pipes")


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# algorithmic bytes per launch: compulsory reads and writes of the persistent
# particle state and of the grid nodes with mass.  Positions are FP64 on both
# paths (8 B); wr is the byte size of every other particle and grid value
# (8 on the FP64 path, 4 on the mixed path).
def kernel_bytes(name, p, Np, Ga, G, wr=8.0):
    d = p.dim
    dd = d * d
    ns = 6 if d == 3 else 3
    w8 = 8.0  # positions and node velocities: FP64 on both paths
    if name == "k_p2g":
        return Np * (w8 * d + wr * (d + dd + ns + (1 if p.use_mibf else 0))) + Ga * wr * (1 + 2 * d)
    if name == "k_g2p":
        return (Np * (w8 * d + wr * (d + dd + 5)) + Ga * (w8 * d + wr * d)
                + Np * (w8 * d + wr * (d + 2 * dd + 6 + ns) + 4))
    if name == "k_g2p_musl":
        return Np * (w8 * d + wr * d) + Ga * (w8 * d + wr * d) + Np * (w8 * d + wr * (d + dd) + 4) + Ga * w8 * d
    if name == "k_defgrad":
        return Np * (w8 * d + wr * (dd + 5)) + Ga * w8 * d + Np * wr * (dd + 6 + ns)
    if name == "k_grid":
        return G * (2 * wr * (2 + 2 * d) + w8 * d + wr * (d + 1))
    if name == "k_musl_norm":
        return G * (wr + 2 * w8 * d)
    if name.startswith("k_sort_hist"):
        return Np * (w8 * d + 4) if "keys" in name else Np * 4
    if name == "k_sort_scatter":
        return Np * 16
    if name == "k_bbox":
        return Np * (w8 * d + wr * d)
    return None


def roofline_of(kernel_ms, p, Np, Ga, G, wr):
    """Roofline of the dominant kernel among per-launch kernel times
    (`kernel_ms`: name -> ms per launch): its algorithmic bytes per launch
    (kernel_bytes) over its time, against the measured HBM peak."""
    peak, peak_kind = hbm_peak()
    dom = max((k for k in kernel_ms if k.startswith("k_")), key=lambda k: kernel_ms[k])
    dom_bytes = kernel_bytes(dom, p, Np, Ga, G, wr)
    achieved = dom_bytes / (kernel_ms[dom] / 1e3) / 1e9 if dom_bytes else None
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
            "kernel_ms": kernel_ms[dom], "kernel_algorithmic_bytes": dom_bytes, "active_nodes": Ga,
            "grid_nodes": G}


def step_bytes(p, Np, Ga, wr=8.0):
    """Whole-step algorithmic bytes: the persistent particle state read and
    written once (x v F B + 3 plastic scalars read; the same + 3 diagnostics
    written), plus the grid term (mass and momentum written and read,
    velocity and flip written and read) per node with mass."""
    d = p.dim
    dd = d * d
    per_particle = 2 * 8.0 * d + wr * ((d + 2 * dd + 3) + (d + 2 * dd + 6))
    per_node = (1 + d) * 2 + 2 * d * 2
    return Np * per_particle + Ga * wr * per_node


# ---------------------------------------------------------------------------
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_threads(Np):
    """OpenMP threads for the reference: all host threads, bounded by memory
    (its G2P allocates three Np-sized arrays per thread every step,
    g2p.cpp:19-21)."""
    n = cpu_threads()
    per_thread = Np * 8.0 * (3 + 3 + 9) * 1.2
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        avail = 16e9
    return max(1, min(n, int(0.5 * avail / per_thread)))


class quiet_stdout:
    """Silences fd 1 while the reference runs (Simulation prints banners)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False


def run_cpu_reference(scene, budget_s, max_steps=None, warmup=1):
    with quiet_stdout():
        return _run_cpu_reference(scene, budget_s, max_steps, warmup)


def _run_cpu_reference(scene, budget_s, max_steps=None, warmup=1):
    """Times the reference's own OpenMP step (oracle/_ref) on the workload.
    Returns (particle-steps/s, threads, kind, sample description)."""
    from oracle.checkers import Oracle, Reference, reference_available
    if reference_available(scene.params.dim, scene.params.spline_deg):
        threads = reference_threads(scene.Np)
        c = Reference(scene.params, n_threads=threads)
        kind = "reference"
    else:
        threads = 1
        c = Oracle(scene.params)
        kind = "port"
    c.set_particles(scene.x, scene.v, scene.F, scene.B, scene.scalars)
    c.set_objects(scene.plates, scene.objects)
    c.step(warmup)
    t0 = time.perf_counter()
    n = c.step(1)
    t1 = time.perf_counter()
    per = max(t1 - t0, 1e-6)
    steps = max(1, int(budget_s / per) - 1)
    if max_steps is not None:
        steps = min(steps, max_steps)
    t0 = time.perf_counter()
    n += c.step(steps)
    el = time.perf_counter() - t0 + per
    c.close()
    rate = scene.Np * n / el
    sample = (f"{n} steps of the full {scene.Np}-particle workload after {warmup} warm-up step(s), "
              f"{threads} OpenMP thread(s), wall clock")
    return rate, threads, kind, sample, el / n


def build_scene(args, rank):
    from matter_tests_b200 import scenes
    sc = scenes.WORKLOADS[args.workload](scale=args.scale)
    return sc


def config_of(args, sc):
    p = sc.params
    sym = 6 if p.dim == 3 else 3
    return {"workload": f"{sc.name}: {args.workload} scale {args.scale}", "Np": sc.Np, "dim": p.dim,
            "spline_deg": p.spline_deg, "musl": bool(p.use_musl), "flip_ratio": p.flip_ratio,
            "plastic_model": int(p.plastic_model), "dx": p.dx, "precision": "fp64",
            "l2": "inputs larger than L2: particle state 2 x %.0f MB (FP64), 2 x %.0f MB (mixed)" % (
                sc.Np * (8 * (2 * p.dim + 2 * p.dim ** 2 + 6 + sym)) / 1e6,
                sc.Np * (8 * p.dim + 4 * (p.dim + 2 * p.dim ** 2 + 6 + sym)) / 1e6),
            "parallelism": "replicas"}


# ---------------------------------------------------------------------------
def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    sc = build_scene(args, rank)
    budget = max(5.0, min(240.0, 6.0 * (args.steps + args.warmup)))
    rate, threads, kind, sample, sec_per_step = run_cpu_reference(
        sc, budget, max_steps=args.steps, warmup=max(1, min(args.warmup, 3)))
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec_per_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded jittered lattice)", "config": config_of(args, sc),
            "cpu_baseline": {"value": rate, "unit": METRIC, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def measure(args, world, rank, local, sc, precision, sampler=None):
    """Times one precision of the step on the scene: device-timed K steps,
    per-kernel profile, roofline of the dominant kernel, and the end-to-end
    run through the C ABI with pinned host buffers.  Returns a dict and the
    particle state after warmup + K steps."""
    import ctypes
    import copy
    import numpy as np
    import torch
    from matter_tests_b200.abi import PREC_MIXED
    from matter_tests_b200.gpu import GpuSim

    p = copy.copy(sc.params)
    p.precision = precision
    wr = 4.0 if precision == PREC_MIXED else 8.0
    g = GpuSim(p, device=local)
    g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
    g.set_objects(sc.plates, sc.objects)
    g.step(args.warmup)
    # block shapes of the tile kernels, tuned on the warmed-up scene (setup, untimed)
    if not args.no_autotune:
        g.autotune(args.tune_reps)
    shapes = {"threads": g.tile_threads, "lanes_per_particle": g.tile_lanes}
    stream = torch.cuda.ExternalStream(g.stream, device=torch.device("cuda", local))
    barrier(world)
    torch.cuda.synchronize(local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    g.step(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize(local)
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    launches = g.launch_count()
    ck = g.clock()
    state = g.particles()
    ms_max = max_over_ranks(world, ms, local)
    value = sc.Np * args.steps * world / (ms_max / 1e3)

    # per-kernel profile of the same state (CUDA events between launches),
    # after one untimed profiled step
    g.profile(1)
    slots = g.profile(args.profile_steps)
    Ga, G = g.active_nodes()
    peak, peak_kind = hbm_peak()
    agg = {}
    for name, t in slots:
        agg[name] = agg.get(name, 0.0) + t
    dom = max((k for k in agg if k.startswith("k_")), key=lambda k: agg[k])
    dom_ms = agg[dom] / sum(1 for n, _ in slots if n == dom)
    dom_bytes = kernel_bytes(dom, p, sc.Np, Ga, G, wr)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9 if dom_bytes else None
    step_ms = sum(t for _, t in slots)
    whole = step_bytes(p, sc.Np, Ga, wr) / (ms / args.steps / 1e3) / 1e9

    # end to end through the C ABI with pinned host buffers
    d = p.dim
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hx, hv, hF, hB, hs = pin(sc.Np * d), pin(sc.Np * d), pin(sc.Np * d * d), pin(sc.Np * d * d), pin(sc.Np * 6)
    hx[:] = sc.x.reshape(-1)
    hv[:] = 0.0 if sc.v is None else sc.v.reshape(-1)
    hF[:] = np.tile(np.eye(d).reshape(-1), sc.Np) if sc.F is None else sc.F.reshape(-1)
    hB[:] = 0.0 if sc.B is None else sc.B.reshape(-1)
    hs[:] = 0.0 if sc.scalars is None else sc.scalars.reshape(-1)
    ox, ov, oF, oB, os_ = pin(sc.Np * d), pin(sc.Np * d), pin(sc.Np * d * d), pin(sc.Np * d * d), pin(sc.Np * 6)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    barrier(world)
    t0 = time.perf_counter()
    g.upload(hx, hv, hF, hB, hs)
    g.set_objects(sc.plates, sc.objects)
    t1 = time.perf_counter()
    g.step(args.steps)
    t2 = time.perf_counter()
    rc = g.lib.mtr_download(g.h, dp(ox), dp(ov), dp(oF), dp(oB), dp(os_))
    assert rc == 0, rc
    t3 = time.perf_counter()
    e2e_s = max_over_ranks(world, t3 - t0, local)
    io_bytes = 8 * sc.Np * (2 * d + 2 * d * d + 6)
    status, _ = g.status()
    g.close()
    # the first upload into a fresh context (allocation included), for reference
    g2 = GpuSim(p, device=local)
    t4 = time.perf_counter()
    g2.upload(hx, hv, hF, hB, hs)
    t5 = time.perf_counter()
    g2.close()
    e2e = {"value": sc.Np * args.steps * world / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": io_bytes / args.steps, "d2h_bytes_per_step": io_bytes / args.steps,
           "split_ms": {"upload": (t1 - t0) * 1e3, "steps": (t2 - t1) * 1e3, "download": (t3 - t2) * 1e3},
           "fresh_context_upload_ms": (t5 - t4) * 1e3,
           "timed": "mtr_upload (pinned host) + mtr_step(K) + mtr_download, wall clock, into a context already "
                    "holding a scene of this size"}
    traffic, traffic_src = measured_traffic(args.workload, args.scale, dom,
                                            "mixed" if precision == PREC_MIXED else "fp64")
    out = {"value": value, "ms_per_step": ms_max / args.steps,
           "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                        "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                        "traffic": traffic, "traffic_source": traffic_src,
                        "pipes": measured_pipes(args.workload, args.scale, dom,
                                                "mixed" if precision == PREC_MIXED else "fp64"),
                        "peak_source": peak_kind,
                        "kernel_ms": dom_ms, "kernel_algorithmic_bytes": dom_bytes,
                        "step_algorithmic_GBps": whole, "step_frac": whole / peak,
                        "active_nodes": Ga, "grid_nodes": G},
           "kernel_ms": {k: round(v / max(1, sum(1 for n, _ in slots if n == k)), 5) for k, v in agg.items()},
           "profiled_step_ms": step_ms, "e2e": e2e, "gpu_launches": launches, "tile_threads": shapes,
           "sim_clock": {"step": ck["step"], "time": ck["time"]}, "status_flags": status}
    return out, state


def hencky_tau(F, E, nu):
    """Kirchhoff stress of the Hencky model for a batch of F (n, d, d)."""
    import numpy as np
    lam = nu * E / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    U, S, _ = np.linalg.svd(F)
    h = np.log(np.maximum(np.abs(S), 1e-300))
    e = 2 * mu * h + lam * h.sum(axis=1, keepdims=True)
    return np.einsum("nij,nj,nkj->nik", U, e, U)


def mixed_error(sc, ref, got):
    """Error of the mixed-precision state against the FP64 state after the
    same steps: positions in units of dx, velocity and Kirchhoff stress
    relative to their largest magnitude."""
    import numpy as np
    p = sc.params
    dxp = np.abs(got["x"] - ref["x"]) / p.dx
    vs = np.abs(ref["v"]).max()
    Fr = np.transpose(ref["F"], (0, 2, 1))  # column-major host layout -> (n, r, c)
    Fg = np.transpose(got["F"], (0, 2, 1))
    tr, tg = hencky_tau(Fr, p.E, p.nu), hencky_tau(Fg, p.E, p.nu)
    ts = np.abs(tr).max()
    return {"x_max_over_dx": float(dxp.max()), "x_rms_over_dx": float(np.sqrt((dxp ** 2).mean())),
            "v_max_rel": float(np.abs(got["v"] - ref["v"]).max() / vs) if vs > 0 else None,
            "tau_max_rel": float(np.abs(tg - tr).max() / ts) if ts > 0 else None,
            "F_max_abs": float(np.abs(got["F"] - ref["F"]).max())}


# the single-scene workloads at full size and their full lengths
CONFIG_RUNS = (("collapse2d", 2000), ("collapse3d_mui", 1000), ("incline3d_mcc", 3000))


def config_runs(args, local):
    """Each single-scene workload at full size over its full length, plain
    FP64 and mixed: device-timed particle-steps/s (16 untimed steps first,
    which capture the step graphs; the block shapes tuned after them), the
    per-kernel times of 3 profiled steps after the run with the roofline of
    the dominant kernel there, and the mixed state's error against the FP64
    state at the last step."""
    import copy
    import torch
    from matter_tests_b200 import scenes
    from matter_tests_b200.abi import PREC_FP64, PREC_MIXED
    from matter_tests_b200.gpu import GpuSim
    out = {}
    for name, nsteps in CONFIG_RUNS:
        sc = scenes.WORKLOADS[name](scale=1.0)
        res, states = {}, {}
        for prec, key in ((PREC_FP64, "fp64"), (PREC_MIXED, "mixed")):
            p = copy.copy(sc.params)
            p.precision = prec
            g = GpuSim(p, device=local)
            g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
            g.set_objects(sc.plates, sc.objects)
            warm = 16
            g.step(warm)
            if not args.no_autotune:
                g.autotune(args.tune_reps)
            st = torch.cuda.ExternalStream(g.stream, device=torch.device("cuda", local))
            torch.cuda.synchronize(local)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            g.step(nsteps - warm)
            b.record(st)
            b.synchronize()
            ms = a.elapsed_time(b)
            ck = g.clock()
            states[key] = g.particles()
            status, _ = g.status()
            slots = g.profile(3)
            Ga, G = g.active_nodes()
            agg, cnt = {}, {}
            for kn, t in slots:
                agg[kn] = agg.get(kn, 0.0) + t
                cnt[kn] = cnt.get(kn, 0) + 1
            g.close()
            kms = {k: agg[k] / cnt[k] for k in agg}
            res[key] = {"value": sc.Np * (nsteps - warm) / (ms / 1e3), "ms_per_step": ms / (nsteps - warm),
                        "steps": int(ck["step"]), "status_flags": status,
                        "kernel_ms": {k: round(v, 5) for k, v in kms.items()},
                        "roofline": roofline_of(kms, p, sc.Np, Ga, G, 4.0 if prec == PREC_MIXED else 8.0)}
        err = mixed_error(sc, states["fp64"], states["mixed"])
        out[name] = {"Np": sc.Np, "steps": nsteps, "fp64": res["fp64"], "mixed": res["mixed"],
                     "mixed_over_fp64": res["mixed"]["value"] / res["fp64"]["value"],
                     "mixed_error_vs_fp64": err}
    return out


def ensemble_measure(args, local):
    """The batched ensemble: args.ensemble_size seeded DP column collapses
    (5k-300k particles, half 3D), mixed precision, stepped together through
    mtr_batch (one launch per phase per group, CUDA graphs) for
    args.ensemble_steps timed steps after args.warmup and the shape tuner,
    against the same scenes run one after another through their own contexts
    (each tuned too).  Step latency: wall time of each mtr_batch_step(8) / 8.
    shapes_ab: tuned against default shapes, interleaved on the same batch."""
    import numpy as np
    import torch
    from matter_tests_b200 import scenes
    from matter_tests_b200.abi import PREC_MIXED
    from matter_tests_b200.gpu import GpuBatch, GpuSim
    scs = scenes.ensemble(n=args.ensemble_size)
    for sc in scs:
        sc.params.precision = PREC_MIXED
    ntot = sum(sc.Np for sc in scs)
    K, W = args.ensemble_steps, max(args.warmup, 3)

    def make(sc):
        g = GpuSim(sc.params, device=local)
        g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
        g.set_objects(sc.plates, sc.objects)
        return g

    def timed(b, k):
        st = torch.cuda.ExternalStream(b.stream, device=torch.device("cuda", local))
        torch.cuda.synchronize(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        b.step(k)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    sims = [make(sc) for sc in scs]
    batch = GpuBatch(sims)
    batch.step(W)
    default = [(gr["tile_threads"], gr["tile_lanes"]) for gr in batch.groups()]
    if not args.no_autotune:
        batch.autotune(args.tune_reps)  # setup, untimed: trial steps leave the scenes as they are
        batch.set_retune(args.tune_reps)  # and again inside the timed steps when a group's grids double
    ms = timed(batch, K)
    launches = batch.launch_count()
    retunes = batch.retunes()  # re-tunes inside the timed steps (a group's grids doubled)
    groups = batch.groups()    # the shapes after the timed steps
    # tuned against default shapes on the same batch, interleaved in rounds of
    # 16 steps so that both see the same states; after each switch 8 untimed
    # steps rebuild the batch's graph outside the timed window
    ab = None
    if not args.no_autotune:
        tuned = [(gr["tile_threads"], gr["tile_lanes"]) for gr in groups]
        t_ms = {"tuned": 0.0, "default": 0.0}
        for _ in range(4):
            for name, shapes in (("default", default), ("tuned", tuned)):
                for gi, (th, ln) in enumerate(shapes):
                    batch.set_tile_threads(gi, th)
                    batch.set_tile_lanes(gi, ln)
                batch.step(8)
                t_ms[name] += timed(batch, 16)
        ab = {"tuned_over_default": t_ms["default"] / t_ms["tuned"], "steps_each": 64,
              "timed": "4 interleaved rounds of 16 batched steps per shape set (after 8 untimed steps each), "
                       "CUDA events"}
    lat = []
    for _ in range(max(8, K // 8)):
        t0 = time.perf_counter()
        batch.step(8)
        lat.append((time.perf_counter() - t0) / 8 * 1e3)
    steps_done = [g.clock()["step"] for g in sims]
    batch.close()
    for g in sims:
        g.close()
    # the same scenes one at a time, each through its own graphs
    serial_ms = 0.0
    for sc in scs:
        g = make(sc)
        g.step(W)
        if not args.no_autotune:
            g.autotune(args.tune_reps)
        st = torch.cuda.ExternalStream(g.stream, device=torch.device("cuda", local))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        g.step(K)
        b.record(st)
        b.synchronize()
        serial_ms += a.elapsed_time(b)
        g.close()
    n3 = sum(1 for sc in scs if sc.dim == 3)
    value = ntot * K / (ms / 1e3)
    serial = ntot * K / (serial_ms / 1e3)
    return {"metric": "ensemble particle-steps/s", "value": value, "unit": METRIC, "scenes": len(scs),
            "scenes_3d": n3, "particles": ntot, "steps": K, "warmup": W, "ms_per_batched_step": ms / K,
            "step_latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                "samples": len(lat), "timed": "wall time of mtr_batch_step(8) / 8"},
            "serial": {"value": serial, "ms_total": serial_ms,
                       "timed": "each scene alone through its own context and graphs, CUDA events"},
            "batched_over_serial": value / serial, "gpu_launches": launches, "dtype": "f32+f64",
            "groups": groups, "retunes": retunes, "shapes_ab": ab,
            "config": "seeded DP column collapses: Np log-uniform 5k-300k, P(3D) 0.5, aspect U(0.5,4), "
                      "friction angle U(20,40) deg, E log-uniform 1e5-1e7 Pa, APIC USL, quadratic",
            "all_scenes_advanced": bool(min(steps_done) >= W + K)}


def serve_measure(args, local):
    """The serving loop: args.serve_requests seeded requests (2D/3D, collapse
    or incline, 10k-2M particles, DP / Cam-Clay / mu(I), 200 steps each)
    arriving as a Poisson process at 20 per second, admitted within a 150 GB
    device-memory budget, mixed precision, stepped together in ticks of up to
    8 steps sized to a 16 ms frame interval; and the same requests again in
    ticks of 8 steps each (`fixed_ticks`).
    Against it: the same requests one after another through the plain FP64
    single-scene path and the mixed single-scene path (device-timed steps)."""
    import copy
    import torch
    from matter_tests_b200.abi import PREC_FP64, PREC_MIXED
    from matter_tests_b200.gpu import GpuSim
    import numpy as np
    from matter_tests_b200 import scenes
    from matter_tests_b200.serve import Request, Server, poisson_requests
    # start-up, untimed: one 200k-particle request of every kind (dimension x
    # collapse or incline x material) through a warm-up server loads the
    # batched kernels of every group the measured run will meet and tunes
    # their shapes (the measured server starts from those shapes); two 2M
    # requests besides them take the device allocations up to the largest
    # request's size once
    rng = np.random.default_rng(1)
    kinds = [(d, k, m, 200_000) for d in (2, 3) for k in ("collapse", "incline") for m in ("dp", "mcc", "mui")]
    kinds += [(3, "collapse", "dp", 2_000_000)] * 2
    warm = [Request(rid=i, scene=scenes.granular_scene(rng, dim, kind, n, mat, 1e6, 30.0, 2.0), steps=16,
                    arrival=0.0)
            for i, (dim, kind, mat, n) in enumerate(kinds)]
    warm_srv = Server(budget_bytes=150e9, device=local, tick_steps=8, precision=PREC_MIXED)
    warm_srv.run(warm, realtime=False)
    reqs = poisson_requests(args.serve_requests, rate=20.0, seed=4242, steps=200)
    # the measured run: ticks sized to a 16 ms frame interval (1-8 steps)
    srv = Server(budget_bytes=150e9, device=local, tick_steps=8, precision=PREC_MIXED, shapes=warm_srv.shapes,
                 frame_ms=16.0)
    done = srv.run(reqs)
    rep = srv.report(done)
    # beside it, the same requests with every tick 8 steps (no frame interval)
    fixed_srv = Server(budget_bytes=150e9, device=local, tick_steps=8, precision=PREC_MIXED, shapes=warm_srv.shapes)
    fixed = fixed_srv.report(fixed_srv.run(poisson_requests(args.serve_requests, rate=20.0, seed=4242, steps=200)))
    serial = {}
    for prec, name in ((PREC_FP64, "fp64"), (PREC_MIXED, "mixed")):
        ms, ps = 0.0, 0
        for r in reqs:
            p = copy.copy(r.scene.params)
            p.precision = prec
            g = GpuSim(p, device=local)
            sc = r.scene
            g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
            g.set_objects(sc.plates, sc.objects)
            st = torch.cuda.ExternalStream(g.stream, device=torch.device("cuda", local))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            g.step(r.steps, check=False)
            b.record(st)
            b.synchronize()
            ms += a.elapsed_time(b)
            ps += sc.Np * g.clock()["step"]
            g.close()
        serial[name] = ps / (ms / 1e3)
    rep.update({"metric": "served particle-steps/s", "unit": METRIC, "dtype": "f32+f64",
                "single_scene_fp64": serial["fp64"], "single_scene_mixed": serial["mixed"],
                "served_over_single_scene_fp64": rep["throughput"] / serial["fp64"],
                "served_over_single_scene_mixed": rep["throughput"] / serial["mixed"],
                "fixed_ticks": {"throughput": fixed["throughput"],
                                "served_over_single_scene_mixed": fixed["throughput"] / serial["mixed"],
                                "frame_latency_ms": fixed["frame_latency_ms"], "ticks": fixed["ticks"]},
                "config": "Poisson arrivals 20/s (seed 4242), Np log-uniform 10k-2M, 2D/3D collapse or incline, "
                          "DP/MCC/mu(I), 200 steps, 150 GB budget, ticks of up to 8 steps sized to a 16 ms "
                          "frame interval (fixed_ticks: every tick 8 steps)",
                "timed": "throughput = particle-steps of the served requests / (last completion - first "
                         "arrival), wall clock; single-scene figures are device time of the steps alone"})
    return rep


def gpu_arm(args, world, rank, local):
    import torch
    from matter_tests_b200.abi import PREC_FP64, PREC_MIXED

    torch.cuda.set_device(local)
    sc = build_scene(args, rank)
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    if args.precision != "both":  # one form alone (profiler captures): a reduced line
        prec = PREC_FP64 if args.precision == "fp64" else PREC_MIXED
        one, _ = measure(args, world, rank, local, sc, prec)
        clocks = sampler.stop()
        if rank == 0:
            cfg = config_of(args, sc)
            cfg["precision"] = args.precision
            print(json.dumps({"metric": METRIC, "value": one["value"], "unit": METRIC, "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": one["ms_per_step"],
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "f64" if prec == PREC_FP64 else "f32+f64",
                              "data": "synthetic (seeded jittered lattice)", "config": cfg,
                              "roofline": one["roofline"], "kernel_ms": one["kernel_ms"], "e2e": one["e2e"],
                              "gpu_launches": one["gpu_launches"], "clocks": clocks}), flush=True)
        return 0
    fp64, st64 = measure(args, world, rank, local, sc, PREC_FP64)
    mixed, st32 = measure(args, world, rank, local, sc, PREC_MIXED)
    cfgs = None
    if rank == 0 and world == 1 and not args.no_configs:
        try:
            cfgs = config_runs(args, local)
        except Exception as e:  # reported, not fatal: the headline line still prints
            cfgs = {"error": f"{type(e).__name__}: {e}"}
    ens = None
    if rank == 0 and world == 1 and not args.no_ensemble:
        try:
            ens = ensemble_measure(args, local)
        except Exception as e:  # reported, not fatal: the headline line still prints
            ens = {"error": f"{type(e).__name__}: {e}"}
    served = None
    if rank == 0 and world == 1 and not args.no_serve:
        try:
            served = serve_measure(args, local)
        except Exception as e:  # reported, not fatal: the headline line still prints
            served = {"error": f"{type(e).__name__}: {e}"}
    clocks = sampler.stop()
    err = mixed_error(sc, st64, st32)
    err["steps"] = args.warmup + args.steps

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, threads, kind, sample, _ = run_cpu_reference(sc, args.cpu_seconds)
        cpu = {"value": rate, "unit": METRIC, "cores": threads, "kind": kind, "sample": sample}

    if rank == 0:
        cfg = config_of(args, sc)
        line = {"metric": METRIC, "value": fp64["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": fp64["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded jittered lattice)", "config": cfg,
                "roofline": fp64["roofline"], "kernel_ms": fp64["kernel_ms"],
                "profiled_step_ms": fp64["profiled_step_ms"], "cpu_baseline": cpu, "e2e": fp64["e2e"],
                "gpu_launches": fp64["gpu_launches"], "clocks": clocks, "tile_threads": fp64["tile_threads"],
                "mixed": {"value": mixed["value"], "unit": METRIC, "ms_per_step": mixed["ms_per_step"],
                          "dtype": "f32+f64",
                          "precision": "FP32 state and transfers; FP64 positions, SVD, Hencky log/exp, return "
                                       "mapping projections, balances",
                          "mixed_over_fp64": mixed["value"] / fp64["value"], "error_vs_fp64": err,
                          "roofline": mixed["roofline"], "kernel_ms": mixed["kernel_ms"], "e2e": mixed["e2e"],
                          "gpu_launches": mixed["gpu_launches"], "tile_threads": mixed["tile_threads"],
                          "status_flags": mixed["status_flags"]},
                "configs": cfgs, "ensemble": ens, "serving": served,
                "sim_clock": fp64["sim_clock"], "status_flags": fp64["status_flags"]}
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            return reference_arm(args, world, rank)
        return gpu_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
