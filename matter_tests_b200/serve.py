"""Serving loop: scenes arrive as requests, are admitted by their device-memory
footprint, and every admitted scene advances in one batch (mtr_batch: one
launch per step phase for all scenes of a group, replayed from a CUDA graph).

Continuous batching: a request that arrives while others run is prepared
(context created, particles uploaded) on a worker thread while the batch
keeps stepping, and joins at the next tick; a finished scene leaves at the
tick it completes, its result is read back and its memory freed on the
worker, and the memory it frees admits the next waiting request.  One batch
lives through the whole run: joining and leaving replace its members
(mtr_batch_set_members), which keeps its stream, its groups' block shapes
and its step graph, updated in place rather than instantiated again.  A tick
advances every member by `tick_steps` steps; each member has a step limit,
so it stops exactly after the steps it asked for.

Frame interval: with `frame_ms` set, a tick takes as many steps (1 to
`tick_steps`) as a step-time model predicts will fit into `frame_ms` for the
particles admitted at the time, so that ticks keep their cadence when a burst
of arrivals makes the batch large.  The model is a least-squares line, ms per
step against particles stepped, over the recent ticks that neither followed a
membership change nor regrew a grid; until it has four, ticks take one step.

Finished contexts are released lazily: a request's result is read back when
it completes, but its device memory is freed only when the budget needs the
room for a waiting request (or at the end of the run), because freeing device
memory waits for the whole GPU to go idle and would stall the running batch.

Block shapes of the tile kernels: the first batch that holds a group key
(dimension, spline, precision, USL/MUSL, return-mapping kernel) is tuned
(mtr_batch_autotune, trial steps that leave the scenes as they were); later
batches take the shapes cached for their keys.

No counterpart in the reference, which runs one Simulation per process.
"""
import collections
import concurrent.futures as cf
import copy
import time
from dataclasses import dataclass, field

import numpy as np

from .abi import PREC_MIXED
from .gpu import GpuBatch, GpuSim, footprint


@dataclass
class Request:
    rid: int
    scene: object
    steps: int
    arrival: float                 # seconds after the start of the run
    footprint: int = 0
    admitted: float = None
    started: float = None          # first tick it took part in
    done: float = None
    result: dict = None
    sim: object = field(default=None, repr=False)


class Server:
    """Admits requests under `budget_bytes` of device memory and steps all
    admitted scenes together.  `precision` overrides each scene's precision
    (None keeps it)."""

    def __init__(self, budget_bytes, device=0, tick_steps=8, precision=PREC_MIXED, keep_result=("x", "v"),
                 autotune=True, tune_reps=3, workers=1, shapes=None, frame_ms=None):
        self.frame_ms = frame_ms  # target wall time of a tick (None: every tick takes tick_steps steps)
        self._fit = collections.deque(maxlen=64)  # (particles, ms per step) of clean ticks
        self.workers = int(workers)  # threads that prepare, read back and release requests
        self.autotune = autotune
        self.tune_reps = int(tune_reps)
        # group key -> tile-kernel block shapes; a server can start from the
        # shapes another one tuned (a warm-up run at start-up)
        self.shapes = dict(shapes or {})
        self.budget = int(budget_bytes)
        self.device = device
        self.tick_steps = int(tick_steps)
        self.precision = precision
        self.keep = keep_result
        self.tick_ms = []        # wall time of each tick
        self.tick_members = []   # scenes stepped in each tick
        self.tick_particles = []  # particles stepped in each tick
        self.tick_rebuilt = []   # the tick's batch was (re)built just before it
        self.tick_regrown = []   # a member's grid outgrew its capacity inside the tick
        self.tick_worker = []    # a request was being prepared or read back during the tick
        self.tick_nsteps = []    # steps the tick took
        self.peak_members = 0
        self.peak_bytes = 0
        # wall time outside the ticks, by cause (seconds)
        self.host_s = {"idle": 0.0, "batch_build": 0.0, "release": 0.0}
        self.graph_updates = 0   # batch rebuilds that updated the step graph in place
        self.wall_s = 0.0        # wall time of the last run()

    # -- worker-thread jobs -------------------------------------------------
    def _prepare(self, req):
        sc = req.scene
        p = copy.copy(sc.params)
        if self.precision is not None:
            p.precision = self.precision
        g = GpuSim(p, device=self.device)
        g.upload(sc.x, sc.v, sc.F, sc.B, sc.scalars)
        g.set_objects(sc.plates, sc.objects)
        g.set_step_limit(req.steps)
        return g

    def _finish(self, req):
        st = req.sim.particles(fields=self.keep)  # only what the result keeps is read back
        req.result = {k: st[k] for k in self.keep}
        req.result["clock"] = req.sim.clock()
        req.result["status"] = req.sim.status()

    @staticmethod
    def _release(req):
        req.sim.close()
        req.sim = None

    # -- the loop -------------------------------------------------------------
    def run(self, requests, realtime=True):
        """Serves `requests` (arrival times relative to the start) and
        returns them completed.  With realtime=False arrivals are ignored and
        everything is queued at the start."""
        queue_in = collections.deque(sorted(requests, key=lambda r: r.arrival))
        for r in queue_in:
            if r.footprint == 0:
                p = copy.copy(r.scene.params)
                if self.precision is not None:
                    p.precision = self.precision
                r.footprint = footprint(p, r.scene.x)
            if r.footprint > self.budget:
                raise ValueError(f"request {r.rid} needs {r.footprint} bytes, more than the budget")
        waiting = collections.deque()
        preparing = {}      # future -> request
        finishing = []      # futures
        retired = collections.deque()  # (finish future, request): read back, memory still held
        active = []
        used = 0
        batch = None
        members_key = None
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        done = []
        with cf.ThreadPoolExecutor(max_workers=self.workers) as pool:
            while queue_in or waiting or preparing or active:
                t = now()
                while queue_in and (not realtime or queue_in[0].arrival <= t):
                    waiting.append(queue_in.popleft())
                # lazy release: free finished requests' memory only when a waiting one needs it
                while waiting and used + waiting[0].footprint > self.budget and retired:
                    tr = now()
                    f, r = retired.popleft()
                    f.result()
                    pool.submit(self._release, r).result()
                    used -= r.footprint
                    self.host_s["release"] += now() - tr
                # admission: first come, first served, within the memory budget
                while waiting and used + waiting[0].footprint <= self.budget:
                    r = waiting.popleft()
                    r.admitted = now()
                    used += r.footprint
                    self.peak_bytes = max(self.peak_bytes, used)
                    preparing[pool.submit(self._prepare, r)] = r
                for f in [f for f in preparing if f.done()]:
                    r = preparing.pop(f)
                    r.sim = f.result()
                    active.append(r)
                if not active:
                    ti = now()
                    if preparing:
                        cf.wait(list(preparing), return_when=cf.FIRST_COMPLETED)
                    elif queue_in:
                        time.sleep(max(0.0, min(0.05, queue_in[0].arrival - now())))
                    self.host_s["idle"] += now() - ti
                    continue
                key = tuple(r.rid for r in active)
                rebuilt = key != members_key
                if rebuilt:
                    tb = now()
                    if batch is None:
                        batch = GpuBatch([r.sim for r in active])
                    else:
                        batch.set_members([r.sim for r in active])
                    members_key = key
                    if self.autotune:
                        self._shape(batch)
                    self.host_s["batch_build"] += now() - tb
                ts = now()
                for r in active:
                    if r.started is None:
                        r.started = ts
                worker = bool(preparing) or any(not f.done() for f in finishing)
                regrowths = batch.stats()["regrowths"]
                particles = sum(r.scene.Np for r in active)
                nsteps = self._tick_steps(particles)
                batch.step(nsteps)
                tick_ms = (now() - ts) * 1e3
                regrown = batch.stats()["regrowths"] > regrowths
                self.tick_ms.append(tick_ms)
                self.tick_nsteps.append(nsteps)
                self.tick_members.append(len(active))
                self.tick_particles.append(particles)
                self.tick_rebuilt.append(rebuilt)
                self.tick_regrown.append(regrown)
                self.tick_worker.append(worker or any(not f.done() for f in preparing))
                if not rebuilt and not regrown:
                    self._fit.append((particles, tick_ms / nsteps))
                self.peak_members = max(self.peak_members, len(active))
                still = []
                for r, ck in zip(active, batch.clocks()):
                    if ck["step"] >= r.steps or ck["done"]:
                        r.done = now()
                        f = pool.submit(self._finish, r)
                        finishing.append(f)
                        retired.append((f, r))
                        done.append(r)
                    else:
                        still.append(r)
                if len(still) != len(active):
                    # the finished members leave the batch before their contexts are freed
                    if still:
                        batch.set_members([r.sim for r in still])
                        members_key = tuple(r.rid for r in still)
                    else:
                        self.graph_updates += batch.graph_updates()
                        batch.close()
                        batch = None
                        members_key = None
                active = still
            if batch is not None:
                self.graph_updates += batch.graph_updates()
                batch.close()
            for f in finishing:
                f.result()
            self.wall_s = now()
            for f, r in retired:
                pool.submit(self._release, r).result()
        return done

    def _tick_steps(self, particles):
        """Steps of the next tick: tick_steps, or with frame_ms set, the steps
        the step-time model fits into frame_ms (at least 1)."""
        if self.frame_ms is None:
            return self.tick_steps
        if len(self._fit) < 4:  # no model yet: one step, the shortest tick there is
            return 1
        P = np.array([p for p, _ in self._fit], dtype=np.float64)
        T = np.array([t for _, t in self._fit], dtype=np.float64)
        a, b = np.linalg.lstsq(np.stack([np.ones_like(P), P], 1), T, rcond=None)[0]
        if a < 0.0 or b <= 0.0:  # degenerate fit (too narrow a spread of batch sizes): proportional
            a, b = 0.0, float(np.mean(T / P))
        est = a + b * particles
        return int(np.clip(np.floor(self.frame_ms / est), 1, self.tick_steps))

    @staticmethod
    def _key(gr):
        return (gr["dim"], gr["spline_deg"], gr["fp32"], gr["musl"], gr["plastic_model_kernel"])

    def _shape(self, batch):
        """Applies the cached block shapes of the batch's groups; tunes the
        batch when a group key is new."""
        groups = batch.groups()
        if any(self._key(gr) not in self.shapes for gr in groups):
            groups = batch.autotune(self.tune_reps)
            for gr in groups:
                self.shapes.setdefault(self._key(gr), {"threads": gr["tile_threads"], "lanes": gr["tile_lanes"]})
        for i, gr in enumerate(groups):
            sh = self.shapes[self._key(gr)]
            if gr["tile_threads"] != sh["threads"]:
                batch.set_tile_threads(i, sh["threads"])
            if gr["tile_lanes"] != sh["lanes"]:
                batch.set_tile_lanes(i, sh["lanes"])

    # -- report ---------------------------------------------------------------
    def _split(self, frame):
        rb = np.array(self.tick_rebuilt, dtype=bool)
        rg = np.array(self.tick_regrown, dtype=bool)
        wk = np.array(self.tick_worker, dtype=bool)
        mp = np.array(self.tick_particles, dtype=np.float64) / 1e6
        out = {}
        for name, m in (("after_rebuild", rb), ("steady", ~rb), ("with_regrowth", rg),
                        ("worker_busy", wk & ~rg), ("neither", ~rg & ~wk)):
            if m.any():
                out[name] = {"ticks": int(m.sum()), "p50": float(np.percentile(frame[m], 50)),
                             "p99": float(np.percentile(frame[m], 99)),
                             "per_mparticle_p50": float(np.percentile(frame[m] / np.maximum(mp[m], 1e-9), 50)),
                             "per_mparticle_p99": float(np.percentile(frame[m] / np.maximum(mp[m], 1e-9), 99))}
        return out

    def report(self, done):
        lat = np.array([r.done - r.arrival for r in done])
        wait = np.array([r.admitted - r.arrival for r in done])
        psteps = sum(r.scene.Np * r.steps for r in done)
        per_step = np.array(self.tick_ms) / np.array(self.tick_nsteps, dtype=np.float64)
        frame = np.array(self.tick_ms)
        span = max(r.done for r in done) - min(r.arrival for r in done)
        return {
            "requests": len(done),
            "requests_with_device_status": sum(1 for r in done if r.result and r.result["status"][0]),
            "particle_steps": psteps,
            "throughput": psteps / span,
            "request_latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "queue_wait_s": {"p50": float(np.percentile(wait, 50)), "p99": float(np.percentile(wait, 99))},
            "step_latency_ms": {"p50": float(np.percentile(per_step, 50)), "p99": float(np.percentile(per_step, 99))},
            # a frame of the serving loop = one tick: tick_steps steps of every admitted
            # scene, or with frame_ms set, the steps that fit into it
            "frame_latency_ms": {"p50": float(np.percentile(frame, 50)), "p99": float(np.percentile(frame, 99))},
            # the same, split into ticks right after a membership change (their batch
            # was rebuilt: new tables and a new step graph) and the other ticks; into
            # ticks in which a member's grid regrew, ticks that ran while the worker
            # prepared or read back a request, and the rest; and per million
            # particles stepped, which takes out the batch's size
            "frame_latency_split_ms": self._split(frame),
            "ticks_s": float(frame.sum() / 1e3),
            "wall_s": float(self.wall_s),
            "tick_steps": self.tick_steps,
            "frame_ms": self.frame_ms,
            "steps_per_tick": {"p1": float(np.percentile(self.tick_nsteps, 1)),
                               "p50": float(np.percentile(self.tick_nsteps, 50)),
                               "mean": float(np.mean(self.tick_nsteps))},
            "ticks": len(self.tick_ms),
            "peak_members": self.peak_members,
            "mean_members": float(np.mean(self.tick_members)) if self.tick_members else 0.0,
            "peak_bytes": self.peak_bytes,
            "host_s": dict(self.host_s),
            "graph_updates": self.graph_updates,
            "budget_bytes": self.budget,
            "tile_threads": {"/".join(str(int(v)) for v in k): sh for k, sh in self.shapes.items()},
        }


def poisson_requests(n, rate, seed, steps=200, builder=None):
    """n seeded requests arriving as a Poisson process of `rate` per second."""
    from . import scenes
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        sc = (builder or scenes.serving_request)(rng)
        out.append(Request(rid=i, scene=sc, steps=steps, arrival=t))
    return out
