"""Continuous-batching run server.

A request asks for `steps` steps of one active KA system (N particles, T, f0,
tau_p) from a seeded lattice, with the overlap Q(t), chi4(t), MSD and Fs
accumulated in place on the log-time schedule of the run (no trajectory is
written).  Requests arrive over time; the server admits a queued request as
soon as its device footprint fits the memory budget and an active slot is
free, keeps its whole state on the device in its own engine and CUDA stream,
and advances every active run in chunks of CUDA-graph launches, so the work of
runs admitted at different times overlaps on the GPU.  When a run ends its
observables and energies are read back, its memory is released and the next
queued request is admitted.  Latency is arrival -> results.

Runs are independent and deterministic, so each result is bit-identical
whether the run was served alone or in a mix (tested).
"""
from __future__ import annotations

import dataclasses
import math
import time

import numpy as np

from .engine import Engine, default_params, footprint, qvectors, release_retired
from .init import lattice_state


@dataclasses.dataclass
class RunRequest:
    rid: int
    n: int
    steps: int
    T: float = 0.45
    f0: float = 1.0
    tau_p_steps: int = 200
    seed: int = 0
    arrival: float = 0.0     # seconds after the start of serving
    precision: int = 1       # ACG_PREC_FP32 pair forces
    num_origins: int = 20
    max_live_origins: int = 16
    q: float = 7.25          # |q| of the Fs(q,t) shell


@dataclasses.dataclass
class RunResult:
    rid: int
    n: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    observables: tuple       # (offsets, per-bin sums) of acg_obs_sums
    pe: float
    ke: float

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_params(req: RunRequest):
    return default_params(req.n, T=req.T, f0=req.f0, tau_p_steps=req.tau_p_steps, precision=req.precision,
                          seed=1000003 * req.seed + 17, list_mode=1, rebuild_factor=4.0)


def request_footprint(req: RunRequest) -> int:
    return footprint([request_params(req)]) + req.max_live_origins * req.n * 24 + (4 << 20)


_QCACHE: dict = {}


def _qvectors_cached(L: float, q: float, count: int):
    key = (L, q, count)
    if key not in _QCACHE:
        _QCACHE[key] = qvectors(L, q, count)
    return _QCACHE[key]


def start_run(req: RunRequest, device: int = 0, setup_priority: int = 0) -> Engine:
    """A request's engine, loaded and primed.  With `setup_priority` > 0 the
    set-up work (upload, first lists and forces, observable buffers) runs at
    that stream priority, so it does not wait behind the queued steps of the
    runs already on the device (the set-up reads results back, which would
    otherwise block the host for as long as that queue takes)."""
    e = Engine(request_params(req), device=device)
    if req.n < 60000:
        # a small system's force blocks hold few particles each: more threads
        # per particle shorten each thread's share of the pair loop (measured
        # step latency: N = 4505 44.8 us at 8 threads per particle against
        # 47.4 at 4; N = 11154 best at 4)
        e.set_group_tpp(4)
        if req.n < 8000:
            e.set_launch(8, 128)
    if setup_priority > 0:
        e.set_priority(setup_priority)
    st = lattice_state(req.n, req.T, seed=req.seed)
    e.set_state(0, st)
    rng = np.random.default_rng(req.seed)
    q = e.thermo(0)["q"]
    e.set_nhc(0, np.zeros(3), np.sqrt(req.T * q) * rng.standard_normal(3))
    e.obs_configure(0, req.steps, min(req.num_origins, max(1, req.steps // 2)), 1.4, 0, 0.3,
                    _qvectors_cached(st.L, req.q, 24), req.max_live_origins)
    return e


def finish_run(e: Engine, req: RunRequest, arrival, admitted, finished) -> RunResult:
    th = e.thermo(0)
    return RunResult(req.rid, req.n, req.steps, arrival, admitted, finished, e.obs_sums(0), th["pe"], th["ke"])


class Server:
    """Admit-as-memory-frees scheduler over per-run engines and streams.

    Each active run keeps `depth` chunks of steps queued on its stream (a CUDA
    event marks the end of each), so the GPU has work from every run while the
    host admits new requests or builds their graphs."""

    def __init__(self, device=0, hbm_budget=None, max_active=16, chunk_work=2.0e7, depth=2, priority="time",
                 max_big=None, big_n=20000):
        self.device = device
        if hbm_budget is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget = int(0.8 * free)
        self.budget = int(hbm_budget)
        self.max_active = max_active
        self.chunk_work = chunk_work
        self.depth = max(1, int(depth))
        # stream priority of a run: "time" = the runs expected to take longest
        # first (a small system with many steps is bound by per-step latency
        # and sets the end of the stream; queued behind the kernels of other
        # runs it ends later still), "size" = larger systems first, "none"
        self.priority = priority
        # at most max_big runs of more than big_n particles active at once (None:
        # no limit); a big request waits while smaller ones behind it are admitted
        self.max_big = max_big
        self.big_n = big_n

    def _level(self, req) -> int:
        if self.priority == "size":
            return int(np.clip(2.0 * (math.log10(req.n) - 3.0), 0, 4))
        if self.priority == "time":
            # expected device time alone: a step costs at least ~45 us (kernel
            # latency) and about 1 ns per particle beyond that
            est = req.steps * max(45e-6, 1.0e-9 * req.n)
            return int(np.clip(np.floor(np.log2(max(est, 1.0))), 0, 4))
        return 0

    def _chunk(self, n, left):
        # about chunk_work particle-steps, and no more than ~20 ms of device
        # time for small systems, whose steps cost ~50 us whatever their size
        k = min(self.chunk_work / max(n, 1), 0.02 / 5e-5)
        k = int(max(32, min(8192, round(k / 32) * 32)))
        return min(k, left)

    def _feed(self, run):
        """Queue chunks until `depth` are in flight or the run is fully queued."""
        import torch
        while len(run["inflight"]) < self.depth and run["left"] > 0:
            k = self._chunk(run["req"].n, run["left"])
            run["engine"].step(k)
            ev = torch.cuda.Event()
            ev.record(run["stream"])
            run["inflight"].append(ev)
            run["left"] -= k

    def run(self, requests, clock=time.perf_counter):
        import collections

        import torch
        pending = sorted(requests, key=lambda r: r.arrival)
        queue, active, results = [], {}, []
        used = 0
        t0 = clock()
        while pending or queue or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.pop(0))
            # admission in arrival order while memory and slots allow (a big
            # request over the max_big limit waits; the next in line goes first)
            while queue and len(active) < self.max_active:
                k = next_admissible(queue, [a["req"].n for a in active.values()], self.max_big, self.big_n)
                if k < 0:
                    break
                fp = request_footprint(queue[k])
                if used + fp > self.budget and active:
                    break
                req = queue.pop(k)
                e = start_run(req, self.device, setup_priority=5)
                # stepping priority by the policy (`priority`)
                e.set_priority(self._level(req))
                used += fp
                run = {"engine": e, "req": req, "left": req.steps, "adm": clock() - t0, "fp": fp,
                       "stream": torch.cuda.ExternalStream(e.stream, device=torch.device("cuda", self.device)),
                       "inflight": collections.deque()}
                # graphs built now (this can wait for the work queued on the
                # device, which the time-bounded chunks keep short)
                e.prepare()
                self._feed(run)
                active[req.rid] = run
            progressed = False
            for rid in list(active):
                run = active[rid]
                while run["inflight"] and run["inflight"][0].query():
                    run["inflight"].popleft()
                    progressed = True
                if run["left"] == 0 and not run["inflight"]:
                    e, req = run["engine"], run["req"]
                    e.sync()
                    results.append(finish_run(e, req, req.arrival, run["adm"], clock() - t0))
                    e.close()
                    used -= run["fp"]
                    del active[rid]
                else:
                    self._feed(run)
            if not active:
                release_retired()  # nothing in flight: destroying graphs stalls nothing
            if not progressed:
                nxt = pending[0].arrival - (clock() - t0) if (pending and not queue and not active) else 2e-4
                time.sleep(max(5e-5, min(nxt, 2e-3)))
        release_retired()
        return sorted(results, key=lambda r: r.rid)


def run_serial(requests, device=0, precision=0, clock=time.perf_counter, sample_steps=None):
    """The same requests one after another, each alone on the GPU (the
    serial baseline); returns (results, wall seconds).  With sample_steps,
    each request runs only its first sample_steps steps and its stepping time
    is scaled to its full length (set-up time counted as measured): a bounded
    estimate of the serial wall time."""
    out = []
    wall = 0.0
    for req in requests:
        r = dataclasses.replace(req, precision=precision)
        t0 = clock()
        e = start_run(r, device)
        e.sync()
        t1 = clock()
        k = r.steps if sample_steps is None else min(r.steps, int(sample_steps))
        e.step(k)
        e.sync()
        t2 = clock()
        wall += (t1 - t0) + (t2 - t1) * (r.steps / k)
        out.append(finish_run(e, r, t0, t1, t2))
        e.close()
    return out, wall


def poisson_requests(count, rate=20.0, n_range=(1000, 256000), step_range=(10000, 1000000), scale=1.0,
                     seed=0, precision=1):
    """Poisson arrivals at `rate` per second; N and steps log-uniform; T, f0,
    tau_p drawn from the batched workload's sets.  `scale` multiplies the step
    counts (a bounded sample of the workload)."""
    from .batch import F0_SET, T_SET, TAU_SET
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        n = int(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1]))))
        steps = int(math.exp(rng.uniform(math.log(step_range[0]), math.log(step_range[1]))) * scale)
        reqs.append(RunRequest(i, n, max(64, steps), float(rng.choice(T_SET)), float(rng.choice(F0_SET)),
                               int(rng.choice(TAU_SET)), seed=10000 * seed + i, arrival=t, precision=precision))
    return reqs


def next_admissible(queue, active_n, max_big=None, big_n=20000) -> int:
    """Index in `queue` (arrival order) of the next request to admit, or -1:
    the first one, except that a request of more than `big_n` particles
    waits while `max_big` such runs are active (sizes `active_n`), and the
    first smaller request behind it goes instead."""
    if not queue:
        return -1
    if max_big is None:
        return 0
    nbig = sum(1 for n in active_n if n > big_n)
    for k, req in enumerate(queue):
        if req.n <= big_n or nbig < max_big:
            return k
    return -1


def latency_stats(results):
    lat = np.array([r.latency for r in results])
    work = sum(r.n * r.steps for r in results)
    span = max(r.finished for r in results) - min(r.arrival for r in results)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "particle_steps_per_s": work / span, "requests": len(results), "span_s": span}
