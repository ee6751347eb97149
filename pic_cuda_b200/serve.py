"""Serving: a request loop that admits simulation jobs of different sizes as HBM budget and
job slots free up, keeps their particle and grid state resident on the device, steps every
admitted job together (continuous batching: a request that arrives while others run joins
at the next step boundary), and reports time-to-completion percentiles beside aggregate
particle-steps/s.  The comparison is the same request stream served one job at a time in
arrival order with the plain step.

The request mix follows the served configuration: grid side from {129, 257, 513, 1025},
particles per cell per species uniform in [20, 200], steps uniform in [200, 2000], argon
density log-uniform in [1e20, 1e22] m^-3, Poisson arrivals at a rate that saturates the GPU.
`ppc_scale` and `steps_scale` shrink the work for quick runs.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .batch import JobSpec, bytes_needed, job_config, load_job


@dataclass
class Request:
    arrival: float          # seconds after the stream starts
    spec: JobSpec
    index: int = 0


# Aggregate particle-steps/s of one B200 on the batched mix (measured: 2.1e10), rounded up: the
# arrival rate used when no capacity measured in the run is given (see measure_capacity).
B200_CAPACITY = 2.5e10


def measure_capacity(specs: list[JobSpec], device: int = 0, budget_bytes: int = 40 * 10**9, steps: int = 20,
                     warmup: int = 3) -> float:
    """Particle-steps/s this GPU sustains on a sample of the request mix: the sample's jobs
    (as many as fit `budget_bytes`) stepped together, `steps` steps timed with CUDA events
    after `warmup` untimed ones.  The served bench sets its arrival rate from this figure."""
    import torch
    from .engine import Engine
    eng = Engine(device)
    jobs, used, work = [], 0, 0.0
    try:
        for sp in specs:
            need = bytes_needed(job_config(sp))
            if jobs and used + need > budget_bytes:
                continue
            job = eng.add_job(job_config(sp))
            load_job(job, sp, device=torch.device("cuda", device))
            jobs.append(job)
            used += need
            work += 2.0 * sp.n_per_species
        stream = torch.cuda.Stream(device=device)
        eng.step_graph(warmup, stream=stream.cuda_stream)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.step_graph(steps, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(device)
        return work * steps / (e0.elapsed_time(e1) / 1000.0)
    finally:
        for job in jobs:
            job.destroy()
        eng.close()


def served_requests(n_requests: int = 2000, seed: int = 5, ppc_scale: float = 1.0, steps_scale: float = 1.0,
                    rate: float | None = None, saturation: float = 1.5, capacity: float = B200_CAPACITY,
                    deposit: int = L.DEPOSIT_F32) -> list[Request]:
    """Seeded request stream.  Without an explicit rate (requests/s), the Poisson rate is
    `saturation` times what a GPU of `capacity` particle-steps/s can serve on average."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n_requests):
        n = int(rng.choice([129, 257, 513, 1025]))
        ppc = max(1, int(round(int(rng.integers(20, 201)) * ppc_scale)))
        steps = max(1, int(round(int(rng.integers(200, 2001)) * steps_scale)))
        dens = float(10 ** rng.uniform(20.0, 22.0))
        specs.append(JobSpec(n=n, ppc=ppc, Te=float(rng.uniform(1.0, 5.0)), density=dens, steps=steps,
                             seed=int(seed * 1_000_000 + k), deposit=deposit))
    if rate is None:
        mean_work = float(np.mean([s.particle_steps for s in specs]))
        rate = saturation * capacity / mean_work
    gaps = rng.exponential(1.0 / rate, n_requests)
    t = np.cumsum(gaps) - gaps[0]
    return [Request(float(t[k]), specs[k], k) for k in range(n_requests)]


@dataclass
class Completion:
    index: int
    arrival: float
    admitted: float
    finished: float
    diagnostics: dict
    result: object = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def percentiles(latencies) -> dict:
    a = np.asarray(latencies, dtype=np.float64)
    if a.size == 0:
        return {"p50": None, "p99": None, "mean": None}
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)), "mean": float(a.mean())}


@dataclass
class Server:
    """One engine; FIFO admission under `budget_bytes` and `max_jobs`; all admitted jobs step
    together in quanta of at most `quantum` steps (never past any job's remaining steps)."""
    engine: object
    budget_bytes: int
    quantum: int = 20
    max_jobs: int = 4096
    device: object = None
    keep_results: bool = False
    # Stream-ordered steps by default: the job set changes every quantum or two, and a CUDA
    # graph would be rebuilt each time.  Measured on B200 (64 requests, ppc x 0.05, steps x 0.1):
    # graphs on every quantum 7.5e9 particle-steps/s, graphs once the set was stable for a
    # quantum 7.6e9, stream-ordered always 11.2e9.  With use_graph the stable quanta use graphs.
    use_graph: bool = False
    # map the HBM budget into the engine's job pool before the first request (server start-up),
    # so that admissions take memory that is already mapped
    reserve: bool = True
    clock: object = time.perf_counter
    sleep: object = time.sleep
    log: list = field(default_factory=list)
    # one entry per quantum: (start s, steps, active jobs, job set changed, seconds)
    quanta: list = field(default_factory=list)

    def _admit(self, req: Request, now: float):
        cfg = job_config(req.spec)
        job = self.engine.add_job(cfg)
        load_job(job, req.spec, device=self.device)
        return job

    def _result(self, job):
        if not self.keep_results:
            return None
        return {"phi": job.get_grid(L.GRID_PHI), "species": [job.export_species(s) for s in (0, 1)]}

    def run(self, requests: list[Request]) -> dict:
        if self.reserve:
            self.engine.reserve(self.budget_bytes)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        active = []   # [req, job, steps_left, bytes, admitted]
        used = 0
        done: list[Completion] = []
        t0 = self.clock()
        particle_steps = 0.0
        spent = {"admit": 0.0, "step": 0.0, "complete": 0.0, "idle": 0.0}
        changed = True   # the job set differs from the last quantum's
        while pending or active:
            now = self.clock() - t0
            while pending and pending[0].arrival <= now and len(active) < self.max_jobs:
                need = bytes_needed(job_config(pending[0].spec))
                if active and used + need > self.budget_bytes:
                    break  # head of line waits for memory
                req = pending.popleft()
                ta = self.clock()
                job = self._admit(req, now)
                spent["admit"] += self.clock() - ta
                used += need
                changed = True
                active.append([req, job, req.spec.steps, need, self.clock() - t0])
                self.log.append(("admit", req.index, self.clock() - t0, len(active), used))
            if not active:
                ti = self.clock()
                self.sleep(max(0.0, min(0.01, pending[0].arrival - now)))
                spent["idle"] += self.clock() - ti
                continue
            k = min(self.quantum, min(a[2] for a in active))
            ts = self.clock()
            (self.engine.step_graph if self.use_graph and not changed else self.engine.step)(k)
            self.engine.sync()
            self.quanta.append((ts - t0, k, len(active), changed, self.clock() - ts))
            changed = False
            spent["step"] += self.clock() - ts
            particle_steps += k * sum(2.0 * a[0].spec.n_per_species for a in active)
            tc = self.clock()
            still = []
            for a in active:
                a[2] -= k
                if a[2] == 0:
                    req, job = a[0], a[1]
                    diag = job.diagnostics()
                    res = self._result(job)
                    job.destroy()
                    used -= a[3]
                    changed = True
                    done.append(Completion(req.index, req.arrival, a[4], self.clock() - t0, diag, res))
                    self.log.append(("done", req.index, self.clock() - t0, len(active) - 1, used))
                else:
                    still.append(a)
            active = still
            spent["complete"] += self.clock() - tc
        makespan = self.clock() - t0
        lat = [c.latency for c in done]
        return {"completions": sorted(done, key=lambda c: c.index), "makespan": makespan,
                "particle_steps": particle_steps, "rate": particle_steps / makespan if makespan > 0 else 0.0,
                "seconds_in": spent, **percentiles(lat)}


def fifo_replay(requests: list[Request], durations: list[float]) -> dict:
    """Completion times of the request stream served one job at a time in arrival order,
    given each job's measured run time alone."""
    order = sorted(range(len(requests)), key=lambda k: requests[k].arrival)
    t = 0.0
    lat = [0.0] * len(requests)
    for k in order:
        t = max(t, requests[k].arrival) + durations[k]
        lat[k] = t - requests[k].arrival
    makespan = t - min(r.arrival for r in requests) if requests else 0.0
    ps = sum(r.spec.particle_steps for r in requests)
    return {"makespan": makespan, "particle_steps": ps, "rate": ps / makespan if makespan > 0 else 0.0,
            "latencies": lat, **percentiles(lat)}


def run_alone(spec: JobSpec, device: int = 0, keep_result: bool = False, clock=time.perf_counter):
    """One job by itself in its own engine, from creation to the read-back of its result."""
    import torch
    from .engine import Engine
    t0 = clock()
    eng = Engine(device)
    job = eng.add_job(job_config(spec))
    load_job(job, spec, device=torch.device("cuda", device))
    eng.step_graph(spec.steps)
    eng.sync()
    diag = job.diagnostics()
    res = {"phi": job.get_grid(L.GRID_PHI), "species": [job.export_species(s) for s in (0, 1)]} if keep_result \
        else None
    job.destroy()
    eng.close()
    return clock() - t0, diag, res
