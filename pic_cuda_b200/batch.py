"""Batched simulations: many independent PIC jobs of uneven size stepped together by one
engine (one set of launches per step, captured in a CUDA graph), in waves that fit an HBM
budget, against the same jobs run one after another with the plain step.

The job mix follows the batched configuration: grid side drawn from {65, 129, 257, 513},
particles per cell per species uniform in [50, 400], Te uniform in [1, 5] eV, argon density
uniform in [1e20, 1e22] m^-3, electrons + Ar+ with the synthetic argon tables, 300 steps.
The cell size is the small configuration's (1 cm / 128), so the domain grows with the grid.
`ppc_scale` shrinks the particle counts for quick runs (the full mix needs ~1e10 particles,
more than one B200 holds, hence the waves).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from . import configs as cf

DX = 0.01 / 128  # cell size of the small configuration (1 cm over 128 cells)
N0 = 1e15        # plasma density behind the macro-particle weight (m^-3)


@dataclass
class JobSpec:
    n: int                    # grid side (nodes)
    ppc: int                  # macro-particles per cell per species
    Te: float                 # electron temperature (eV)
    density: float            # argon density (m^-3)
    steps: int
    seed: int
    Ti: float = 0.03
    deposit: int = L.DEPOSIT_F32
    tol: float = 1e-6

    @property
    def L(self) -> float:
        return (self.n - 1) * DX

    @property
    def n_per_species(self) -> int:
        return max(1, self.ppc * (self.n - 1) ** 2)

    @property
    def particle_steps(self) -> float:
        return 2.0 * self.n_per_species * self.steps


def batched_specs(n_jobs: int = 256, seed: int = 4, ppc_scale: float = 1.0, steps: int = 300,
                  deposit: int = L.DEPOSIT_F32) -> list[JobSpec]:
    """The batched job mix, seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_jobs):
        n = int(rng.choice([65, 129, 257, 513]))
        ppc = int(rng.integers(50, 401))
        out.append(JobSpec(n=n, ppc=max(1, int(round(ppc * ppc_scale))), Te=float(rng.uniform(1.0, 5.0)),
                           density=float(rng.uniform(1e20, 1e22)), steps=steps, seed=int(seed * 100_000 + k),
                           deposit=deposit))
    return out


def job_config(spec: JobSpec, sort_every: int = 10) -> L.JobConfig:
    cap = int(spec.n_per_species * 1.25) + 1024
    w = N0 * spec.L * spec.L / spec.n_per_species
    return cf.make_config(spec.n, spec.L, 1e-11, [(-cf.QE, cf.ME, w, cap), (cf.QE, cf.M_AR, w, cap)],
                          tol=spec.tol, deposit=spec.deposit, sort_every=sort_every, seed=spec.seed,
                          mcc=cf.argon_mcc(spec.density), warm_start=1, omega=cf.MG_OMEGA_1E9)


def bytes_needed(cfg: L.JobConfig) -> int:
    b = L.C.c_int64()
    L.check(L.lib().pic_engine_bytes_needed(L.C.byref(cfg), L.C.byref(b)), "pic_engine_bytes_needed")
    return int(b.value)


def plan_waves(specs: list[JobSpec], budget_bytes: int, max_jobs: int = 4096) -> list[list[int]]:
    """Greedy first-fit of jobs (largest first) into waves whose summed device footprint
    stays within the budget.  A job larger than the budget on its own gets a wave alone."""
    sizes = [bytes_needed(job_config(s)) for s in specs]
    order = sorted(range(len(specs)), key=lambda k: -sizes[k])
    waves: list[list[int]] = []
    used: list[int] = []
    for k in order:
        for w, members in enumerate(waves):
            if used[w] + sizes[k] <= budget_bytes and len(members) < max_jobs:
                members.append(k)
                used[w] += sizes[k]
                break
        else:
            waves.append([k])
            used.append(sizes[k])
    return [sorted(w) for w in waves]


def load_job(job, spec: JobSpec, device=None) -> None:
    cf.load_plasma(job, spec.n_per_species, spec.L, spec.Te, spec.Ti, seed=spec.seed, device=device)


@dataclass
class RunResult:
    seconds: float                      # device time of the stepping (CUDA events)
    wall_seconds: float                 # including job creation and particle loading
    particle_steps: float
    waves: int = 1
    per_job: list = field(default_factory=list)

    @property
    def rate(self) -> float:
        return self.particle_steps / self.seconds if self.seconds > 0 else 0.0


def _timed_steps(engine, steps: int, stream) -> float:
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    engine.step_graph(steps, stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1000.0


def run_batched(specs: list[JobSpec], budget_bytes: int, device: int = 0, tuner=None) -> RunResult:
    """All jobs, wave by wave; every job of a wave steps in the same launches.  `tuner`
    (an autotune.Tuner) may pick engine options from the wave's first steps, which count
    towards the jobs' steps."""
    import torch
    from .engine import Engine
    dev = torch.device("cuda", device)
    stream = torch.cuda.Stream(device=dev)
    waves = plan_waves(specs, budget_bytes)
    secs = wall = ps = 0.0
    per_job = []
    for members in waves:
        t0 = time.perf_counter()
        eng = Engine(device)
        jobs = []
        for k in members:
            j = eng.add_job(job_config(specs[k]))
            load_job(j, specs[k], device=dev)
            jobs.append(j)
        steps = specs[members[0]].steps
        assert all(specs[k].steps == steps for k in members), "a wave steps its jobs together"
        done = 0
        if tuner is not None:
            done = tuner.tune(eng, jobs, stream, max_steps=steps)
        secs += _timed_steps(eng, steps - done, stream)
        # particle-steps of the timed steps (the loaded populations; tuning steps excluded)
        ps += sum(specs[k].particle_steps for k in members) * (steps - done) / steps
        for k, j in zip(members, jobs):
            per_job.append((k, j.diagnostics()))
            j.destroy()
        eng.close()
        wall += time.perf_counter() - t0
    return RunResult(seconds=secs, wall_seconds=wall, particle_steps=ps, waves=len(waves), per_job=per_job)


def run_sequential(specs: list[JobSpec], device: int = 0) -> RunResult:
    """The same jobs one after another, each alone in an engine, with the plain step."""
    import torch
    from .engine import Engine
    dev = torch.device("cuda", device)
    stream = torch.cuda.Stream(device=dev)
    secs = wall = ps = 0.0
    per_job = []
    for k, s in enumerate(specs):
        t0 = time.perf_counter()
        eng = Engine(device)
        j = eng.add_job(job_config(s))
        load_job(j, s, device=dev)
        secs_j = _timed_steps(eng, s.steps, stream)
        secs += secs_j
        ps += s.particle_steps
        per_job.append((k, secs_j))
        j.destroy()
        eng.close()
        wall += time.perf_counter() - t0
    return RunResult(seconds=secs, wall_seconds=wall, particle_steps=ps, waves=len(specs), per_job=per_job)
