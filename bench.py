#!/usr/bin/env python
"""Benchmark of the full 2D electrostatic PIC step (particle-steps/s).

Workload (default, `--workload large`): 4097^2 nodes over 20 cm^2, 1e8 electrons + 1e8 Ar+
(FP32 state, uniform positions, Maxwellian Te 2 eV, Ti 0.03 eV), argon 3.2e21 m^-3
null-collision MCC with 512-point synthetic tables, FP32 V-cycles inside FP64 defect
correction to 1e-9 relative residual, absorbing walls, counting sort every 10 steps; the
FP32 deposit gives `value`, the int64 fixed-point deposit is timed beside it (`int64`).
Synthetic seeded data; the particle state (~5.6 GB) is larger than L2, so no flush is needed
between steps.  `--workload mcc_mixed` is the 1025^2, 2e7-particle configuration.

  value     device-timed throughput (CUDA events on the launching stream, inputs resident)
  e2e       one complete job through the public C ABI with host buffers: load from pinned
            host memory, the workload's own step count with a diagnostics read-back after
            every step, export to pinned host memory
  roofline  the fused particle pass (dominant kernel): algorithmic bytes / event time
  cpu_baseline  the FP64 CPU oracle (OpenMP) on a bounded sample of the same workload
  reference_particle_kernels  the reference's own four FP64 particle kernels (built from its
            sources) on the same particle count and grid on the same GPU, against the mover

`--impl reference` times the reference path's CPU implementation: the reference has none
(its only implementation is CUDA), so the FP64 oracle port of its step runs on all host
threads.  Multi-GPU (torchrun): one independent replica per rank ("replicas only"), no
collective on the data path; the timed region is bracketed by barriers, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s full PIC step at 1 B200; batched/served vs plain; p50/p99"
UNIT = "particle-steps/s"
BYTES_PER_PARTICLE = {"collisionless": 32, "mcc": 44}  # algorithmic bytes per particle-step


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="large",
                    choices=["plain_small", "mcc_mixed", "large", "batched", "served", "embedded"])
    ap.add_argument("--jobs", type=int, default=None, help="batched: jobs; served: requests")
    ap.add_argument("--ppc-scale", type=float, default=None, help="batched/served: particles-per-cell factor")
    ap.add_argument("--steps-scale", type=float, default=None, help="served: request step-count factor")
    ap.add_argument("--budget-gb", type=float, default=None, help="batched/served: HBM budget")
    ap.add_argument("--n-per-species", type=int, default=None)
    ap.add_argument("--deposit", choices=["f32", "i64"], default="f32")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=None,
                    help="oracle steps timed for the CPU baseline (default 1 on large, else 3)")
    ap.add_argument("--no-ref-cuda", action="store_true")
    ap.add_argument("--no-int64", action="store_true", help="large: skip the int64-deposit timing")
    ap.add_argument("--step-path", choices=["graph", "stream"], default="graph",
                    help="timed steps as CUDA-graph launches (default) or stream-ordered launches")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload(args):
    from pic_cuda_b200 import _lib as L
    from pic_cuda_b200 import configs as cf
    w = cf.WORKLOADS[args.workload]
    n = args.n_per_species or w["n"]
    dep = L.DEPOSIT_I64 if args.deposit == "i64" else L.DEPOSIT_F32
    cfg = w["builder"](n_per_species=n, deposit=dep) if args.workload != "plain_small" else cf.plasma(
        129, 0.01, n, tol=1e-6, deposit=dep, warm_start=1)
    steps_job = {"plain_small": 100, "mcc_mixed": 500, "large": 200}[args.workload]
    return cfg, n, w["Te"], w["Ti"], cfg.Lx, steps_job


def cpu_steps(args):
    if args.cpu_steps is not None:
        return max(1, args.cpu_steps)
    return 1 if args.workload == "large" else 3


def cpu_baseline(args, cfg, n, Te, Ti, Ld, steps=None):
    """FP64 oracle step on the host cores, bounded sample: `steps` full steps of the whole
    workload (every particle, the full grid) after one untimed step."""
    import gc
    from oracle import oracle as orc
    from pic_cuda_b200 import configs as cf
    steps = steps or cpu_steps(args)
    sim = orc.Sim(cfg)
    for k, (T, m, seed) in enumerate(((Te, cf.ME, 1234), (Ti, cf.M_AR, 1235))):
        st = cf.maxwellian_state(n, Ld, T, m, seed)
        sim.load(k, *st)
        del st
        gc.collect()
    sim.step(1)  # warm-up (first-touch allocation of the multigrid hierarchy)
    t0 = time.perf_counter()
    sim.step(steps)
    dt = time.perf_counter() - t0
    np_ = sum(len(sim.export(k)["x"]) for k in (0, 1))
    return {"value": np_ * steps / dt, "unit": UNIT, "cores": orc.num_threads(), "kind": "port",
            "sample": f"{steps} full FP64 oracle step(s) of {args.workload} ({2 * n} particles, "
                      f"{cfg.nx}x{cfg.ny}) after 1 untimed step", "seconds": dt, "steps": steps}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg, n, Te, Ti, Ld, _ = workload(args)
    steps = max(1, min(args.steps, args.cpu_steps or (2 if args.workload == "large" else 3)))
    cb = cpu_baseline(args, cfg, n, Te, Ti, Ld, steps=steps)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": 1, "ms_per_step": 1000.0 * cb["seconds"] / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": args.workload, "grid": f"{cfg.nx}x{cfg.ny}", "particles": 2 * n,
                       "note": "the reference has no CPU implementation; its step is restated in FP64 "
                               "(oracle/pic_oracle.cpp) and run with OpenMP on every host thread"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# The reference's demo species and walls: Particles2D's default species (q=0.1, m=1,
# particles.cu:146-149), the species main.cu:188 adds (m=1, q=-1), the domain box plus the
# two interior walls of main.cu:193-194; main.cu's solver settings (main.cu:113,
# Multigrid.cu:573) and time step (main.cu:150).
REF_Q, REF_M = [0.1, -1.0], [1.0, 1.0]
REF_WALLS = [[0, 0, 1, 0], [1, 0, 1, 1], [1, 1, 0, 1], [0, 1, 0, 0], [0.25, 0.25, 0.25, 0.75],
             [0.75, 0.25, 0.75, 0.75]]


def reference_cuda(local, n_per_species=100_000, grid=129, steps=30, warmup=3):
    """The reference's own CUDA step (its kernels built from its sources into oracle/_ref,
    re-sequenced headless as main.cu:60-135, CUDA events around the step loop) and this
    engine on the same seeded state, grid, species, walls and solver settings, in the
    reference's units.  The reference's multigrid cannot run at 1025^2 (its cooperative
    launch fails there), so the comparison is made on the 129^2 configuration."""
    import numpy as np
    import torch
    from oracle import refh
    from pic_cuda_b200 import _lib as L
    from pic_cuda_b200 import configs as cf
    from pic_cuda_b200.engine import Engine
    if not refh.LIB.exists():
        return {"unavailable": "oracle/_ref/libpicref.so not built"}
    rng = np.random.default_rng(1234)
    N = 2 * n_per_species
    x, y = rng.uniform(0.2, 0.8, N), rng.uniform(0.2, 0.8, N)  # main.cu:20-21
    vx, vy = rng.uniform(-0.01, 0.01, N), rng.uniform(-0.01, 0.01, N)
    t = np.repeat(np.arange(2, dtype=np.int32), n_per_species)
    dt = 0.01
    refh.steps(warmup, x, y, vx, vy, t, REF_Q, REF_M, grid, grid, 1.0, 1.0, REF_WALLS, dt)
    ref = refh.steps(steps, x, y, vx, vy, t, REF_Q, REF_M, grid, grid, 1.0, 1.0, REF_WALLS, dt)
    cfg = cf.make_config(grid, 1.0, dt, [(REF_Q[0], REF_M[0], 1.0, N), (REF_Q[1], REF_M[1], 1.0, N)],
                         units=L.UNITS_REF, walls=L.WALLS_SEGMENTS, wall_segments=REF_WALLS, levels=5, omega=1.25,
                         nu_pre=3, nu_post=3, nu_coarse=20, tol=1e-5)
    eng = Engine(local)
    job = eng.add_job(cfg)
    for s in (0, 1):
        sel = t == s
        job.load_species(s, x[sel], y[sel], vx[sel], vy[sel])
    stream = torch.cuda.Stream()
    eng.step_graph(warmup, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    eng.step_graph(steps, stream=stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    ours = ev0.elapsed_time(ev1) / steps
    job.destroy()
    eng.close()
    return {"config": f"{grid}x{grid}, {N} particles (2 species), reference units, main.cu demo walls, "
                      f"5-level V-cycles omega 1.25 3/3/20 to 1e-5, dt {dt}, {steps} steps, no MCC",
            "reference_ms_per_step": ref["ms_per_step"], "ours_ms_per_step": ours,
            "reference_particle_steps_per_s": N / (ref["ms_per_step"] / 1000.0),
            "ours_particle_steps_per_s": N / (ours / 1000.0),
            "speedup": ref["ms_per_step"] / ours,
            "timing": "CUDA events around each implementation's step loop on the same B200"}


def timed_steps(args, cfg, n, Te, Ti, Ld, local, rank, dist, clocks=None):
    """One job of the workload on a fresh engine: W untimed steps, then K steps timed with CUDA
    events on the launching stream (barriers and synchronisation on both sides), then a
    stream-ordered region with CUDA events around every particle pass and phase."""
    import torch
    from pic_cuda_b200 import configs as cf
    from pic_cuda_b200.engine import Engine
    dev = torch.device("cuda", local)
    eng = Engine(local)
    job = eng.add_job(cfg)
    cf.load_plasma(job, n, Ld, Te, Ti, seed=1234 + 17 * rank, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    run_steps = eng.step_graph if args.step_path == "graph" else eng.step
    run_steps(args.warmup, stream=sptr)
    torch.cuda.synchronize(dev)
    n0 = sum(job.diagnostics()["count"])
    eng.stats(reset=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # timed region: whole steps as CUDA graph launches (no host synchronisation inside)
    with (clocks if clocks is not None else ClockSampler(local)) as clk:
        ev0.record(stream)
        run_steps(args.steps, stream=sptr)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    st = eng.stats(reset=True)
    d1 = job.diagnostics()
    n1 = sum(d1["count"])
    # second region of the same workload, stream-ordered with CUDA events around every
    # particle pass and phase (the per-kernel figures of the roofline)
    prof_steps = min(args.steps, 50)
    eng.profile(True)
    eng.step(prof_steps, stream=sptr)
    torch.cuda.synchronize(dev)
    pst = eng.stats(reset=True)
    eng.profile(False)
    job.destroy()
    eng.close()
    return {"ms": ms, "stats": st, "prof": pst, "prof_steps": prof_steps, "particles": 0.5 * (n0 + n1),
            "relres": d1["relres"], "clocks": clk}


def reference_particle_kernels(cfg, particles, mover_ms, Te, Ti, iters=5):
    """The reference's own FP64 particle kernels of a step (update_coordinates,
    detect_intersections with its memsets, updateDensity with the rho memset,
    updateParticleVelocities; kernels.cu:8-131, collisions.cu:7-54, launched as
    main.cu:64-127 does) on the same particle count and grid, on this GPU, against the fused
    particle pass.  The reference's multigrid cannot run at these sizes (its cooperative
    launch fails above 513^2), so only the particle work is compared."""
    import math
    from oracle import refh
    from pic_cuda_b200 import configs as cf
    if not refh.available():
        return {"unavailable": "oracle/_ref/libpicref.so not built or no device"}
    n = int(particles)
    vmax = (math.sqrt(3.0 * Te * cf.QE / cf.ME), math.sqrt(3.0 * Ti * cf.QE / cf.M_AR))
    q = [cfg.species[0].charge * cfg.species[0].weight, cfg.species[1].charge * cfg.species[1].weight]
    m = [cfg.species[0].mass * cfg.species[0].weight, cfg.species[1].mass * cfg.species[1].weight]
    ms = refh.particle_kernels_timed(n, cfg.nx, cfg.ny, cfg.Lx, cfg.Ly, cfg.dt, q, m, vmax, iters=iters)
    total = sum(ms)
    return {"particles": n, "grid": f"{cfg.nx}x{cfg.ny}",
            "ms": {"update_coordinates": ms[0], "detect_intersections": ms[1], "updateDensity": ms[2],
                   "updateParticleVelocities": ms[3]},
            "ms_per_pass": total, "ours_mover_ms": mover_ms, "speedup_per_pass": total / mover_ms,
            "note": "reference FP64 AoS state, unsorted (it never sorts), box walls, no collisions, CUDA events per "
                    "kernel over %d launches; ours: the fused pass including the null-collision MCC" % iters}


def run_ours(args):
    import torch
    from pic_cuda_b200 import _lib as L
    from pic_cuda_b200 import shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    cfg, n, Te, Ti, Ld, steps_job = workload(args)
    r = timed_steps(args, cfg, n, Te, Ti, Ld, local, rank, dist)
    ms, st, pst, prof_steps, particles = r["ms"], r["stats"], r["prof"], r["prof_steps"], r["particles"]
    ms_max, particles_all = shard.reduce_timing(ms, particles, dist, dev)
    value = particles_all * args.steps / (ms_max / 1000.0)

    # the int64 fixed-point deposit on the same workload (every rank takes the same steps)
    int64 = None
    if args.workload == "large" and args.deposit == "f32" and not args.no_int64:
        a64 = argparse.Namespace(**{**vars(args), "deposit": "i64"})
        cfg64 = workload(a64)[0]
        r64 = timed_steps(a64, cfg64, n, Te, Ti, Ld, local, rank, dist)
        ms64, p64 = shard.reduce_timing(r64["ms"], r64["particles"], dist, dev)
        int64 = {"ms_per_step": ms64 / args.steps, "value": p64 * args.steps / (ms64 / 1000.0), "unit": UNIT,
                 "vcycles_per_step": r64["stats"]["vcycles"] / max(r64["stats"]["steps"], 1),
                 "mover_ms": r64["prof"]["mover_ms"] / max(r64["prof"]["mover_launches"], 1),
                 "clocks": r64["clocks"].summary()}

    # roofline of the fused particle pass
    peak, peak_kind = peaks()
    mcc_on = cfg.mcc_mode != 0
    bpp = BYTES_PER_PARTICLE["mcc" if mcc_on else "collisionless"]
    mover_ms = pst["mover_ms"] / max(pst["mover_launches"], 1)
    achieved = particles * bpp / (mover_ms / 1000.0) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "mover_traffic.json"
    if tf.exists():
        t = json.loads(tf.read_text()).get(args.workload)
        if t and "bytes_per_particle" in t:
            traffic = t["bytes_per_particle"] * particles
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "mover_kernel (fused kick/MCC/drift/walls/deposit)",
                "bytes_per_particle": bpp, "mover_ms": mover_ms, "peak_source": f"{peak_kind} hbm_gbs",
                "mover_share_of_step": mover_ms / (ms / args.steps) if ms > 0 else None,
                "timing": f"CUDA events around each mover launch over {prof_steps} stream-ordered steps"}

    # the whole step against HBM (per GPU): B = Np Bp + Nnodes (16 + k_vc Bvc) + k_dc Nnodes 40,
    # Bvc = (4/3)(12 (nu_pre + nu_post) + 16) + 8 bytes per node and V-cycle, one FP64 defect
    # correction update per V-cycle (k_dc = k_vc), k_vc measured over the timed steps
    nodes = cfg.nx * cfg.ny
    kvc = st["vcycles"] / max(st["steps"], 1)
    bvc = (4.0 / 3.0) * (12 * (cfg.nu_pre + cfg.nu_post) + 16) + 8
    step_bytes = particles * bpp + nodes * (16 + kvc * bvc) + kvc * nodes * 40
    step_ach = step_bytes / (ms / args.steps / 1000.0) / 1e9
    step_roofline = {"bound": "hbm", "achieved": step_ach, "peak": peak, "unit": "GB/s", "frac": step_ach / peak,
                     "bytes_per_step": step_bytes, "vcycles_per_step": kvc,
                     "formula": "Np*Bp + Nnodes*(16 + k_vc*Bvc) + k_vc*Nnodes*40"}

    # end to end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, cfg, n, Te, Ti, Ld, steps_job, local, rank)
        if dist:
            # the whole job over all ranks: every rank's particle-steps over the slowest rank's time
            sec, work = shard.reduce_timing(e2e["seconds"], e2e["value"] * e2e["seconds"], dist, dev)
            e2e.update(value=work / sec, seconds=sec, ranks=world,
                       h2d_bytes_per_step=e2e["h2d_bytes_per_step"] * world,
                       d2h_bytes_per_step=e2e["d2h_bytes_per_step"] * world)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "grid": f"{cfg.nx}x{cfg.ny}", "particles": 2 * n,
                   "mcc": mcc_on, "deposit": args.deposit, "tol": cfg.tol, "sort_every": cfg.sort_every,
                   "precision": "FP32 particles and V-cycles, FP64 defect correction and diagnostics",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "state larger than L2 (no flush needed)",
                   "vcycles_per_step": kvc,
                   "phase_ms_per_step_stream_ordered": {k: v / prof_steps for k, v in pst["phase_ms"].items()},
                   "step_path": ("pic_step_graph (CUDA graph per step, V-cycle loop as a conditional WHILE node)"
                                 if args.step_path == "graph" else "pic_step (stream-ordered launches)")},
        "int64": int64,
        "roofline": roofline,
        "step_roofline": step_roofline,
        "gpu_launches": st["kernel_launches"],
        "clocks": r["clocks"].summary(),
        "e2e": e2e,
    }
    if rank == 0 and world == 1 and not args.no_ref_cuda:
        if args.workload in ("large", "mcc_mixed"):
            try:
                line["reference_particle_kernels"] = reference_particle_kernels(cfg, particles, mover_ms, Te, Ti)
            except (OSError, AssertionError) as e:
                line["reference_particle_kernels"] = {"unavailable": str(e)}
        line["reference_cuda_demo"] = reference_cuda(local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(args, cfg, n, Te, Ti, Ld)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_e2e(args, cfg, n, Te, Ti, Ld, steps_job, local, rank):
    import torch
    from pic_cuda_b200 import configs as cf
    from pic_cuda_b200.engine import Engine
    steps = args.e2e_steps or steps_job
    host = []
    for s, (T, m, seed) in enumerate([(Te, cf.ME, 2000 + rank), (Ti, cf.M_AR, 3000 + rank)]):
        arrs = cf.maxwellian_state(n, Ld, T, m, seed)
        host.append([torch.from_numpy(a).pin_memory() for a in arrs])
    out = [[torch.empty(cfg.species[s].capacity, dtype=torch.float64).pin_memory() for _ in range(5)] for s in (0, 1)]
    eng = Engine(local)
    job = eng.add_job(cfg)
    torch.cuda.synchronize()
    import ctypes as C
    from pic_cuda_b200 import _lib as L
    t0 = time.perf_counter()
    for s in (0, 1):
        job.load_species(s, *host[s])
    t_load = time.perf_counter() - t0
    for _ in range(steps):
        eng.step_graph(1)
        job.diagnostics()
    t_steps = time.perf_counter() - t0 - t_load
    counts = []
    for s in (0, 1):
        nn = C.c_int64()
        p = [C.c_void_p(t.data_ptr()) for t in out[s]]
        L.check(L.lib().pic_job_export_species(eng.h, job.id, s, cfg.species[s].capacity, *p, None, C.byref(nn),
                                               L.MEM_HOST), "export")
        counts.append(nn.value)
    dt = time.perf_counter() - t0
    h2d = 2 * n * 5 * 8
    d2h = sum(counts) * 5 * 8 + steps * L.C.sizeof(L.Diagnostics)
    job.destroy()
    eng.close()
    return {"value": 2 * n * steps / dt, "unit": UNIT, "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps, "steps": steps, "seconds": dt,
            "seconds_load": t_load, "seconds_steps": t_steps, "seconds_export": dt - t_load - t_steps,
            "path": "pic_job_load_species (pinned host) -> pic_step_graph + pic_job_diagnostics per step -> "
                    "pic_job_export_species (pinned host)"}


def run_batched_bench(args):
    """Batched mix in HBM-budgeted waves (one set of launches per step for a wave's jobs,
    autotuned) against the same jobs one after another with the plain step.  Under torchrun
    the jobs are split over the ranks by work (shard.shard_jobs), each rank runs its share,
    and the line reports the whole mix: work summed, time the slowest rank's."""
    import torch
    from pic_cuda_b200 import autotune, batch, shard
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    n_jobs = args.jobs or 256
    scale = args.ppc_scale if args.ppc_scale is not None else 0.02
    all_specs = batch.batched_specs(n_jobs, seed=4, ppc_scale=scale, steps=300)
    mine = shard.shard_jobs([sp.particle_steps for sp in all_specs], world)[rank]
    specs = [all_specs[j] for j in mine]
    budget = int((args.budget_gb or 120.0) * 1e9)
    torch.cuda.synchronize()
    tuner = autotune.Tuner()
    with ClockSampler(local) as clk:
        b = batch.run_batched(specs, budget, device=local, tuner=tuner)
        seq = batch.run_sequential(specs, device=local)
    dev = torch.device("cuda", local)
    sec, work = shard.reduce_timing(b.seconds, b.particle_steps, dist, dev)
    seq_sec, seq_work = shard.reduce_timing(seq.seconds, seq.particle_steps, dist, dev)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    rate, seq_rate = work / sec, seq_work / seq_sec
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": 300, "warmup": 0,
            "ms_per_step": 1000.0 * sec / 300, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "mode": "batched",
            "config": {"workload": "batched", "jobs": n_jobs, "ppc_scale": scale,
                       "grids": "uniform over {65,129,257,513}^2", "ppc": "U[50,400] x ppc_scale per species",
                       "waves": b.waves, "budget_gb": budget / 1e9, "tuned": tuner.chosen,
                       "particle_steps": work, "parallelism": f"jobs sharded over {world} ranks by work"
                       if world > 1 else "single GPU"},
            "sequential": {"value": seq_rate, "seconds": seq_sec, "particle_steps": seq_work},
            "speedup_vs_sequential": rate / seq_rate if seq_rate > 0 else None,
            "seconds": sec, "wall_seconds": b.wall_seconds, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_served_bench(args):
    """Poisson request stream through the continuous-batching server, against the same
    stream served one job at a time (each job's measured alone time, replayed FIFO).  Under
    torchrun the stream holds N times the requests at N times the rate and every rank serves
    every N-th request in arrival order (shard.shard_requests), so each GPU sees the one-GPU
    load; the line reports the whole stream (work summed, makespan the slowest rank's,
    p50/p99 over all requests)."""
    import torch
    from pic_cuda_b200 import serve, shard
    from pic_cuda_b200.engine import Engine
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    n_req = (args.jobs or 48) * world
    scale = args.ppc_scale if args.ppc_scale is not None else 0.05
    sscale = args.steps_scale if args.steps_scale is not None else 0.1
    # the arrival rate: 1.5 x the particle-steps/s this GPU sustains on a sample of the mix,
    # measured here (every rank measures its own; rank 0's figure sets the stream)
    sample = serve.served_requests(32, seed=6, ppc_scale=scale, steps_scale=sscale)
    capacity = serve.measure_capacity([r.spec for r in sample], device=local)
    if dist:
        cap_t = torch.tensor([capacity], dtype=torch.float64, device=torch.device("cuda", local))
        dist.broadcast(cap_t, 0)
        capacity = float(cap_t.item())
    all_reqs = serve.served_requests(n_req, seed=5, ppc_scale=scale, steps_scale=sscale,
                                     capacity=capacity * world)
    reqs = [all_reqs[k] for k in shard.shard_requests([r.arrival for r in all_reqs], world, rank)]
    budget = int((args.budget_gb or 150.0) * 1e9)
    dev = torch.device("cuda", local)
    eng = Engine(local)
    with ClockSampler(local) as clk:
        out = serve.Server(engine=eng, budget_bytes=budget, quantum=20, device=dev).run(reqs)
        eng.close()
        durations = [serve.run_alone(r.spec, device=local)[0] for r in reqs]
    seq = serve.fifo_replay(reqs, durations)
    makespan, work = shard.reduce_timing(out["makespan"], out["particle_steps"], dist, dev)
    seq_makespan, seq_work = shard.reduce_timing(seq["makespan"], seq["particle_steps"], dist, dev)
    lat = shard.gather_latencies([c.latency for c in out["completions"]], dist)
    seq_lat = shard.gather_latencies(seq["latencies"], dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    pct, seq_pct = serve.percentiles(lat), serve.percentiles(seq_lat)
    rate, seq_rate = work / makespan, seq_work / seq_makespan
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": None, "warmup": 0,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "mode": "served",
            "config": {"workload": "served", "requests": n_req, "ppc_scale": scale, "steps_scale": sscale,
                       "grids": "uniform over {129,257,513,1025}^2",
                       "arrivals": "Poisson at 1.5x the capacity measured in this run on a 32-request sample",
                       "capacity_measured": capacity,
                       "budget_gb": budget / 1e9, "quantum_steps": 20,
                       "parallelism": f"every {world}-th request per rank" if world > 1 else "single GPU"},
            "p50_s": pct["p50"], "p99_s": pct["p99"], "makespan_s": makespan,
            "server_seconds_in": out["seconds_in"],
            "sequential": {"value": seq_rate, "p50_s": seq_pct["p50"], "p99_s": seq_pct["p99"],
                           "makespan_s": seq_makespan},
            "speedup_vs_sequential": rate / seq_rate if seq_rate > 0 else None,
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


# Embedded-boundary multigrid (Multigrid_embedded.cu) on its own: 4097^2 nodes (the large
# configuration's grid; ~0.55 GB of level arrays, larger than L2), an electrode at 2.5 whose
# edges sit on odd and even nodes and a solid block, random charge, V(2,2) cycles over 10
# levels with the coarsening the reference's comment states and bilinear prolongation.
EMB_N, EMB_LEVELS = 4097, 10


def embedded_problem(n):
    import numpy as np
    rng = np.random.default_rng(4242)
    mask = np.zeros((n, n), np.uint8)
    mask[n // 4: n // 2, n // 4: n // 2 + 1] = 1
    mask[3 * n // 5: 3 * n // 4, 3 * n // 5: 4 * n // 5] = 2
    bc = np.where(mask == 1, 2.5, 0.0)
    return np.zeros((n, n)), rng.standard_normal((n, n)), mask, bc


def embedded_bytes_per_cycle(n, levels):
    """Algorithmic HBM bytes of one V-cycle, counted once: per level above the one-CTA ones,
    pre-smoothing with the restriction (phi, rhs, kinds read: 17 B/node; phi written: 8 B/node;
    coarse rhs, kinds and phi written: 17 B per coarse node) and prolongation + post-smoothing
    (phi, rhs, kinds read and phi written: 25 B/node; coarse phi read: 8 B per coarse node);
    the one-CTA levels read and write their arrays once (25 B/node)."""
    b, a = 0, n
    for l in range(levels):
        N, Nc = a * a, ((a - 1) // 2 + 1) ** 2
        if N <= 65 * 65:
            b += 25 * N
        else:
            b += 25 * N + 17 * Nc + 25 * N + 8 * Nc
        a = (a - 1) // 2 + 1
    return b


def run_embedded_bench(args):
    import numpy as np
    import torch
    from oracle import oracle as orc
    from pic_cuda_b200 import _lib as L
    from pic_cuda_b200.engine import solve_embedded_f64
    unit = "V-cycles/s"
    n, levels = EMB_N, EMB_LEVELS
    h = 1.0 / (n - 1)
    phi, rhs, mask, bc = embedded_problem(n)
    opts = L.EMB_COARSEN_ANY | L.EMB_PROLONG_BILINEAR
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        cyc = max(1, min(args.steps, args.cpu_steps))
        orc.emb_vcycles(phi, rhs, mask, bc, h, levels, 1, options=opts)
        t0 = time.perf_counter()
        orc.emb_vcycles(phi, rhs, mask, bc, h, levels, cyc, options=opts)
        v = cyc / (time.perf_counter() - t0)
        print(json.dumps({"metric": f"embedded-boundary multigrid {unit}", "value": v, "unit": unit, "impl": "reference",
                          "n_gpus": args.gpus, "steps": cyc, "warmup": 1, "higher_is_better": True,
                          "dtype": "f64", "data": "synthetic", "config": {"workload": "embedded", "grid": f"{n}x{n}"},
                          "cpu_baseline": {"value": v, "unit": unit, "cores": orc.num_threads(), "kind": "port",
                                           "sample": f"{cyc} oracle V-cycles"},
                          "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    dev = torch.device("cuda", 0)
    d = {k: torch.tensor(a, device=dev) for k, a in (("phi", phi), ("rhs", rhs), ("mask", mask), ("bc", bc))}
    stream = torch.cuda.current_stream(dev)
    solve_embedded_f64(d["phi"], d["rhs"], d["mask"], d["bc"], levels, h, 2, 2, opts, tol=0.0,
                       max_cycles=max(args.warmup, 3))
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        ev0.record(stream)
        solve_embedded_f64(d["phi"], d["rhs"], d["mask"], d["bc"], levels, h, 2, 2, opts, tol=0.0,
                           max_cycles=args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    peak, peak_kind = peaks()
    bpc = embedded_bytes_per_cycle(n, levels)
    # end to end: pinned host arrays in, a solve to 1e-8 (at most 200 V-cycles) through the C ABI,
    # phi back to the host
    e2e = None
    if not args.no_e2e:
        hp = {k: torch.from_numpy(a).pin_memory() for k, a in (("phi", phi), ("rhs", rhs), ("mask", mask),
                                                                ("bc", bc))}
        out = torch.empty_like(hp["phi"]).pin_memory()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dd = {k: v.to(dev, non_blocking=True) for k, v in hp.items()}
        cyc, rel, ok = solve_embedded_f64(dd["phi"], dd["rhs"], dd["mask"], dd["bc"], levels, h, 2, 2, opts,
                                          tol=1e-8, max_cycles=200)
        out.copy_(dd["phi"])
        e2e_s = time.perf_counter() - t0
        e2e = {"value": cyc / e2e_s, "unit": unit, "h2d_bytes_per_step": 25 * n * n / cyc,
               "d2h_bytes_per_step": 8 * n * n / cyc, "cycles": cyc, "relres": rel, "converged": ok,
               "seconds": e2e_s}
    # the reference's own kernels in its V-cycle sequence on the same B200 and problem
    ref = None
    if not args.no_ref_cuda:
        try:
            from oracle import refh
            if refh.available():
                _, ref_ms = refh.emb_vcycles_timed(phi, rhs, mask, bc, h, levels, 20, warmup=3)
                ref = {"ms_per_vcycle": ref_ms, "vcycles_per_s": 1000.0 / ref_ms, "speedup": ref_ms / ms,
                       "path": "Multigrid::vcycle (Multigrid_embedded.cu:159-188) re-sequenced on the reference's "
                               "kernels, 8x8 blocks, legacy stream; its colour test races (:22)"}
        except (OSError, AssertionError) as e:
            ref = {"unavailable": str(e)}
    line = {"metric": f"embedded-boundary multigrid {unit}", "value": 1000.0 / ms, "unit": unit, "n_gpus": 1,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "embedded", "grid": f"{n}x{n}", "levels": levels, "sweeps": "2+2",
                       "options": "coarsen any + bilinear prolongation",
                       "l2": "level arrays larger than L2 (no flush needed)"},
            "roofline": {"bound": "hbm", "achieved": bpc / (ms / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": bpc / (ms / 1000.0) / 1e9 / peak, "traffic": None, "kernel": "whole V-cycle",
                         "bytes_per_vcycle": bpc, "peak_source": f"{peak_kind} hbm_gbs"},
            "clocks": clk.summary(),
            "e2e": e2e,
            "reference_cuda": ref}
    if not args.no_cpu_baseline:
        cyc_cpu = max(1, args.cpu_steps)
        orc.emb_vcycles(phi, rhs, mask, bc, h, levels, 1, options=opts)
        t0 = time.perf_counter()
        orc.emb_vcycles(phi, rhs, mask, bc, h, levels, cyc_cpu, options=opts)
        line["cpu_baseline"] = {"value": cyc_cpu / (time.perf_counter() - t0), "unit": unit,
                                "cores": orc.num_threads(), "kind": "port", "sample": f"{cyc_cpu} oracle V-cycles"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "embedded":
        run_embedded_bench(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched_bench(args)
    elif args.workload == "served":
        run_served_bench(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
