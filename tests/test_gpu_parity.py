"""GPU parity of the engine (through the C ABI) against the FP64 CPU oracle.

Tolerances (stated per result, as the FP32 engine is checked against an FP64 oracle):
  deposited rho, FP32 mode             <= 1e-6 relative L2 (sorted particles)
  deposited rho, int64 fixed point     <= 1e-6 relative L2, total exact, order independent
  phi after k identical V-cycles       <= 1e-6 relative L2
  phi after FP64 defect correction     relative residual (FP64, recomputed here) <= 1e-9
  one-step pushed x, v                 <= 1e-6 relative (x to the domain size; v as relative L2
                                       over the species and per particle to the species' RMS
                                       speed: a particle slower than its own kick carries the
                                       FP32 rounding of v + dv, ~6e-8 of |dv|)
  absorbed set for given positions     exact
"""
import numpy as np
import pytest

from conftest import rel_l2
from pic_cuda_b200 import _lib as L
from pic_cuda_b200 import configs as cf

pytestmark = pytest.mark.gpu


def _state(job, species):
    return job.export_species(species)


def _small_plasma(engine, n=100_000, nx=129, deposit=L.DEPOSIT_F32, seed=1234, **kw):
    cfg = cf.plasma(nx, 0.01, n, deposit=deposit, **kw)
    job = engine.add_job(cfg)
    cf.load_plasma(job, n, 0.01, 2.0, 0.03, seed=seed)
    return cfg, job


@pytest.mark.parametrize("mode", [L.DEPOSIT_F32, L.DEPOSIT_I64])
def test_deposit_matches_oracle(engine, orc, mode):
    cfg, job = _small_plasma(engine, deposit=mode)
    try:
        dx = cfg.Lx / (cfg.nx - 1)
        e, i = _state(job, 0), _state(job, 1)
        w = cfg.species[0].weight
        q = np.concatenate([np.full(len(e["x"]), -cf.QE * w), np.full(len(i["x"]), cf.QE * w)])
        ref = orc.deposit(np.concatenate([e["x"], i["x"]]), np.concatenate([e["y"], i["y"]]), q, cfg.nx, cfg.ny,
                          dx, dx)
        job.sort()
        job.zero_rho()
        job.run_phases(L.PHASE_DEPOSIT)
        rho = job.get_grid(L.GRID_RHO)
        assert rel_l2(rho, ref) < 1e-6
        if mode == L.DEPOSIT_I64:
            # exact total: every particle's four weights sum to its quantised charge
            units = np.rint(rho / (cf.QE * w) * 2.0 ** 40).astype(np.int64)
            assert units.sum() == (len(i["x"]) - len(e["x"])) * 2 ** 40
            # bit-identical when deposited from an unsorted order
            job2 = engine.add_job(cfg)
            perm = np.random.default_rng(5).permutation(len(e["x"]))
            job2.load_species(0, e["x"][perm], e["y"][perm], e["vx"][perm], e["vy"][perm], e["vz"][perm])
            job2.load_species(1, i["x"], i["y"], i["vx"], i["vy"], i["vz"])
            job2.zero_rho()
            job2.run_phases(L.PHASE_DEPOSIT)
            assert np.array_equal(job2.get_grid(L.GRID_RHO), rho)
            job2.destroy()
    finally:
        job.destroy()


@pytest.mark.parametrize("n,levels,omega,nu,tol_cycles", [
    (33, 0, 1.0, (2, 2, 2), 5), (65, 0, 1.0, (2, 2, 2), 5), (129, 0, 1.0, (2, 2, 2), 6),
    (257, 0, 1.0, (2, 2, 2), 6), (129, 5, 1.25, (3, 3, 20), 4), (513, 0, 1.0, (2, 2, 2), 4),
    (513, 6, 1.25, (3, 3, 20), 3), (1025, 0, 1.0, (2, 2, 2), 5)])
def test_multigrid_cycles_match_oracle(orc, n, levels, omega, nu, tol_cycles):
    import torch
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(n)
    f = rng.standard_normal((n, n))
    phi0 = np.zeros((n, n))
    phi0[0, :] = 0.5  # a Dirichlet value on one side
    from pic_cuda_b200.engine import solve_multigrid_f64
    dphi = torch.tensor(phi0, device="cuda")
    drho = torch.tensor(f, device="cuda")
    cyc, rel, ok = solve_multigrid_f64(dphi, drho, n, n, levels, h, omega, *nu, tol=0.0, max_cycles=tol_cycles)
    assert cyc == tol_cycles and not ok
    ref = orc.mg_vcycles(phi0, f, h, tol_cycles, levels=levels, omega=omega, nu1=nu[0], nu2=nu[1], nuc=nu[2])
    got = dphi.cpu().numpy()
    assert rel_l2(got, ref) < 1e-6
    assert np.all(got[0, :] == 0.5)
    # FP64 defect correction reaches 1e-9 (residual recomputed in FP64 on the host)
    dphi = torch.tensor(phi0, device="cuda")
    cyc, rel, ok = solve_multigrid_f64(dphi, drho, n, n, levels, h, omega, *nu, tol=1e-9, max_cycles=60)
    assert ok and rel < 1e-9
    assert orc.relres(dphi.cpu().numpy(), f, h) < 1.5e-9


@pytest.mark.parametrize("n", [257, 513, 1025])
def test_multigrid_cluster_coarse_solver_matches_oracle(orc, monkeypatch, n):
    """The thread-block-cluster coarse solver (levels up to 513^2 in one 16-CTA cluster),
    selected with PIC_MG_CLUSTER_TOP, gives the oracle's V-cycles.  nu_coarse = 4 keys a
    solver instance of its own, created while the variable is set."""
    import torch
    from pic_cuda_b200.engine import solve_multigrid_f64
    monkeypatch.setenv("PIC_MG_CLUSTER_TOP", "513")
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(n + 1)
    f = rng.standard_normal((n, n))
    phi0 = np.zeros((n, n))
    phi0[:, 0] = -0.25
    dphi = torch.tensor(phi0, device="cuda")
    drho = torch.tensor(f, device="cuda")
    cyc, rel, ok = solve_multigrid_f64(dphi, drho, n, n, 0, h, 1.0, 2, 2, 4, tol=0.0, max_cycles=4)
    assert cyc == 4 and not ok
    ref = orc.mg_vcycles(phi0, f, h, 4, levels=0, omega=1.0, nu1=2, nu2=2, nuc=4)
    assert rel_l2(dphi.cpu().numpy(), ref) < 1e-6


@pytest.mark.parametrize("n", [257, 1025])
def test_multigrid_levels_kernel_matches_oracle(orc, monkeypatch, n):
    """Levels 1..lc as phases of one cooperative launch (PIC_MG_LEVELS_KERNEL=1) give the
    oracle's V-cycles.  nu_coarse = 5 keys a solver instance of its own."""
    import torch
    from pic_cuda_b200.engine import solve_multigrid_f64
    monkeypatch.setenv("PIC_MG_LEVELS_KERNEL", "1")
    h = 1.0 / (n - 1)
    rng = np.random.default_rng(n + 2)
    f = rng.standard_normal((n, n))
    phi0 = np.zeros((n, n))
    phi0[-1, :] = 0.75
    dphi = torch.tensor(phi0, device="cuda")
    drho = torch.tensor(f, device="cuda")
    cyc, rel, ok = solve_multigrid_f64(dphi, drho, n, n, 0, h, 1.0, 2, 2, 5, tol=0.0, max_cycles=4)
    assert cyc == 4 and not ok
    ref = orc.mg_vcycles(phi0, f, h, 4, levels=0, omega=1.0, nu1=2, nu2=2, nuc=5)
    assert rel_l2(dphi.cpu().numpy(), ref) < 1e-6


def test_manufactured_solution_second_order_gpu(orc):
    import math
    import torch
    from pic_cuda_b200.engine import solve_multigrid_f64
    errs = []
    for n in (129, 257, 513):
        h = 1.0 / (n - 1)
        X, Y = np.meshgrid(np.arange(n) * h, np.arange(n) * h)
        exact = np.sin(math.pi * X) * np.sin(math.pi * Y)
        dphi = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        drho = torch.tensor(-2 * math.pi ** 2 * exact, device="cuda")
        _, rel, ok = solve_multigrid_f64(dphi, drho, n, n, 0, h, 1.0, 2, 2, 2, tol=1e-10, max_cycles=60)
        assert ok
        errs.append(np.abs(dphi.cpu().numpy() - exact).max())
    assert 3.8 < errs[0] / errs[1] < 4.2 and 3.8 < errs[1] / errs[2] < 4.2


def test_kick_drift_walls_match_oracle(engine, orc):
    cfg, job = _small_plasma(engine, n=50_000, dt=2e-11)
    try:
        n = cfg.nx
        dx = cfg.Lx / (n - 1)
        X, Y = np.meshgrid(np.arange(n) * dx, np.arange(n) * dx)
        phi = 3.0 * np.sin(np.pi * X / cfg.Lx) * np.sin(2 * np.pi * Y / cfg.Lx) + 50.0 * X / cfg.Lx
        job.set_grid(L.GRID_PHI, phi)
        before = [_state(job, s) for s in (0, 1)]
        job.run_phases(L.PHASE_KICK)
        Ex, Ey = orc.efield(job.get_grid(L.GRID_PHI), dx, dx)
        for s in (0, 1):
            b = before[s]
            q, m = cfg.species[s].charge, cfg.species[s].mass
            vx, vy = orc.kick(b["x"], b["y"], b["vx"], b["vy"], q, m, Ex, Ey, dx, dx, cfg.dt)
            a = _state(job, s)
            err = np.hypot(a["vx"] - vx, a["vy"] - vy)
            vrms = np.sqrt(np.mean(vx ** 2 + vy ** 2))
            assert np.max(err) / vrms < 1e-6
            assert np.linalg.norm(err) / np.linalg.norm(np.hypot(vx, vy)) < 1e-6
        mid = [_state(job, s) for s in (0, 1)]
        job.run_phases(L.PHASE_DRIFT | L.PHASE_WALLS)
        keep = {}
        for s in (0, 1):
            m0 = mid[s]
            x, y = orc.drift(m0["x"], m0["y"], m0["vx"], m0["vy"], cfg.dt)
            a = _state(job, s)
            assert np.max(np.abs(a["x"] - x)) / cfg.Lx < 1e-6 and np.max(np.abs(a["y"] - y)) / cfg.Lx < 1e-6
            # absorbed set for the engine's own drifted positions: exact
            hit = orc.walls_box(a["x"], a["y"], n, n, dx, dx)
            assert set(job.hits(s).tolist()) == set(np.nonzero(hit)[0].tolist())
            keep[s] = (set(a["pid"][~hit].tolist()), len(a["x"]) - int(hit.sum()))
        assert len(job.hits(0)) > 0  # electrons reach the walls within one step
        job.compact()
        for s in (0, 1):
            after = _state(job, s)
            assert set(after["pid"].tolist()) == keep[s][0]  # survivor set, exact
            assert len(after["x"]) == keep[s][1]
    finally:
        job.destroy()


def test_full_step_matches_oracle(engine, orc):
    cfg, job = _small_plasma(engine, n=20_000, nx=129, tol=1e-9)
    try:
        init = [_state(job, s) for s in (0, 1)]
        sim = orc.Sim(cfg)
        for s in (0, 1):
            d = init[s]
            sim.load(s, d["x"], d["y"], d["vx"], d["vy"], d["vz"], d["pid"])
        engine.step(1)
        sim.step(1)
        assert rel_l2(job.get_grid(L.GRID_RHO), sim.grid(L.GRID_RHO)) < 1e-6
        assert rel_l2(job.get_grid(L.GRID_PHI), sim.grid(L.GRID_PHI)) < 1e-6
        diag = job.diagnostics()
        assert diag["relres"] < 1e-9 and diag["converged"]
        for s in (0, 1):
            a, b = _state(job, s), sim.export(s)
            ia, ib = np.argsort(a["pid"]), np.argsort(b["pid"])
            assert np.array_equal(a["pid"][ia], b["pid"][ib])
            a = {k: v[ia] for k, v in a.items()}
            b = {k: v[ib] for k, v in b.items()}
            assert np.max(np.abs(a["x"] - b["x"])) / cfg.Lx < 1e-6
            err = np.hypot(a["vx"] - b["vx"], a["vy"] - b["vy"])
            assert np.max(err) / np.sqrt(np.mean(b["vx"] ** 2 + b["vy"] ** 2)) < 1e-6
            assert np.linalg.norm(err) / np.linalg.norm(np.hypot(b["vx"], b["vy"])) < 1e-6
    finally:
        job.destroy()


def test_multi_step_conservation_and_sort(engine):
    cfg, job = _small_plasma(engine, n=50_000, deposit=L.DEPOSIT_I64, sort_every=2)
    try:
        for _ in range(5):
            engine.step(1)
            d = job.diagnostics()
            w = cfg.species[0].weight
            # int64 deposit: total charge equals (N_i - N_e) q w to FP64 rounding of the export
            assert abs(d["total_charge"] - cf.QE * w * (d["count"][1] - d["count"][0])) < 1e-6 * cf.QE * w
            assert d["converged"] and d["relres"] < 1e-6
        assert d["step"] == 5
    finally:
        job.destroy()


def test_extrapolated_warm_start_matches_oracle(engine, orc):
    """mg_warm_start = 1: per step, the engine's V-cycle count follows the oracle's, and phi
    agrees with a run using the reference's warm start to the solver tolerance."""
    n = 30_000
    runs = {}
    for ws in (0, 1):
        cfg = cf.plasma(129, 0.01, n, tol=1e-9, warm_start=ws, deposit=L.DEPOSIT_I64)
        job = engine.add_job(cfg)
        cf.load_plasma(job, n, 0.01, 2.0, 0.03, seed=21)
        sim = orc.Sim(cfg)
        for s in (0, 1):
            d = _state(job, s)
            sim.load(s, d["x"], d["y"], d["vx"], d["vy"], d["vz"], d["pid"])
        cyc_e, cyc_o = [], []
        for _ in range(6):
            engine.step(1)
            sim.step(1)
            cyc_e.append(job.diagnostics()["vcycles"])
            cyc_o.append(sim.stats()["cycles"])
            assert job.diagnostics()["relres"] < 1e-9
        runs[ws] = (cyc_e, job.get_grid(L.GRID_PHI))
        assert all(abs(a - b) <= 1 for a, b in zip(cyc_e, cyc_o)), (cyc_e, cyc_o)
        assert rel_l2(job.get_grid(L.GRID_PHI), sim.grid(L.GRID_PHI)) < 1e-5
        job.destroy()
    assert sum(runs[1][0][2:]) < sum(runs[0][0][2:])
    assert rel_l2(runs[1][1], runs[0][1]) < 1e-6


def test_kinetic_energy_diagnostic(engine):
    """The FP64 kinetic-energy diagnostic equals sum 1/2 m W v^2 over the velocities a read-back
    returns (collisionless plasma, so no pair is created by the read-back's own pass; without
    collisions vz never changes and the diagnostic counts the in-plane velocity)."""
    cfg, job = _small_plasma(engine, n=100_000)
    try:
        engine.step(3)
        ex = [job.export_species(s) for s in (0, 1)]
        d = job.diagnostics()
        for s in (0, 1):
            e = ex[s]
            v2 = e["vx"].astype(np.float64) ** 2 + e["vy"].astype(np.float64) ** 2
            sp = cfg.species[s]
            ref = 0.5 * sp.mass * sp.weight * v2.sum()
            assert abs(d["kinetic_energy"][s] - ref) <= 1e-6 * ref, (s, d["kinetic_energy"][s], ref)
    finally:
        job.destroy()
