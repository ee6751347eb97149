"""GPU parity at the benchmark configurations, through the C ABI, against the FP64 CPU oracle.

  plain_small  129^2, 1e5 + 1e5 particles, 100 steps, no collisions, multigrid to 1e-6:
               run side by side with the oracle from one loaded state.  Every step: particle
               counts + absorbed = loaded (exact), total charge = (N_i - N_e) q W (FP32 deposit:
               within 1e-5 of q W N), relres < 1e-6.  After 100 steps (the FP32 engine and the
               FP64 oracle drift apart by rounding; measured with an FP32-rounded oracle run:
               <= 5e-6 of the domain in position, <= 1e-5 in phi, one survivor differing):
               survivor sets differ by <= 10 pids per species, positions of common pids within
               1e-5 of the domain at the 99.9th percentile and 1e-4 at most, phi within 1e-4
               and rho within 1e-2 relative L2.
  mcc_mixed    1025^2, 1e7 + 1e7 particles, argon null-collision MCC, absorbing walls, FP32
               V-cycles in FP64 defect correction to 1e-9.  Three consecutive steps; before each
               step the oracle is loaded with the engine's state (particles, phi, step index,
               next particle id), so every step is checked from one input:
                 rho, phi               <= 1e-6 relative L2
                 relres                 <= 1e-9 (engine) and <= 1.5e-9 recomputed in FP64 here
                 survivor pid set       exact
                 x, y per pid           <= 1e-6 of the domain
                 v per pid              particles the oracle did not collide: <= 1e-6 of the
                                        species' RMS speed; collided ones: <= 3e-4 of their
                                        speed + 1e-6 of the RMS speed (FP32 isotropic
                                        directions lose precision as sin(chi) -> 0); at most
                                        40 exceptions per species (collision outcomes that
                                        differ: FP32 against FP64 process choice at a boundary)
                 collisions per process, ionisations   within 10 of the oracle's
  large        4097^2, 1e8 + 1e8 particles, same MCC, one step with the FP32 deposit and one
               with the int64 deposit from the same loaded state:
                 int64 rho              total = (N_i - N_e) 2^40 units exactly
                 FP32 rho vs int64 rho  <= 1e-6 relative L2
                 FP32 rho vs the oracle's FP64 deposit of the engine's positions   <= 1e-6
                 relres                 <= 1e-9 (engine) and <= 1.5e-9 recomputed here
"""
import numpy as np
import pytest

from conftest import rel_l2
from pic_cuda_b200 import _lib as L
from pic_cuda_b200 import configs as cf

pytestmark = pytest.mark.gpu


def _by_pid(d):
    o = np.argsort(d["pid"], kind="stable")
    return {k: v[o] for k, v in d.items()}


def _common(a, b):
    """Indices into pid-sorted a and b of the pids both hold."""
    com = np.intersect1d(a["pid"], b["pid"], assume_unique=True)
    return np.searchsorted(a["pid"], com), np.searchsorted(b["pid"], com)


def test_plain_small_100_steps_against_oracle(engine, orc):
    n, steps = 100_000, 100
    cfg = cf.plain_small()
    job = engine.add_job(cfg)
    try:
        cf.load_plasma(job, n, cfg.Lx, 2.0, 0.03, seed=1234)
        init = [job.export_species(s) for s in (0, 1)]
        sim = orc.Sim(cfg)
        for s in (0, 1):
            d = init[s]
            sim.load(s, d["x"], d["y"], d["vx"], d["vy"], d["vz"], d["pid"])
        qw = cf.QE * cfg.species[0].weight
        absorbed = [0, 0]
        for _ in range(steps):
            engine.step(1)
            sim.step(1)
            d = job.diagnostics()
            for s in (0, 1):
                absorbed[s] += d["absorbed"][s]
                assert d["count"][s] + absorbed[s] == n  # no collisions: absorption only
            assert d["converged"] and d["relres"] < 1e-6
            exact = qw * (d["count"][1] - d["count"][0])
            assert abs(d["total_charge"] - exact) < 1e-5 * qw * 2 * n
        assert absorbed[0] > 0
        assert rel_l2(job.get_grid(L.GRID_PHI), sim.grid(L.GRID_PHI)) < 1e-4
        assert rel_l2(job.get_grid(L.GRID_RHO), sim.grid(L.GRID_RHO)) < 1e-2
        for s in (0, 1):
            a, b = _by_pid(job.export_species(s)), _by_pid(sim.export(s))
            assert len(np.setxor1d(a["pid"], b["pid"])) <= 10
            ia, ib = _common(a, b)
            err = np.maximum(np.abs(a["x"][ia] - b["x"][ib]), np.abs(a["y"][ia] - b["y"][ib])) / cfg.Lx
            assert np.quantile(err, 0.999) < 1e-5 and err.max() < 1e-4, (s, np.quantile(err, 0.999), err.max())
    finally:
        job.destroy()


def test_mcc_mixed_three_steps_against_oracle(engine, orc):
    n = 10_000_000
    cfg = cf.mcc_mixed(n_per_species=n)
    job = engine.add_job(cfg)
    try:
        cf.load_plasma(job, n, cfg.Lx, 3.0, 0.03, seed=1234)
        h = cfg.Lx / (cfg.nx - 1)
        rhs_scale = -1.0 / (8.8541878128e-12 * h * h)
        for k in range(3):
            # the oracle continues from the engine's state as it stands
            state = [job.export_species(s) for s in (0, 1)]
            d0 = job.diagnostics()
            sim = orc.Sim(cfg)
            for s in (0, 1):
                st = state[s]
                sim.load(s, st["x"], st["y"], st["vx"], st["vy"], st["vz"], st["pid"])
            sim.set_grid(L.GRID_PHI, job.get_grid(L.GRID_PHI))
            sim.set_counters(d0["step"], d0["next_pid"])
            engine.step(1)
            # the oracle's step phase by phase, to know which particles its collisions changed
            sim.drift_walls()
            sim.deposit()
            sim.solve()
            sim.kick()
            kicked = [_by_pid(sim.export(s)) for s in (0, 1)]
            sim.mcc()
            rho, phi = job.get_grid(L.GRID_RHO), job.get_grid(L.GRID_PHI)
            assert rel_l2(rho, sim.grid(L.GRID_RHO)) < 1e-6, k
            assert rel_l2(phi, sim.grid(L.GRID_PHI)) < 1e-6, k
            d = job.diagnostics()
            assert d["converged"] and d["relres"] < 1e-9, (k, d["relres"])
            assert orc.relres(phi, rhs_scale * rho, h) < 1.5e-9
            # the read-back applies the step's deferred kick and collisions (the oracle's step
            # ends with them); the collision counters then hold this step's
            after = [job.export_species(s) for s in (0, 1)]
            d = job.diagnostics()
            st = sim.stats()
            for s in (0, 1):
                a, b = _by_pid(after[s]), _by_pid(sim.export(s))
                old_a, old_b = a["pid"] < d0["next_pid"], b["pid"] < d0["next_pid"]
                # survivors among the particles that entered the step: exact
                assert np.array_equal(a["pid"][old_a], b["pid"][old_b]), (k, s)
                ia, ib = np.nonzero(old_a)[0], np.nonzero(old_b)[0]
                for c in ("x", "y"):
                    assert np.max(np.abs(a[c][ia] - b[c][ib])) / cfg.Lx < 1e-6, (k, s, c)
                vb = np.stack([b["vx"][ib], b["vy"][ib], b["vz"][ib]])
                va = np.stack([a["vx"][ia], a["vy"][ia], a["vz"][ia]])
                vk = np.stack([kicked[s]["vx"], kicked[s]["vy"], kicked[s]["vz"]])
                assert np.array_equal(kicked[s]["pid"], b["pid"][ib])
                collided = np.any(vk != vb, axis=0)
                vrms = np.sqrt(np.mean(np.sum(vb ** 2, axis=0)))
                err = np.linalg.norm(va - vb, axis=0)
                bound = np.where(collided, 3e-4 * np.linalg.norm(vb, axis=0), 0.0) + 1e-6 * vrms
                assert collided.sum() > 0
                assert (err > bound).sum() <= 40, (k, s, int((err > bound).sum()), int(collided.sum()))
                for p in range(4):
                    assert abs(d["collisions"][s][p] - st["collisions"][s][p]) <= 10, (k, s, p)
                # the pairs the step's ionisations appended (pid >= the step's first new id)
                assert abs(int((~old_a).sum()) - int((~old_b).sum())) <= 20, (k, s)
            assert st["ionizations"] > 0
            assert abs(d["ionizations"] - st["ionizations"]) <= 10, k
            assert sum(st["collisions"][0][:3]) > 1000 and st["collisions"][1][3] > 0
    finally:
        job.destroy()


def _oracle_deposit_of_engine_positions(orc, job, cfg, first_new_pid, chunk=20_000_000):
    """The oracle's FP64 CIC deposit of the engine's current positions (taken from its FP32
    cell-relative layout on the device, chunk by chunk), over the particles that existed at
    the last deposit (pid below first_new_pid)."""
    nx = cfg.nx
    h = cfg.Lx / (nx - 1)
    rho = np.zeros((nx, nx))
    for s in (0, 1):
        raw = job.export_raw(s)
        q = cfg.species[s].charge * cfg.species[s].weight
        n = raw["cell"].shape[0]
        for a in range(0, n, chunk):
            cell = raw["cell"][a:a + chunk].cpu().numpy().view(np.uint32)
            pid = raw["pid"][a:a + chunk].cpu().numpy().view(np.uint32)
            keep = (pid < first_new_pid) & (cell != 0xFFFFFFFF)
            cell = cell[keep]
            fx = raw["fx"][a:a + chunk].cpu().numpy()[keep].astype(np.float64)
            fy = raw["fy"][a:a + chunk].cpu().numpy()[keep].astype(np.float64)
            x = ((cell & 0xFFFF).astype(np.float64) + fx) * h
            y = ((cell >> 16).astype(np.float64) + fy) * h
            rho += orc.deposit(x, y, q, nx, nx, h, h)
        del raw
    return rho


def test_large_one_step_both_deposits(engine, orc):
    import torch
    n = 100_000_000
    dev = torch.device("cuda", 0)
    out = {}
    for mode in (L.DEPOSIT_F32, L.DEPOSIT_I64):
        cfg = cf.large(n_per_species=n, deposit=mode)
        job = engine.add_job(cfg)
        try:
            cf.load_plasma(job, n, cfg.Lx, 2.0, 0.03, seed=99, device=dev)
            torch.cuda.synchronize()
            engine.step(1)
            d = job.diagnostics()
            rho, phi = job.get_grid(L.GRID_RHO), job.get_grid(L.GRID_PHI)
            h = cfg.Lx / (cfg.nx - 1)
            assert d["converged"] and d["relres"] < 1e-9, d["relres"]
            assert orc.relres(phi, -rho / (8.8541878128e-12 * h * h), h) < 1.5e-9
            # one step of thermal motion: only particles within a cell of the walls can leave
            assert min(d["count"]) > 0.99 * n, d["count"]
            qw = cf.QE * cfg.species[0].weight
            if mode == L.DEPOSIT_I64:
                units = np.rint(rho / qw * 2.0 ** 40).astype(np.int64)
                # exact sum in Python integers (the total exceeds int64 for ~1e7 net charges)
                total = int((units >> 20).sum()) * 2 ** 20 + int((units & (2 ** 20 - 1)).sum())
                assert total == (d["count"][1] - d["count"][0]) * 2 ** 40
            else:
                ref = _oracle_deposit_of_engine_positions(orc, job, cfg, d["next_pid"])
                assert rel_l2(rho, ref) < 1e-6
            out[mode] = (rho, d["count"])
        finally:
            job.destroy()
    assert out[L.DEPOSIT_F32][1] == out[L.DEPOSIT_I64][1]
    assert rel_l2(out[L.DEPOSIT_F32][0], out[L.DEPOSIT_I64][0]) < 1e-6
