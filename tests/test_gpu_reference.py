"""Pins the oracle to the reference's own CUDA kernels (oracle/_ref/libpicref.so, built from
the reference's sources by oracle/Makefile) and checks the engine against both on the
reference's own nondimensional setup (REF units, segment walls)."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle import refh
from pic_cuda_b200 import _lib as L
from pic_cuda_b200 import configs as cf

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refh.LIB.exists(), reason="reference CUDA build (oracle/_ref) not present")]

# The reference's demo species: Particles2D sets q[0]=0.1, m[0]=1 (particles.cu:146-149) and
# main.cu:188 adds (m=1, q=-1); walls: the domain box plus the two interior walls of main.cu:193-194.
Q, M = [0.1, -1.0], [1.0, 1.0]
WALLS = [[0, 0, 1, 0], [1, 0, 1, 1], [1, 1, 0, 1], [0, 1, 0, 0], [0.25, 0.25, 0.25, 0.75], [0.75, 0.25, 0.75, 0.75]]


def test_reference_deposit_matches_oracle(orc):
    rng = np.random.default_rng(0)
    n = 50_000
    x, y = rng.random(n), rng.random(n)
    t = rng.integers(0, 2, n)
    rho_ref = refh.deposit(x, y, t, Q, 65, 65, 1 / 64, 1 / 64)
    rho_orc = orc.deposit(x, y, np.array(Q)[t], 65, 65, 1 / 64, 1 / 64)
    assert rel_l2(rho_orc, rho_ref) < 1e-12


def test_reference_solver_matches_oracle(orc):
    rng = np.random.default_rng(1)
    n = 129
    f = rng.standard_normal((n, n))
    phi_ref = refh.solve(np.zeros((n, n)), f, 1 / 128, levels=5, omega=1.25)
    phi_orc, cyc, rel = orc.mg_solve(np.zeros((n, n)), f, 1 / 128, levels=5, omega=1.25, nu1=3, nu2=3, nuc=20,
                                     tol=1e-5, max_cycles=50, ref_convergence=True)
    assert rel_l2(phi_orc, phi_ref) < 1e-10


def test_reference_efield_matches_oracle(orc):
    rng = np.random.default_rng(2)
    phi = rng.standard_normal((33, 65))
    ex_r, ey_r = refh.efield(phi, 0.1, 0.2)
    ex_o, ey_o = orc.efield(phi, 0.1, 0.2)
    assert np.max(np.abs(ex_r - ex_o)) < 1e-12 and np.max(np.abs(ey_r - ey_o)) < 1e-12


def _ref_state(n=20_000, seed=3):
    rng = np.random.default_rng(seed)
    x, y = rng.random(n) * 0.98 + 0.01, rng.random(n) * 0.98 + 0.01
    vx, vy = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    t = rng.integers(0, 2, n)
    dt = 0.01
    # put every particle whose first drift crosses a wall at the front, so the reference's
    # hole filling (particles.cu:217-262) sees no tail hits and at most 256 holes
    import oracle.oracle as o
    x1, y1 = x + vx * dt, y + vy * dt
    hit = o.walls_segments(x, y, x1, y1, WALLS)
    order = np.concatenate([np.nonzero(hit)[0], np.nonzero(~hit)[0]])
    return x[order], y[order], vx[order], vy[order], t[order], dt, int(hit.sum())


def test_reference_step_matches_oracle(orc):
    x, y, vx, vy, t, dt, k = _ref_state()
    assert 0 < k <= 256
    out = refh.steps(1, x, y, vx, vy, t, Q, M, 129, 129, 1.0, 1.0, WALLS, dt)
    # hit set before removal: exact
    assert set(out["hits"].tolist()) == set(range(k))
    cfg = cf.make_config(129, 1.0, dt, [(Q[0], M[0], 1.0, 30000), (Q[1], M[1], 1.0, 30000)], units=L.UNITS_REF,
                         walls=L.WALLS_SEGMENTS, wall_segments=WALLS, levels=5, omega=1.25, nu_pre=3, nu_post=3,
                         nu_coarse=20, tol=1e-5)
    sim = orc.Sim(cfg)
    for s in (0, 1):
        sel = t == s
        sim.load(s, x[sel], y[sel], vx[sel], vy[sel])
    orc.set_reference_convergence(True)
    try:
        sim.step(1)
    finally:
        orc.set_reference_convergence(False)
    assert rel_l2(sim.grid(L.GRID_RHO), out["rho"]) < 1e-12
    assert rel_l2(sim.grid(L.GRID_PHI), out["phi"]) < 1e-9
    for s in (0, 1):
        o = sim.export(s)
        sel = out["type"] == s
        a = np.lexsort((out["y"][sel], out["x"][sel]))
        b = np.lexsort((o["y"], o["x"]))
        assert sel.sum() == len(o["x"])
        np.testing.assert_allclose(out["x"][sel][a], o["x"][b], rtol=0, atol=1e-12)
        np.testing.assert_allclose(out["vx"][sel][a], o["vx"][b], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(out["vy"][sel][a], o["vy"][b], rtol=1e-9, atol=1e-12)


def test_engine_step_matches_reference(engine):
    x, y, vx, vy, t, dt, k = _ref_state(seed=4)
    out = refh.steps(1, x, y, vx, vy, t, Q, M, 129, 129, 1.0, 1.0, WALLS, dt)
    cfg = cf.make_config(129, 1.0, dt, [(Q[0], M[0], 1.0, 30000), (Q[1], M[1], 1.0, 30000)], units=L.UNITS_REF,
                         walls=L.WALLS_SEGMENTS, wall_segments=WALLS, levels=5, omega=1.25, nu_pre=3, nu_post=3,
                         nu_coarse=20, tol=1e-9)
    job = engine.add_job(cfg)
    try:
        for s in (0, 1):
            sel = t == s
            job.load_species(s, x[sel], y[sel], vx[sel], vy[sel])
        engine.step(1)
        assert rel_l2(job.get_grid(L.GRID_RHO), out["rho"]) < 1e-6
        # the engine solves to 1e-9, the reference stops at 1e-5: compare against the converged field
        phi = job.get_grid(L.GRID_PHI)
        assert rel_l2(phi, out["phi"]) < 1e-4
        for s in (0, 1):
            o = job.export_species(s)
            sel = out["type"] == s
            assert sel.sum() == len(o["x"])
            a = np.lexsort((out["y"][sel], out["x"][sel]))
            b = np.lexsort((o["y"], o["x"]))
            assert np.max(np.abs(out["x"][sel][a] - o["x"][b])) < 1e-6
    finally:
        job.destroy()


def test_reference_removal_loses_survivors_with_tail_hits():
    # documents the reference's hole-filling defect (particles.cu:63-66): with hits in the
    # tail, dead tail particles are copied into holes and live ones are dropped.
    x, y, vx, vy, t, dt, k = _ref_state(seed=5)
    n = len(x)
    # half of the hitting particles in the head, half in the tail
    h = k // 2
    order = np.concatenate([np.arange(h), np.arange(k, n), np.arange(h, k)])
    x, y, vx, vy, t = x[order], y[order], vx[order], vy[order], t[order]
    out = refh.steps(1, x, y, vx, vy, t, Q, M, 129, 129, 1.0, 1.0, WALLS, dt)
    assert out["n_alive"] == n - k
    import oracle.oracle as o
    xs, ys = x + vx * dt, y + vy * dt
    dead = o.walls_segments(x, y, xs, ys, WALLS)
    assert dead.sum() == k
    dead_positions = set(zip(np.round(xs[dead], 12).tolist(), np.round(ys[dead], 12).tolist()))
    kept = zip(np.round(out["x"], 12).tolist(), np.round(out["y"], 12).tolist())
    kept_dead = sum(1 for p in kept if p in dead_positions)
    # the reference keeps n - k particles, but some of them are ones that hit a wall
    assert kept_dead > 0
