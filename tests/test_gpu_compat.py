"""The reference's host API (include/compat: Grid2D, Particles2D, Boundaries2D,
solve_multigrid, read_cross_section, elasticCollisions, updateSimulationCUDA), called from a
C++ program built against those headers, against the FP64 oracle."""
import numpy as np
import pytest

import compat_io
from conftest import rel_l2
from pic_cuda_b200 import _lib as L
from pic_cuda_b200 import configs as cf

pytestmark = pytest.mark.gpu

# main.cu's demo: species 0 is Particles2D's default (q=0.1, m=1, particles.cu:146-149),
# species 1 is added as (m=1, q=-1) (main.cu:188); walls: the domain box plus main.cu:193-194.
Q, M = [0.1, -1.0], [1.0, 1.0]
WALLS = [[0, 0, 1, 0], [1, 0, 1, 1], [1, 1, 0, 1], [0, 1, 0, 0], [0.25, 0.25, 0.25, 0.75], [0.75, 0.25, 0.75, 0.75]]
GM, DT = 129, 0.01


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    return compat_io.build_driver(tmp_path_factory.mktemp("compat"))


def _state(n=20_000, seed=3):
    rng = np.random.default_rng(seed)
    x, y = rng.random(n) * 0.98 + 0.01, rng.random(n) * 0.98 + 0.01
    vx, vy = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    t = rng.integers(0, 2, n).astype(np.int32)
    return x, y, vx, vy, t


def _step(driver, tmp, st, steps=1, calls=1, maxp=30_000, phi0=None):
    x, y, vx, vy, t = st
    phi0 = np.zeros(GM * GM) if phi0 is None else phi0
    hdr = np.array([GM, 2, len(WALLS), steps, maxp, calls], np.int32)
    out = compat_io.run(driver, "step", tmp,
                        [hdr, np.array([1.0, 1.0, DT]), np.array(Q), np.array(M), np.array(WALLS, float).ravel(),
                         x, y, vx, vy, t, phi0],
                        [np.int32, np.float64, np.float64, np.float64, np.int32, np.int32, np.float64, np.float64,
                         np.float64, np.float64])
    head, r, r_old, v, typ, coll, rho, phi, E, timing = out
    return dict(n=int(head[0]), k=int(head[1]), r=r.reshape(-1, 2), r_old=r_old.reshape(-1, 2), v=v.reshape(-1, 2),
                type=typ, collided=coll, rho=rho.reshape(GM, GM), phi=phi.reshape(GM, GM), E=E.reshape(GM, GM, 2),
                timing=timing)


def _oracle_steps(orc, st, steps, tol=1e-5):
    x, y, vx, vy, t = st
    cfg = cf.make_config(GM, 1.0, DT, [(Q[0], M[0], 1.0, 30000), (Q[1], M[1], 1.0, 30000)], units=L.UNITS_REF,
                         walls=L.WALLS_SEGMENTS, wall_segments=WALLS, levels=5, omega=1.25, nu_pre=3, nu_post=3,
                         nu_coarse=20, tol=tol)
    sim = orc.Sim(cfg)
    idx = np.arange(len(x), dtype=np.uint32)
    for s in (0, 1):
        sel = t == s
        sim.load(s, x[sel], y[sel], vx[sel], vy[sel], None, idx[sel])
    sim.step(steps)
    n = len(x)
    pos = np.full((n, 2), np.nan)
    vel = np.full((n, 2), np.nan)
    for s in (0, 1):
        o = sim.export(s)
        pos[o["pid"], 0], pos[o["pid"], 1] = o["x"], o["y"]
        vel[o["pid"], 0], vel[o["pid"], 1] = o["vx"], o["vy"]
    alive = ~np.isnan(pos[:, 0])
    return sim, alive, pos, vel


def test_update_simulation_one_step_matches_oracle(driver, tmp_path, orc):
    st = _state()
    x, y, vx, vy, t = st
    c = _step(driver, tmp_path, st)
    sim, alive, pos, vel = _oracle_steps(orc, st, 1)
    # removed set: exact, reported as ascending indices into the arrays as passed in
    assert np.array_equal(c["collided"], np.nonzero(~alive)[0])
    assert c["n"] == alive.sum() and c["k"] == (~alive).sum() > 0
    keep = np.nonzero(alive)[0]
    # survivors keep their order and species
    assert np.array_equal(c["type"], t[keep])
    assert np.max(np.abs(c["r"] - pos[keep])) < 1e-7
    # r_old is the position before the drift
    assert np.max(np.abs(c["r_old"][:, 0] - x[keep])) < 1e-6 and np.max(np.abs(c["r_old"][:, 1] - y[keep])) < 1e-6
    # grid: rho exact to the engine's FP32 positions; both solves stop at ||r||/||rho|| < 1e-5
    rho_o = sim.grid(L.GRID_RHO)
    assert rel_l2(c["rho"], rho_o) < 1e-6
    assert orc.relres(c["phi"], c["rho"], 1.0 / (GM - 1)) < 1e-5
    assert rel_l2(c["phi"], sim.grid(L.GRID_PHI)) < 1e-3
    ex, ey = orc.efield(c["phi"], 1.0 / (GM - 1), 1.0 / (GM - 1))
    assert np.max(np.abs(c["E"][..., 0] - ex)) < 1e-9 * max(1.0, np.abs(ex).max())
    assert np.max(np.abs(c["E"][..., 1] - ey)) < 1e-9 * max(1.0, np.abs(ey).max())
    # velocities after the kick: the kick (v1 - v0) agrees to 1e-2 of its own size
    v0 = np.stack([vx, vy], 1)[keep]
    dk = (c["v"] - v0) - (vel[keep] - v0)
    assert np.linalg.norm(dk) <= 1e-2 * np.linalg.norm(vel[keep] - v0) + 1e-6 * np.linalg.norm(v0)
    assert np.all(c["timing"] >= 0) and c["timing"][3] > 0


def test_update_simulation_repeated_calls(driver, tmp_path, orc):
    """Three calls of two steps each: the state carried through the caller's arrays
    (import / export every call) follows the oracle's six steps."""
    st = _state(seed=9)
    c = _step(driver, tmp_path, st, steps=2, calls=3)
    sim, alive, pos, vel = _oracle_steps(orc, st, 6)
    keep = np.nonzero(alive)[0]
    # a particle grazing a wall may be decided differently after six steps of FP32 state
    assert abs(c["n"] - len(keep)) <= 2
    # the last call's removals: ascending indices into the arrays that call received
    assert c["collided"].size == c["k"] and np.all(np.diff(c["collided"]) > 0)
    assert c["k"] > 0 and c["collided"].max() < c["n"] + c["k"]
    if c["n"] == len(keep):  # same survivor set: same order, positions within a small fraction of a cell
        assert np.array_equal(c["type"], st[4][keep])
        assert np.max(np.abs(c["r"] - pos[keep])) < 1e-4


def test_remove_collided_particles(driver, tmp_path):
    rng = np.random.default_rng(5)
    n = 50_000
    r = rng.random((n, 2))
    r_old = rng.random((n, 2))
    v = rng.standard_normal((n, 2))
    t = rng.integers(0, 3, n).astype(np.int32)
    hits = rng.choice(n, 4_000, replace=False)
    idx = np.concatenate([hits, hits[:100], [-1, n, n + 7]]).astype(np.int32)  # repeats and strays are ignored
    rng.shuffle(idx)
    a, r1, ro1, v1, t1 = compat_io.run(driver, "remove", tmp_path,
                                       [np.array([n], np.int32), r.ravel(), r_old.ravel(), v.ravel(), t, idx],
                                       [np.int32, np.float64, np.float64, np.float64, np.int32])
    keep = np.setdiff1d(np.arange(n), hits)
    assert int(a[0]) == len(keep)
    assert np.array_equal(r1.reshape(-1, 2), r[keep])
    assert np.array_equal(ro1.reshape(-1, 2), r_old[keep])
    assert np.array_equal(v1.reshape(-1, 2), v[keep])
    assert np.array_equal(t1, t[keep])


def test_elastic_collisions(driver, tmp_path):
    rng = np.random.default_rng(6)
    n = 400_000
    m = np.array([9.109e-31, 6.63e-26])
    q = np.array([-1.602e-19, 1.602e-19])
    t = rng.integers(0, 2, n).astype(np.int32)
    speed = np.where(t == 0, 2e6, 2e3) * rng.random(n)
    ang = rng.random(n) * 2 * np.pi
    v = np.stack([speed * np.cos(ang), speed * np.sin(ang)], 1)
    E_tab = np.array([0.0, 1.0, 5.0, 10.0, 20.0])
    s_tab = np.array([1e-20, 2e-20, 1.5e-20, 1e-20, 0.5e-20])
    table = tmp_path / "xs.txt"
    table.write_text("# energy(eV) sigma(m^2)\n\n" + "".join(f"{e} {s}\n" for e, s in zip(E_tab, s_tab)))
    density, dt = 1e21, 2e-9
    outs = []
    for _ in range(2):
        outs.append(compat_io.run(driver, "elastic", tmp_path,
                                  [np.array([1], np.int32), np.array([density, dt]), m, q, v.ravel(), t],
                                  [np.float64] * 6, str(table)))
    v1, vabs, energy, crs, te, ts = outs[0]
    assert np.array_equal(te, E_tab) and np.array_equal(ts, s_tab)  # read_cross_section skips '#' and blank lines
    assert np.array_equal(v1, outs[1][0])  # counter-based random numbers: reproducible
    v1 = v1.reshape(-1, 2)
    s2 = v[:, 0] ** 2 + v[:, 1] ** 2
    np.testing.assert_allclose(vabs, np.sqrt(s2), rtol=1e-15)
    np.testing.assert_allclose(energy, 0.5 * m[t] * s2 * 6.25e18, rtol=1e-14)
    np.testing.assert_allclose(crs, np.interp(energy, E_tab, s_tab), rtol=1e-12, atol=1e-35)
    np.testing.assert_allclose(np.hypot(v1[:, 0], v1[:, 1]), np.sqrt(s2), rtol=1e-12)
    changed = np.any(v1 != v, axis=1)
    P = 1.0 - np.exp(-density * crs * np.sqrt(s2) * dt)
    mu, sd = P.sum(), np.sqrt((P * (1 - P)).sum())
    assert abs(changed.sum() - mu) < 4 * sd, (changed.sum(), mu, sd)
    assert 1000 < mu < n / 2
    # scattering angles are isotropic: mean direction of the scattered set ~ 0
    d = v1[changed] / np.hypot(v1[changed, 0], v1[changed, 1])[:, None]
    assert np.all(np.abs(d.mean(0)) < 5 / np.sqrt(changed.sum()))


def test_solve_multigrid(driver, tmp_path, orc):
    n, h = 257, 1.0 / 256
    rng = np.random.default_rng(8)
    rho = rng.standard_normal((n, n))
    phi0 = np.zeros((n, n))
    phi0[0, :] = 1.0  # Dirichlet data carried by phi's boundary
    phi0[:, -1] = np.linspace(1.0, -1.0, n)
    (phi,) = compat_io.run(driver, "solve", tmp_path,
                           [np.array([n, 5], np.int32), np.array([h, 1.25]), phi0.ravel(), rho.ravel()], [np.float64])
    phi = phi.reshape(n, n)
    for sl in (np.s_[0, :], np.s_[-1, :], np.s_[:, 0], np.s_[:, -1]):
        assert np.array_equal(phi[sl], phi0[sl])
    assert orc.relres(phi, rho, h) < 1e-5
    ref, _, _ = orc.mg_solve(phi0, rho, h, levels=5, omega=1.25, nu1=3, nu2=3, nuc=20, tol=1e-12, max_cycles=200)
    assert rel_l2(phi, ref) < 1e-3


def test_reference_kernel_wrappers(driver, tmp_path, orc):
    """kernels.cuh / collisions.cuh host wrappers, run in main.cu's order, against the oracle."""
    rng = np.random.default_rng(11)
    n, gm, dt = 60_000, 65, 0.02
    dx = 1.0 / (gm - 1)
    x, y = rng.random(n) * 1.04 - 0.02, rng.random(n) * 1.04 - 0.02  # a few start outside the grid
    vx, vy = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    t = rng.integers(0, 2, n).astype(np.int32)
    # moves that touch a wall end point exactly, or run along a wall, are in the set
    x[:4], y[:4] = [0.25, 0.1, 0.5, 0.75], [0.2, 0.25, 0.25, 0.1]
    vx[:4], vy[:4] = [0.0, 7.5, 0.0, 0.0], [2.5, 0.0, 0.0, 5.0]
    phi = rng.standard_normal((gm, gm))
    E_tab, s_tab = np.array([0.0, 0.5, 2.0, 8.0]), np.array([3e-20, 2e-20, 1e-20, 4e-21])
    out = compat_io.run(driver, "kernels", tmp_path,
                        [np.array([gm], np.int32), np.array([dx, dt]), np.array(Q), np.array(M),
                         np.array(WALLS, float).ravel(), np.stack([x, y], 1).ravel(), np.stack([vx, vy], 1).ravel(),
                         t, phi.ravel(), E_tab, s_tab],
                        [np.float64] * 2 + [np.int32] + [np.float64] * 6 + [np.float32])
    r, r_old, hits, rho, E, v, vabs, energy, crs, fpos = out
    r, r_old, v, E = r.reshape(-1, 2), r_old.reshape(-1, 2), v.reshape(-1, 2), E.reshape(gm, gm, 2)
    x1, y1 = orc.drift(x, y, vx, vy, dt)
    assert np.array_equal(r[:, 0], x1) and np.array_equal(r[:, 1], y1)
    assert np.array_equal(r_old[:, 0], x) and np.array_equal(r_old[:, 1], y)
    ref_hit = orc.walls_segments(x, y, x1, y1, WALLS)
    assert np.array_equal(np.sort(hits), np.nonzero(ref_hit)[0])
    assert len(np.unique(hits)) == len(hits)
    rho_o = orc.deposit(x1, y1, np.array(Q)[t], gm, gm, dx, dx)
    assert rel_l2(rho.reshape(gm, gm), rho_o) < 1e-13
    ex, ey = orc.efield(phi, dx, dx)
    assert np.max(np.abs(E[..., 0] - ex)) < 1e-12 * np.abs(ex).max()
    assert np.max(np.abs(E[..., 1] - ey)) < 1e-12 * np.abs(ey).max()
    kvx, kvy = orc.kick(x1, y1, vx, vy, np.array(Q)[t], np.array(M)[t], ex, ey, dx, dx, dt)
    np.testing.assert_allclose(v[:, 0], kvx, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(v[:, 1], kvy, rtol=1e-12, atol=1e-13)
    s2 = v[:, 0] ** 2 + v[:, 1] ** 2
    np.testing.assert_allclose(vabs, np.sqrt(s2), rtol=1e-15)
    np.testing.assert_allclose(energy, 0.5 * np.array(M)[t] * s2 * 6.25e18, rtol=1e-14)
    np.testing.assert_allclose(crs, np.interp(energy, E_tab, s_tab), rtol=1e-12, atol=1e-35)
    assert np.array_equal(fpos.reshape(-1, 2), r.astype(np.float32))
