"""The FP64 oracle reproduces outputs of the reference's own CUDA kernels (CPU only).

Fixtures in tests/golden/ were produced by tests/golden/make_golden.py, which runs the
reference's kernels (compiled from its sources by oracle/Makefile into oracle/_ref) on a
B200; they hold the seeded inputs and the reference's outputs.
"""
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2

G = Path(__file__).resolve().parent / "golden"


def load(name):
    p = G / name
    if not p.exists():
        pytest.fail(f"missing fixture {p}: run tests/golden/make_golden.py on a GPU")
    return np.load(p)


def test_golden_deposit(orc):
    d = load("ref_deposit.npz")
    rho = orc.deposit(d["x"], d["y"], d["q"][d["type"]], int(d["m"]), int(d["n"]), float(d["dx"]), float(d["dx"]))
    assert rel_l2(rho, d["rho"]) < 1e-13


@pytest.mark.parametrize("name", ["ref_solve_65.npz", "ref_solve_129.npz"])
def test_golden_solve(orc, name):
    d = load(name)
    phi, cyc, _ = orc.mg_solve(d["phi0"], d["f"], float(d["h"]), levels=int(d["levels"]), omega=1.25, nu1=3, nu2=3,
                               nuc=20, tol=1e-5, max_cycles=50, ref_convergence=True)
    assert rel_l2(phi, d["phi"]) < 1e-11
    assert np.array_equal(phi[0, :], d["phi"][0, :])  # Dirichlet row carried by phi


def test_golden_efield(orc):
    d = load("ref_efield.npz")
    ex, ey = orc.efield(d["phi"], float(d["dx"]), float(d["dy"]))
    assert np.max(np.abs(ex - d["ex"])) < 1e-12 and np.max(np.abs(ey - d["ey"])) < 1e-12


def test_golden_full_step(orc):
    from pic_cuda_b200 import _lib as L
    from pic_cuda_b200 import configs as cf
    d = load("ref_step.npz")
    q, m = d["q"], d["mass"]
    walls = d["walls"]
    dt = float(d["dt"])
    cfg = cf.make_config(int(d["m"]), 1.0, dt, [(q[0], m[0], 1.0, 8000), (q[1], m[1], 1.0, 8000)],
                         units=L.UNITS_REF, walls=L.WALLS_SEGMENTS, wall_segments=walls.tolist(), levels=5,
                         omega=1.25, nu_pre=3, nu_post=3, nu_coarse=20, tol=1e-5)
    # the absorbed set of the first drift equals the reference's hit list
    hit = orc.walls_segments(d["x"], d["y"], d["x"] + d["vx"] * dt, d["y"] + d["vy"] * dt, walls, ref_epsilon=True)
    assert np.array_equal(np.nonzero(hit)[0], d["hits"])
    sim = orc.Sim(cfg)
    for s in (0, 1):
        sel = d["type"] == s
        sim.load(s, d["x"][sel], d["y"][sel], d["vx"][sel], d["vy"][sel])
    orc.set_reference_convergence(True)
    try:
        sim.step(1)
    finally:
        orc.set_reference_convergence(False)
    assert rel_l2(sim.grid(L.GRID_RHO), d["rho1"]) < 1e-13
    assert rel_l2(sim.grid(L.GRID_PHI), d["phi1"]) < 1e-11
    for s in (0, 1):
        o = sim.export(s)
        sel = d["type1"] == s
        assert sel.sum() == len(o["x"])
        a = np.lexsort((d["y1"][sel], d["x1"][sel]))
        b = np.lexsort((o["y"], o["x"]))
        np.testing.assert_allclose(o["x"][b], d["x1"][sel][a], rtol=0, atol=1e-14)
        np.testing.assert_allclose(o["vx"][b], d["vx1"][sel][a], rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(o["vy"][b], d["vy1"][sel][a], rtol=1e-10, atol=1e-14)


def test_golden_embedded_kernels(orc):
    """The kernels of Multigrid_embedded.cu on one seeded rectangular level (65 x 49, an
    electrode with edges on odd and even nodes, a solid block): smooth_redblack with
    redblack = 0 (the colour whose test evaluates as intended), residual_kernel,
    restrict_kernel (coarse rhs and injected coarse kinds) and prolongate_add_kernel."""
    d = load("ref_embedded.npz")
    h2 = float(d["h2"])
    s0 = orc.emb_half_sweep(d["phi"], d["rhs"], d["mask"], d["bc"], h2, 0)
    assert rel_l2(s0, d["phi_sweep0"]) < 1e-14
    res = orc.emb_residual(d["phi"], d["rhs"], d["mask"], 1.0 / h2)
    assert rel_l2(res, d["res"]) < 1e-13
    rc, mc = orc.emb_restrict(d["res"], d["mask"])
    assert np.array_equal(mc, d["mask_c"])
    assert rel_l2(rc, d["rhs_c"]) < 1e-14
    assert np.array_equal(orc.emb_prolong(d["phi_c"], d["phi"], d["mask"]), d["phi_prol"])
