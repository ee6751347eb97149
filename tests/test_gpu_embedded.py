"""Embedded-boundary multigrid (Multigrid_embedded.cu) on the GPU against the FP64 oracle:
pic_solve_embedded_f64 V-cycle by V-cycle on square and rectangular grids, every option, the
one-CTA and tile paths and the sweep-count chunking; the drop-in Multigrid class of
include/compat/Multigrid_embedded.hpp from a C++ program.  Tolerance: 1e-12 relative L2 per
V-cycle (FP64 throughout; only the contraction of a multiply-add into an FMA differs)."""
import numpy as np
import pytest

import compat_io
from conftest import rel_l2
from pic_cuda_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-12


def problem(nx, ny, seed=0, electrode=True, solid=True):
    """Random right-hand side and initial guess, an electrode at 2.5 whose edges fall on odd
    and even nodes, a solid block, 0.3 on one boundary row."""
    rng = np.random.default_rng(seed)
    mask = np.zeros((ny, nx), np.uint8)
    if electrode:
        mask[ny // 4: ny // 2, nx // 4: nx // 2 + 1] = L.NODE_DIRICHLET
    if solid:
        mask[3 * ny // 5: 3 * ny // 4, 3 * nx // 5: 4 * nx // 5] = L.NODE_SOLID
    bc = np.where(mask == L.NODE_DIRICHLET, 2.5, 0.0)
    rhs = rng.standard_normal((ny, nx))
    phi = 0.1 * rng.standard_normal((ny, nx))
    phi[0, :] = 0.3
    return phi, rhs, mask, bc


def gpu_cycles(phi, rhs, mask, bc, h, levels, cycles, nu=(2, 2), options=0):
    import torch
    from pic_cuda_b200.engine import solve_embedded_f64
    d = [torch.tensor(a, device="cuda") for a in (phi, rhs)]
    dm = torch.tensor(mask, device="cuda")
    dbc = torch.tensor(bc, device="cuda") if bc is not None else None
    cyc, rel, ok = solve_embedded_f64(d[0], d[1], dm, dbc, levels, h, nu[0], nu[1], options, tol=0.0,
                                      max_cycles=cycles)
    assert cyc == cycles and not ok
    return d[0].cpu().numpy()


@pytest.mark.parametrize("nx,ny,levels", [(33, 33, 4), (65, 65, 6), (129, 129, 7), (257, 193, 5), (513, 513, 9),
                                          (1025, 1025, 6)])
@pytest.mark.parametrize("options", [0, L.EMB_COARSEN_ANY, L.EMB_COARSEN_ANY | L.EMB_PROLONG_BILINEAR])
def test_vcycles_match_oracle(orc, nx, ny, levels, options):
    h = 1.0 / (nx - 1)
    phi, rhs, mask, bc = problem(nx, ny, seed=nx + options)
    for cycles in (1, 3):
        got = gpu_cycles(phi, rhs, mask, bc, h, levels, cycles, options=options)
        ref = orc.emb_vcycles(phi, rhs, mask, bc, h, levels, cycles, options=options)
        assert rel_l2(got, ref) < TOL, (cycles, rel_l2(got, ref))
        assert np.all(got[mask == L.NODE_DIRICHLET] == 2.5)
        assert np.array_equal(got[mask == L.NODE_SOLID], phi[mask == L.NODE_SOLID])
        assert np.array_equal(got[0, :], phi[0, :]) and np.array_equal(got[:, -1], phi[:, -1])


@pytest.mark.parametrize("nu", [(1, 3), (5, 0), (0, 2), (6, 9)])
def test_sweep_counts_and_chunking(orc, nu):
    """nu above 4 runs as several tile launches; nu_post = 0 as a prolongation-only launch."""
    nx = ny = 257
    h = 1.0 / (nx - 1)
    phi, rhs, mask, bc = problem(nx, ny, seed=7)
    got = gpu_cycles(phi, rhs, mask, bc, h, 6, 2, nu=nu, options=L.EMB_COARSEN_ANY)
    ref = orc.emb_vcycles(phi, rhs, mask, bc, h, 6, 2, nu1=nu[0], nu2=nu[1], options=L.EMB_COARSEN_ANY)
    assert rel_l2(got, ref) < TOL


def test_without_phi_bc_electrodes_keep_phi(orc):
    nx = ny = 129
    h = 1.0 / (nx - 1)
    phi, rhs, mask, _ = problem(nx, ny, seed=3)
    phi[mask == L.NODE_DIRICHLET] = -1.25
    got = gpu_cycles(phi, rhs, mask, None, h, 7, 2, options=L.EMB_COARSEN_ANY)
    ref = orc.emb_vcycles(phi, rhs, mask, None, h, 7, 2, options=L.EMB_COARSEN_ANY)
    assert rel_l2(got, ref) < TOL
    assert np.all(got[mask == L.NODE_DIRICHLET] == -1.25)


@pytest.mark.parametrize("nx,ny,levels", [(257, 257, 8), (513, 385, 9)])
def test_solve_to_tolerance(orc, nx, ny, levels):
    """A charged problem to 1e-10 and a Laplace problem driven by the electrode alone (rhs = 0
    on FLUID nodes: the residual is measured against the initial one) to 1e-8.  The reference's
    V-cycle (two sweeps on the coarsest level, electrodes that grow on every coarser level)
    contracts slowly on these geometries, hence the cycle budget."""
    import torch
    from pic_cuda_b200.engine import solve_embedded_f64
    h = 1.0 / (nx - 1)
    opts = L.EMB_COARSEN_ANY | L.EMB_PROLONG_BILINEAR
    for charged, tol in ((True, 1e-10), (False, 1e-8)):
        phi, rhs, mask, bc = problem(nx, ny, seed=11)
        phi[:] = 0.0
        if not charged:
            rhs[:] = 0.0
        d = torch.tensor(phi, device="cuda")
        cyc, rel, ok = solve_embedded_f64(d, torch.tensor(rhs, device="cuda"), torch.tensor(mask, device="cuda"),
                                          torch.tensor(bc, device="cuda"), levels, h, 2, 2, opts, tol=tol,
                                          max_cycles=300)
        assert ok and rel < tol
        got = d.cpu().numpy()
        ref, rcyc, rrel = orc.emb_solve(phi, rhs, mask, bc, h, levels, tol=tol, max_cycles=300, options=opts)
        assert abs(cyc - rcyc) <= 1
        assert rel_l2(got, ref) < 1e-9
        if not charged:   # discrete maximum principle between the grounded walls and the electrode
            assert got.min() >= -1e-9 and got.max() <= 2.5 + 1e-9


def test_reference_operators_diverge_on_odd_electrode_edges(orc):
    """With the reference's transfer operators an electrode edge on an odd node makes the
    coarse electrode smaller than the fine one, and the V-cycle diverges at 257^2; the
    solver reports it instead of returning a wrong potential."""
    import torch
    from pic_cuda_b200.engine import solve_embedded_f64
    nx = ny = 257
    h = 1.0 / (nx - 1)
    phi, rhs, mask, bc = problem(nx, ny, seed=5)
    d = torch.tensor(phi, device="cuda")
    cyc, rel, ok = solve_embedded_f64(d, torch.tensor(rhs, device="cuda"), torch.tensor(mask, device="cuda"),
                                      torch.tensor(bc, device="cuda"), 8, h, 2, 2, 0, tol=1e-10, max_cycles=30)
    assert not ok and cyc == 30 and rel > 1.0


def test_argument_errors():
    import torch
    from pic_cuda_b200.engine import solve_embedded_f64
    a = torch.zeros((9, 9), dtype=torch.float64, device="cuda")
    m = torch.zeros((9, 9), dtype=torch.uint8, device="cuda")
    with pytest.raises(RuntimeError):
        solve_embedded_f64(a, a, m, None, 0, 0.1)
    with pytest.raises(RuntimeError):
        solve_embedded_f64(a, a, m, None, 2, 0.1, options=8)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    return compat_io.build_driver(tmp_path_factory.mktemp("compat_emb"))


@pytest.mark.parametrize("nx,ny,levels", [(65, 65, 5), (257, 129, 6)])
def test_compat_multigrid_class(driver, tmp_path, orc, nx, ny, levels):
    """The reference's class, filled and cycled as its vcycle is written to be used."""
    h = 1.0 / (nx - 1)
    phi, rhs, mask, bc = problem(nx, ny, seed=21)
    cycles = 3
    out = compat_io.run(driver, "embedded", tmp_path,
                        [np.array([nx, ny, levels, cycles], np.int32), np.array([h]), phi, rhs, bc, mask],
                        [np.float64, np.float64, np.uint8])
    got = out[0].reshape(ny, nx)
    ref = orc.emb_vcycles(phi, rhs, mask, bc, h, levels, cycles)
    assert rel_l2(got, ref) < TOL
    # level 1 holds the restriction of the last cycle's level-0 residual, as in the reference
    nxc, nyc = orc.emb_coarse_shape(nx, ny)
    pre = orc.emb_vcycles(phi, rhs, mask, bc, h, levels, cycles - 1)
    for _ in range(2):
        pre = orc.emb_half_sweep(pre, rhs, mask, bc, h * h, 0)
        pre = orc.emb_half_sweep(pre, rhs, mask, bc, h * h, 1)
    rc, mc = orc.emb_restrict(orc.emb_residual(pre, rhs, mask, 1.0 / (h * h)), mask)
    assert np.array_equal(out[2].reshape(nyc, nxc), mc)
    assert rel_l2(out[1].reshape(nyc, nxc), rc) < TOL
