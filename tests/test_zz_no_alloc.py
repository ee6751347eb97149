"""pic_solve_multigrid_f64_static (working memory compiled into the library, no device
allocation) against pic_solve_multigrid_f64, called through the C ABI.  Collected last, so
it also runs after every other test in the same process."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2
from pic_cuda_b200 import _lib as L

pytestmark = pytest.mark.gpu

OMEGA, NU_PRE, NU_POST, NU_COARSE, TOL, MAX_CYCLES = 1.25, 3, 3, 20, 1e-9, 60


def _solve(name, phi, rho, n, h, levels=0):
    import torch
    torch.cuda.synchronize()
    cyc, rel = C.c_int(), C.c_double()
    rc = getattr(L.lib(), name)(C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()), n, n, levels, h, OMEGA,
                                NU_PRE, NU_POST, NU_COARSE, TOL, MAX_CYCLES, None, C.byref(cyc), C.byref(rel))
    torch.cuda.synchronize()
    return rc, cyc.value, rel.value


def _problem(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    rho = rng.standard_normal((n, n))
    phi0 = np.zeros((n, n))
    phi0[0, :] = 1.0  # Dirichlet data on the boundary of phi
    phi0[:, -1] = np.linspace(1.0, -1.0, n)
    return torch.tensor(phi0, device="cuda"), torch.tensor(rho, device="cuda")


@pytest.mark.parametrize("n", [33, 129, 257])
def test_static_solver_matches_allocating_solver_twice(n):
    h = 1.0 / (n - 1)
    for seed in (1, 2):  # two calls in a row, different right-hand sides
        phi_a, rho = _problem(n, seed)
        phi_b = phi_a.clone()
        rc_a, cyc_a, rel_a = _solve("pic_solve_multigrid_f64", phi_a, rho, n, h)
        rc_b, cyc_b, rel_b = _solve("pic_solve_multigrid_f64_static", phi_b, rho, n, h)
        assert rc_a == L.PIC_OK and rc_b == L.PIC_OK, (rc_a, rc_b, L.lib().pic_last_error())
        assert rel_a < TOL and rel_b < TOL
        assert abs(cyc_a - cyc_b) <= 1
        a, b = phi_a.cpu().numpy(), phi_b.cpu().numpy()
        assert rel_l2(b, a) < 1e-7
        assert np.array_equal(b[0, :], a[0, :]) and np.array_equal(b[:, -1], a[:, -1])


def test_static_solver_rejects_grid_beyond_scratch():
    import torch
    n = 513
    phi = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    rho = torch.zeros_like(phi)
    rc, _, _ = _solve("pic_solve_multigrid_f64_static", phi, rho, n, 1.0 / (n - 1))
    assert rc == L.PIC_ERR_ARG
    assert b"257" in L.lib().pic_last_error()


@pytest.mark.parametrize("n", [3, 5])
def test_static_solver_smallest_grids(n):
    """One- and two-level grids (one and nine interior nodes) give the allocating solver's
    result."""
    h = 1.0 / (n - 1)
    phi_a, rho = _problem(n, 11)
    phi_b = phi_a.clone()
    rc_a, cyc_a, rel_a = _solve("pic_solve_multigrid_f64", phi_a, rho, n, h)
    rc_b, cyc_b, rel_b = _solve("pic_solve_multigrid_f64_static", phi_b, rho, n, h)
    assert rc_a == L.PIC_OK and rc_b == L.PIC_OK, (rc_a, rc_b, L.lib().pic_last_error())
    assert abs(cyc_a - cyc_b) <= 1
    assert rel_l2(phi_b.cpu().numpy(), phi_a.cpu().numpy()) < 1e-7


@pytest.mark.parametrize("n,levels", [(65, 2), (257, 3)])
def test_static_solver_partial_hierarchies(n, levels):
    """Hierarchies cut short of 3 x 3 (the coarsest level only smoothed, so a V-cycle
    contracts slowly): six V-cycles of each solver give the same potential."""
    import torch
    h = 1.0 / (n - 1)
    phi_a, rho = _problem(n, 11)
    phi_b = phi_a.clone()
    out = []
    for name, phi in (("pic_solve_multigrid_f64", phi_a), ("pic_solve_multigrid_f64_static", phi_b)):
        torch.cuda.synchronize()
        cyc, rel = C.c_int(), C.c_double()
        rc = getattr(L.lib(), name)(C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()), n, n, levels, h, OMEGA,
                                    NU_PRE, NU_POST, NU_COARSE, 0.0, 6, None, C.byref(cyc), C.byref(rel))
        torch.cuda.synchronize()
        out.append((rc, cyc.value, rel.value))
    assert out[0][0] == out[1][0] == L.PIC_ERR_NOT_CONVERGED and out[0][1] == out[1][1] == 6
    assert abs(out[0][2] - out[1][2]) <= 1e-6 * out[0][2] + 1e-12
    assert rel_l2(phi_b.cpu().numpy(), phi_a.cpu().numpy()) < 1e-7


def test_static_solver_fixed_cycle_budget_reports_not_converged():
    """tol = 0 runs exactly max_cycles V-cycles and returns PIC_ERR_NOT_CONVERGED, as the
    allocating solver does, with the same potential."""
    import torch
    n, cycles = 129, 4
    h = 1.0 / (n - 1)
    phi_a, rho = _problem(n, 5)
    phi_b = phi_a.clone()
    out = []
    for name, phi in (("pic_solve_multigrid_f64", phi_a), ("pic_solve_multigrid_f64_static", phi_b)):
        torch.cuda.synchronize()
        cyc, rel = C.c_int(), C.c_double()
        rc = getattr(L.lib(), name)(C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()), n, n, 0, h, OMEGA,
                                    NU_PRE, NU_POST, NU_COARSE, 0.0, cycles, None, C.byref(cyc), C.byref(rel))
        torch.cuda.synchronize()
        out.append((rc, cyc.value, rel.value))
    assert out[0][0] == L.PIC_ERR_NOT_CONVERGED and out[1][0] == L.PIC_ERR_NOT_CONVERGED
    assert out[0][1] == cycles and out[1][1] == cycles
    assert rel_l2(phi_b.cpu().numpy(), phi_a.cpu().numpy()) < 1e-7


def test_static_solver_allocates_no_device_memory():
    """After a first call (which looks up the array's address), a second call leaves the
    device's free memory exactly as it was: nothing is allocated or freed."""
    import torch
    n = 257
    h = 1.0 / (n - 1)
    phi, rho = _problem(n, 3)
    rc, _, _ = _solve("pic_solve_multigrid_f64_static", phi.clone(), rho, n, h)
    assert rc == L.PIC_OK
    work = phi.clone()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, _, _ = _solve("pic_solve_multigrid_f64_static", work, rho, n, h)
    free1, _ = torch.cuda.mem_get_info()
    assert rc == L.PIC_OK
    assert free1 == free0


def test_both_solvers_apply_the_same_argument_limits():
    """Arguments outside the solvers' limits give PIC_ERR_ARG from both entry points, before
    any launch."""
    import torch
    n = 33
    phi, rho = _problem(n, 1)
    bad = [dict(omega=2.0), dict(omega=0.0), dict(nu_pre=17), dict(nu_post=-1), dict(nu_coarse=1001),
           dict(max_cycles=0), dict(tol=-1.0), dict(levels=9)]
    for b in bad:
        a = dict(levels=0, omega=OMEGA, nu_pre=NU_PRE, nu_post=NU_POST, nu_coarse=NU_COARSE, tol=TOL,
                 max_cycles=MAX_CYCLES)
        a.update(b)
        for name in ("pic_solve_multigrid_f64", "pic_solve_multigrid_f64_static"):
            cyc, rel = C.c_int(), C.c_double()
            rc = getattr(L.lib(), name)(C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()), n, n, a["levels"],
                                        1.0 / (n - 1), a["omega"], a["nu_pre"], a["nu_post"], a["nu_coarse"],
                                        a["tol"], a["max_cycles"], None, C.byref(cyc), C.byref(rel))
            assert rc == L.PIC_ERR_ARG, (name, b, rc)
    torch.cuda.synchronize()
