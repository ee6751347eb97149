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
