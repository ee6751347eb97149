"""ctypes wrapper of oracle/_ref/libpicref.so: the reference's own CUDA kernels compiled from
its sources by oracle/Makefile and driven headless by oracle/ref_harness.cu.

TEST INFRASTRUCTURE ONLY (used to pin the oracle and to time the reference's CUDA step).
It needs a GPU; available() is False when the library was not built or no device exists.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libpicref.so"
_lib = None
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB))
        L.refh_device_ok.restype = C.c_int
        L.refh_deposit.argtypes = [C.c_int, _D, _D, _I, _D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _D]
        L.refh_solve.argtypes = [_D, _D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
        L.refh_efield.argtypes = [_D, C.c_int, C.c_int, C.c_double, C.c_double, _D]
        L.refh_steps.argtypes = [C.c_int, C.c_int, _D, _D, _D, _D, _I, _D, _D, C.c_int, C.c_int, C.c_int, C.c_double,
                                 C.c_double, _D, C.c_int, C.c_double, _D, _D, _D, _I, _I, _I,
                                 C.POINTER(C.c_float)]
        L.refh_elastic.argtypes = [C.c_int, _D, _D, C.c_double, C.c_double, C.c_double, _D, _D, C.c_int]
        _U8 = C.POINTER(C.c_uint8)
        L.refh_emb_kernels.argtypes = [C.c_int, C.c_int, _D, _D, _U8, _D, C.c_double, _D, _D, _D, _D, _U8, _D]
        L.refh_emb_vcycles.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, _D, _D, _U8, _D,
                                       C.POINTER(C.c_float)]
        L.refh_particle_kernels_timed.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _D,
                                                  _D, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_float)]
        _lib = L
    return _lib


def available() -> bool:
    if not LIB.exists():
        return False
    try:
        return bool(lib().refh_device_ok())
    except OSError:
        return False


def _d(a):
    return a.ctypes.data_as(_D)


def deposit(x, y, types, qtab, m, n, dx, dy):
    x, y = np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64)
    t = np.ascontiguousarray(types, np.int32)
    q = np.ascontiguousarray(qtab, np.float64)
    rho = np.zeros(m * n)
    rc = lib().refh_deposit(len(x), _d(x), _d(y), t.ctypes.data_as(_I), _d(q), len(q), m, n, dx, dy, _d(rho))
    assert rc == 0
    return rho.reshape(n, m)


def solve(phi, rho, h, levels=5, omega=1.25):
    phi = np.ascontiguousarray(phi, np.float64).copy()
    rho = np.ascontiguousarray(rho, np.float64)
    ny, nx = phi.shape
    assert lib().refh_solve(_d(phi), _d(rho), nx, ny, levels, h, omega) == 0
    return phi


def efield(phi, dx, dy):
    phi = np.ascontiguousarray(phi, np.float64)
    n, m = phi.shape
    e = np.empty(2 * m * n)
    assert lib().refh_efield(_d(phi), m, n, dx, dy, _d(e)) == 0
    e = e.reshape(n, m, 2)
    return e[..., 0].copy(), e[..., 1].copy()


def steps(nsteps, x, y, vx, vy, types, q, mass, m, n, X, Y, walls, dt, phi=None):
    """Re-sequenced updateSimulationCUDA (main.cu:60-135); returns the state after nsteps."""
    N = len(x)
    x, y = np.array(x, np.float64), np.array(y, np.float64)
    vx, vy = np.array(vx, np.float64), np.array(vy, np.float64)
    t = np.array(types, np.int32)
    q, mass = np.ascontiguousarray(q, np.float64), np.ascontiguousarray(mass, np.float64)
    w = np.ascontiguousarray(walls, np.float64).reshape(-1)
    ph = np.zeros(m * n) if phi is None else np.ascontiguousarray(phi, np.float64).reshape(-1).copy()
    rho, exy = np.zeros(m * n), np.zeros(2 * m * n)
    hits = np.zeros(max(N, 1), np.int32)
    nh, na = C.c_int(0), C.c_int(0)
    ms = C.c_float(0)
    rc = lib().refh_steps(nsteps, N, _d(x), _d(y), _d(vx), _d(vy), t.ctypes.data_as(_I), _d(q), _d(mass), len(q), m,
                          n, X, Y, _d(w) if len(w) else None, len(w) // 4, dt, _d(ph), _d(rho), _d(exy),
                          hits.ctypes.data_as(_I), C.byref(nh), C.byref(na), C.byref(ms))
    assert rc == 0
    k = na.value
    return {"x": x[:k], "y": y[:k], "vx": vx[:k], "vy": vy[:k], "type": t[:k], "phi": ph.reshape(n, m),
            "rho": rho.reshape(n, m), "E": exy.reshape(n, m, 2), "hits": hits[: nh.value].copy(),
            "n_alive": k, "ms_per_step": ms.value}


def elastic(vx, vy, mass, density, dt, xs_e, xs_s):
    vx, vy = np.array(vx, np.float64), np.array(vy, np.float64)
    e, s = np.ascontiguousarray(xs_e, np.float64), np.ascontiguousarray(xs_s, np.float64)
    assert lib().refh_elastic(len(vx), _d(vx), _d(vy), mass, density, dt, _d(e), _d(s), len(e)) == 0
    return vx, vy


def emb_kernels(phi, rhs, mask, bc, h2, phi_c):
    """The kernels of Multigrid_embedded.cu on one level: smooth_redblack(redblack=0),
    residual_kernel, restrict_kernel of that residual, prolongate_add_kernel of phi_c."""
    phi, rhs, bc = (np.ascontiguousarray(a, np.float64) for a in (phi, rhs, bc))
    mask = np.ascontiguousarray(mask, np.uint8)
    phi_c = np.ascontiguousarray(phi_c, np.float64)
    ny, nx = phi.shape
    nyc, nxc = phi_c.shape
    assert (nxc, nyc) == ((nx - 1) // 2 + 1, (ny - 1) // 2 + 1)
    u8 = C.POINTER(C.c_uint8)
    out = {"phi_sweep0": np.empty_like(phi), "res": np.empty_like(phi), "rhs_c": np.empty((nyc, nxc)),
           "mask_c": np.empty((nyc, nxc), np.uint8), "phi_prol": np.empty_like(phi)}
    rc = lib().refh_emb_kernels(nx, ny, _d(phi), _d(rhs), mask.ctypes.data_as(u8), _d(bc), h2, _d(phi_c),
                                _d(out["phi_sweep0"]), _d(out["res"]), _d(out["rhs_c"]),
                                out["mask_c"].ctypes.data_as(u8), _d(out["phi_prol"]))
    assert rc == 0
    return out


def emb_vcycles_timed(phi, rhs, mask, bc, h, levels, cycles, warmup=2):
    """Multigrid::vcycle re-sequenced on the reference's kernels; returns (phi, ms per V-cycle)."""
    phi = np.ascontiguousarray(phi, np.float64).copy()
    rhs, bc = np.ascontiguousarray(rhs, np.float64), np.ascontiguousarray(bc, np.float64)
    mask = np.ascontiguousarray(mask, np.uint8)
    ny, nx = phi.shape
    ms = C.c_float(0)
    rc = lib().refh_emb_vcycles(nx, ny, levels, h, warmup, cycles, _d(phi), _d(rhs),
                                mask.ctypes.data_as(C.POINTER(C.c_uint8)), _d(bc), C.byref(ms))
    assert rc == 0
    return phi, ms.value


def particle_kernels_timed(n, m, nn, X, Y, dt, q, mass, vmax, iters=5):
    """The reference's four particle kernels of a step (update_coordinates, memsets +
    detect_intersections, rho memset + updateDensity, updateParticleVelocities) on n
    particles of its FP64 AoS state, each timed with CUDA events; ms per launch in that order."""
    q = np.ascontiguousarray(q, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    ms = (C.c_float * 4)()
    rc = lib().refh_particle_kernels_timed(n, m, nn, X, Y, dt, _d(q), _d(mass), vmax[0], vmax[1], iters, ms)
    assert rc == 0
    return list(ms)
