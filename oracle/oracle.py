"""ctypes wrapper of liboracle.so — the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm use this
module; the product (pic_cuda_b200) never imports it.  See pic_oracle.cpp for the
reference file:line each function restates.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None

_D = C.POINTER(C.c_double)
_U8 = C.POINTER(C.c_uint8)
_U32 = C.POINTER(C.c_uint32)
_I64 = C.c_int64


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        sig = {
            "orc_philox4x32_10": (None, [_U32, _U32, _U32]),
            "orc_u01": (C.c_double, [C.c_uint32]),
            "orc_drift": (None, [_I64, _D, _D, _D, _D, _D, _D, C.c_double]),
            "orc_walls_segments_ref": (None, [_I64, _D, _D, _D, _D, _D, C.c_int, _U8]),
            "orc_walls_segments": (None, [_I64, _D, _D, _D, _D, _D, C.c_int, _U8]),
            "orc_walls_box": (None, [_I64, _D, _D, C.c_int, C.c_int, C.c_double, C.c_double, _U8]),
            "orc_deposit": (None, [_I64, _D, _D, _D, C.c_int, C.c_int, C.c_double, C.c_double, _D]),
            "orc_efield": (None, [_D, C.c_int, C.c_int, C.c_double, C.c_double, _D, _D]),
            "orc_kick": (None, [_I64, _D, _D, _D, _D, _D, _D, _D, _D, C.c_int, C.c_int, C.c_double, C.c_double,
                                C.c_double]),
            "orc_mg_solve": (C.c_int, [_D, _D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                       C.c_int, C.c_double, C.c_int, _D]),
            "orc_mg_vcycles": (None, [_D, _D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                      C.c_int, C.c_int]),
            "orc_relres": (C.c_double, [_D, _D, C.c_int, C.c_int, C.c_double]),
            "orc_set_reference_convergence": (None, [C.c_int]),
            "orc_residual": (None, [_D, _D, _D, C.c_int, C.c_int, C.c_double]),
            "orc_auto_levels": (C.c_int, [C.c_int, C.c_int]),
            "orc_sim_create": (C.c_void_p, [C.c_void_p]),
            "orc_sim_destroy": (None, [C.c_void_p]),
            "orc_sim_numax": (C.c_double, [C.c_void_p, C.c_int]),
            "orc_sim_load": (None, [C.c_void_p, C.c_int, _I64, _D, _D, _D, _D, _D, _U32]),
            "orc_sim_count": (_I64, [C.c_void_p, C.c_int]),
            "orc_sim_export": (None, [C.c_void_p, C.c_int, _D, _D, _D, _D, _D, _U32]),
            "orc_sim_get_grid": (None, [C.c_void_p, C.c_int, _D]),
            "orc_sim_set_grid": (None, [C.c_void_p, C.c_int, _D]),
            "orc_sim_set_counters": (None, [C.c_void_p, _I64, C.c_uint32]),
            "orc_sim_stats": (None, [C.c_void_p, C.POINTER(_I64), C.POINTER(C.c_int), _D, C.POINTER(_I64),
                                     C.POINTER(_I64), C.POINTER(_I64)]),
            "orc_sim_drift_walls": (None, [C.c_void_p]),
            "orc_sim_deposit": (None, [C.c_void_p]),
            "orc_sim_solve": (None, [C.c_void_p]),
            "orc_sim_kick": (None, [C.c_void_p]),
            "orc_sim_mcc": (None, [C.c_void_p]),
            "orc_sim_step": (None, [C.c_void_p, C.c_int]),
            "orc_sim_total_charge": (C.c_double, [C.c_void_p]),
            "orc_num_threads": (C.c_int, []),
            "orc_emb_half_sweep": (None, [_D, _D, _U8, _D, C.c_int, C.c_int, C.c_double, C.c_int]),
            "orc_emb_residual": (None, [_D, _D, _D, _U8, C.c_int, C.c_int, C.c_double]),
            "orc_emb_restrict": (None, [_D, _D, _U8, _U8, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_emb_prolong": (None, [_D, _D, _U8, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_emb_vcycles": (None, [_D, _D, _U8, _D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                       C.c_int, C.c_int]),
            "orc_emb_solve": (C.c_int, [_D, _D, _U8, _D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                        C.c_int, C.c_double, C.c_int, _D]),
            "orc_emb_norms": (None, [_D, _D, _U8, C.c_int, C.c_int, C.c_double, _D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_D)


def f64(a):
    return np.ascontiguousarray(a, np.float64)


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def deposit(x, y, q, m, n, dx, dy):
    x, y, q = f64(x), f64(y), f64(np.broadcast_to(q, np.shape(x)))
    rho = np.zeros(m * n)
    lib().orc_deposit(len(x), _d(x), _d(y), _d(q), m, n, dx, dy, _d(rho))
    return rho.reshape(n, m)


def efield(phi, dx, dy):
    phi = f64(phi)
    n, m = phi.shape
    ex, ey = np.empty(m * n), np.empty(m * n)
    lib().orc_efield(_d(phi), m, n, dx, dy, _d(ex), _d(ey))
    return ex.reshape(n, m), ey.reshape(n, m)


def kick(x, y, vx, vy, q, mass, Ex, Ey, dx, dy, dt):
    x, y = f64(x), f64(y)
    vx, vy = f64(vx).copy(), f64(vy).copy()
    q = f64(np.broadcast_to(q, x.shape))
    mass = f64(np.broadcast_to(mass, x.shape))
    Ex, Ey = f64(Ex), f64(Ey)
    n, m = Ex.shape
    lib().orc_kick(len(x), _d(x), _d(y), _d(vx), _d(vy), _d(q), _d(mass), _d(Ex), _d(Ey), m, n, dx, dy, dt)
    return vx, vy


def drift(x, y, vx, vy, dt):
    x, y = f64(x).copy(), f64(y).copy()
    vx, vy = f64(vx), f64(vy)
    xo, yo = np.empty_like(x), np.empty_like(y)
    lib().orc_drift(len(x), _d(x), _d(y), _d(vx), _d(vy), _d(xo), _d(yo), dt)
    return x, y


def walls_segments(x0, y0, x1, y1, walls, ref_epsilon=False):
    x0, y0, x1, y1 = f64(x0), f64(y0), f64(x1), f64(y1)
    w = f64(walls).reshape(-1)
    hit = np.zeros(len(x0), np.uint8)
    f = lib().orc_walls_segments_ref if ref_epsilon else lib().orc_walls_segments
    f(len(x0), _d(x0), _d(y0), _d(x1), _d(y1), _d(w), len(w) // 4, hit.ctypes.data_as(_U8))
    return hit.astype(bool)


def walls_box(x, y, m, n, dx, dy):
    x, y = f64(x), f64(y)
    hit = np.zeros(len(x), np.uint8)
    lib().orc_walls_box(len(x), _d(x), _d(y), m, n, dx, dy, hit.ctypes.data_as(_U8))
    return hit.astype(bool)


def mg_solve(phi, f, h, levels=0, omega=1.0, nu1=2, nu2=2, nuc=2, tol=1e-9, max_cycles=50, ref_convergence=False):
    """ref_convergence: stop like the reference (||r|| < tol * ||f||^2, Multigrid.cu:466-467)."""
    phi = f64(phi).copy()
    f = f64(f)
    ny, nx = phi.shape
    rel = C.c_double()
    set_reference_convergence(ref_convergence)
    try:
        cyc = lib().orc_mg_solve(_d(phi), _d(f), nx, ny, levels, h, omega, nu1, nu2, nuc, tol, max_cycles,
                                 C.byref(rel))
    finally:
        set_reference_convergence(False)
    return phi, cyc, rel.value


def set_reference_convergence(on: bool) -> None:
    lib().orc_set_reference_convergence(1 if on else 0)


def mg_vcycles(phi, f, h, cycles, levels=0, omega=1.0, nu1=2, nu2=2, nuc=2):
    phi = f64(phi).copy()
    f = f64(f)
    ny, nx = phi.shape
    lib().orc_mg_vcycles(_d(phi), _d(f), nx, ny, levels, h, omega, nu1, nu2, nuc, cycles)
    return phi


def relres(phi, f, h):
    phi, f = f64(phi), f64(f)
    ny, nx = phi.shape
    return lib().orc_relres(_d(phi), _d(f), nx, ny, h)


def residual(phi, f, h):
    phi, f = f64(phi), f64(f)
    ny, nx = phi.shape
    r = np.empty_like(phi)
    lib().orc_residual(_d(r), _d(phi), _d(f), nx, ny, h)
    return r


# ---- embedded-boundary multigrid (Multigrid_embedded.cu): mask 0 FLUID, 1 DIRICHLET, 2 SOLID
def _u8(a):
    return a.ctypes.data_as(_U8)


def _mask(m):
    return np.ascontiguousarray(m, np.uint8)


def emb_coarse_shape(nx, ny):
    return (nx - 1) // 2 + 1, (ny - 1) // 2 + 1


def emb_half_sweep(phi, rhs, mask, bc, h2, colour):
    """One colour of smooth_redblack (Multigrid_embedded.cu:15-33), intended colour test."""
    phi = f64(phi).copy()
    rhs, mask = f64(rhs), _mask(mask)
    bcp = _d(f64(bc)) if bc is not None else None
    ny, nx = phi.shape
    lib().orc_emb_half_sweep(_d(phi), _d(rhs), _u8(mask), bcp, nx, ny, h2, colour)
    return phi


def emb_residual(phi, rhs, mask, h2i):
    """residual_kernel (Multigrid_embedded.cu:35-55) into a zeroed array."""
    phi, rhs, mask = f64(phi), f64(rhs), _mask(mask)
    ny, nx = phi.shape
    res = np.zeros_like(phi)
    lib().orc_emb_residual(_d(res), _d(phi), _d(rhs), _u8(mask), nx, ny, h2i)
    return res


def emb_restrict(res, mask, options=0):
    """restrict_kernel (Multigrid_embedded.cu:57-86): coarse rhs and coarse mask (zeroed
    boundary, like the reference's cudaMemset arrays)."""
    res, mask = f64(res), _mask(mask)
    nyf, nxf = res.shape
    nxc, nyc = emb_coarse_shape(nxf, nyf)
    coarse = np.zeros((nyc, nxc))
    mc = np.zeros((nyc, nxc), np.uint8)
    lib().orc_emb_restrict(_d(res), _d(coarse), _u8(mask), _u8(mc), nxf, nyf, nxc, nyc, options)
    return coarse, mc


def emb_prolong(coarse, fine, mask, options=0):
    """prolongate_add_kernel (Multigrid_embedded.cu:88-104)."""
    coarse, fine, mask = f64(coarse), f64(fine).copy(), _mask(mask)
    nyf, nxf = fine.shape
    nyc, nxc = coarse.shape
    lib().orc_emb_prolong(_d(coarse), _d(fine), _u8(mask), nxf, nyf, nxc, nyc, options)
    return fine


def emb_vcycles(phi, rhs, mask, bc, h, levels, cycles, nu1=2, nu2=2, options=0):
    phi = f64(phi).copy()
    rhs, mask = f64(rhs), _mask(mask)
    bcp = _d(f64(bc)) if bc is not None else None
    ny, nx = phi.shape
    lib().orc_emb_vcycles(_d(phi), _d(rhs), _u8(mask), bcp, nx, ny, levels, h, nu1, nu2, options, cycles)
    return phi


def emb_solve(phi, rhs, mask, bc, h, levels, nu1=2, nu2=2, tol=1e-10, max_cycles=100, options=0):
    phi = f64(phi).copy()
    rhs, mask = f64(rhs), _mask(mask)
    bcp = _d(f64(bc)) if bc is not None else None
    ny, nx = phi.shape
    rel = C.c_double()
    cyc = lib().orc_emb_solve(_d(phi), _d(rhs), _u8(mask), bcp, nx, ny, levels, h, nu1, nu2, options, tol,
                              max_cycles, C.byref(rel))
    return phi, cyc, rel.value


def emb_norms(phi, rhs, mask, h):
    phi, rhs, mask = f64(phi), f64(rhs), _mask(mask)
    ny, nx = phi.shape
    out = np.zeros(2)
    lib().orc_emb_norms(_d(phi), _d(rhs), _u8(mask), nx, ny, h, _d(out))
    return out


class Sim:
    """The oracle's full step on the same pic_job_config the engine takes."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.h = lib().orc_sim_create(C.byref(cfg))
        self.nx, self.ny = cfg.nx, cfg.ny

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_sim_destroy(self.h)
            self.h = None

    def load(self, k, x, y, vx, vy, vz=None, pid=None):
        x, y, vx, vy = f64(x), f64(y), f64(vx), f64(vy)
        vz = f64(vz) if vz is not None else None
        pid = np.ascontiguousarray(pid, np.uint32) if pid is not None else None
        lib().orc_sim_load(self.h, k, len(x), _d(x), _d(y), _d(vx), _d(vy), _d(vz) if vz is not None else None,
                           pid.ctypes.data_as(_U32) if pid is not None else None)

    def export(self, k):
        n = lib().orc_sim_count(self.h, k)
        out = {a: np.empty(n) for a in ("x", "y", "vx", "vy", "vz")}
        out["pid"] = np.empty(n, np.uint32)
        lib().orc_sim_export(self.h, k, _d(out["x"]), _d(out["y"]), _d(out["vx"]), _d(out["vy"]), _d(out["vz"]),
                             out["pid"].ctypes.data_as(_U32))
        return out

    def grid(self, which):
        g = np.empty(self.nx * self.ny)
        lib().orc_sim_get_grid(self.h, which, _d(g))
        return g.reshape(self.ny, self.nx)

    def set_grid(self, which, a):
        a = f64(a).reshape(-1)
        lib().orc_sim_set_grid(self.h, which, _d(a))

    def numax(self, k):
        return lib().orc_sim_numax(self.h, k)

    def set_counters(self, step, next_pid):
        """Continue a running engine job: its completed step count and next particle id."""
        lib().orc_sim_set_counters(self.h, int(step), int(next_pid))

    def stats(self):
        step, cyc, rel, nio = C.c_int64(), C.c_int(), C.c_double(), C.c_int64()
        ab = (C.c_int64 * 4)()
        nc = (C.c_int64 * 32)()
        lib().orc_sim_stats(self.h, C.byref(step), C.byref(cyc), C.byref(rel), ab, nc, C.byref(nio))
        ns = self.cfg.n_species
        return {"step": step.value, "cycles": cyc.value, "relres": rel.value, "absorbed": list(ab)[:ns],
                "collisions": [list(nc)[8 * k: 8 * k + 8] for k in range(ns)], "ionizations": nio.value}

    def drift_walls(self):
        lib().orc_sim_drift_walls(self.h)

    def deposit(self):
        lib().orc_sim_deposit(self.h)

    def solve(self):
        lib().orc_sim_solve(self.h)

    def kick(self):
        lib().orc_sim_kick(self.h)

    def mcc(self):
        lib().orc_sim_mcc(self.h)

    def step(self, n=1):
        lib().orc_sim_step(self.h, n)

    def total_charge(self):
        return lib().orc_sim_total_charge(self.h)


def num_threads():
    return lib().orc_num_threads()
