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
