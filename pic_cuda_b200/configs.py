"""Job configurations of the benchmark workloads and seeded synthetic initial states.

Workloads (all synthetic and seeded; no external data set is involved):
  plain_small   129^2 nodes over 1 cm^2, 1e5 electrons + 1e5 Ar+ (40 amu), Te 2 eV, Ti 0.03 eV,
                phi = 0 Dirichlet, absorbing box walls, dt 1e-11 s, multigrid RB-GS 2+2 to 1e-6,
                no collisions.
  mcc_mixed     1025^2 nodes over 5 cm^2, 1e7 + 1e7, Te 3 eV (Ti 0.03 eV), argon 3.2e21 m^-3 at
                300 K, 512-point log-spaced FP32 tables 0.01-1000 eV, null-collision MCC, FP32
                V-cycles (red-black SOR, omega 1.15, 2 + 2 sweeps) in FP64 defect correction
                to 1e-9.
  large         4097^2 nodes (dx as in mcc_mixed: 20 cm^2), 1e8 + 1e8, Te 2 eV, same MCC, sort
                every 10 steps, FP32 or int64 deposit.
Macro-particle weight: a plasma density n0 = 1e15 m^-3 over the domain with 1 m depth
(w = n0 * area / N per species), which gives lambda_D/dx ~ 4-8 and w_p dt ~ 0.02.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib as L

QE = 1.602176634e-19
ME = 9.1093837015e-31
AMU = 1.66053906660e-27
KB = 1.380649e-23
M_AR = 40.0 * AMU  # "singly charged ions (mass 40 amu)"


def argon_tables(n: int = 512, e_min: float = 0.01, e_max: float = 1000.0) -> dict:
    """Synthetic argon cross sections on n log-spaced points, rounded to FP32.
    elastic 1e-19 m^2; excitation 0 below 11.5 eV, linear to 1e-20 at 30 eV, then flat;
    ionisation 0 below 15.76 eV, linear to 3e-20 at 100 eV, then flat; ion charge exchange 5e-19."""
    E = np.logspace(math.log10(e_min), math.log10(e_max), n).astype(np.float32).astype(np.float64)
    ela = np.full(n, 1e-19)
    exc = np.where(E < 11.5, 0.0, np.minimum((E - 11.5) / (30.0 - 11.5), 1.0) * 1e-20)
    iz = np.where(E < 15.76, 0.0, np.minimum((E - 15.76) / (100.0 - 15.76), 1.0) * 3e-20)
    cx = np.full(n, 5e-19)
    f32 = lambda a: np.ascontiguousarray(a.astype(np.float32).astype(np.float64))
    return {"E": np.ascontiguousarray(E), "elastic": f32(ela), "excitation": f32(exc), "ionization": f32(iz),
            "cx": f32(cx)}


def make_config(nx: int, L_dom: float, dt: float, species: list[tuple[float, float, float, int]], *,
                units: int = L.UNITS_SI, walls: int = L.WALLS_BOX, wall_segments=(), tol: float = 1e-6,
                nu_pre: int = 2, nu_post: int = 2, nu_coarse: int = 2, omega: float = 1.0, levels: int = 0,
                max_cycles: int = 50, deposit: int = L.DEPOSIT_F32, sort_every: int = 10, mcc: dict | None = None,
                seed: int = 1234, warm_start: int = 0) -> L.JobConfig:
    """species: (charge C, mass kg, weight, capacity) per species.  mcc: dict with keys
    mode, density, temperature, gas_mass, processes [(type, species, threshold, E, sigma)],
    e_species, i_species."""
    c = L.JobConfig()
    c.nx = c.ny = nx
    c.Lx = c.Ly = L_dom
    c.dt = dt
    c.units = units
    c.n_species = len(species)
    for k, (q, m, w, cap) in enumerate(species):
        c.species[k].charge, c.species[k].mass, c.species[k].weight, c.species[k].capacity = q, m, w, cap
    c.mg_levels, c.nu_pre, c.nu_post, c.nu_coarse = levels, nu_pre, nu_post, nu_coarse
    c.omega, c.tol, c.max_cycles = omega, tol, max_cycles
    c.wall_mode = walls
    c.n_walls = len(wall_segments)
    for k, w in enumerate(wall_segments):
        for a in range(4):
            c.walls[k][a] = w[a]
    c.deposit_mode = deposit
    c.sort_every = sort_every
    c.seed = seed
    c.mg_warm_start = warm_start
    keep = []
    if mcc:
        c.mcc_mode = mcc.get("mode", L.MCC_NULL_COLLISION)
        c.gas_density = mcc["density"]
        c.gas_temperature = mcc.get("temperature", 300.0)
        c.gas_mass = mcc.get("gas_mass", M_AR)
        c.n_processes = len(mcc["processes"])
        for k, (typ, sp, thr, E, sig) in enumerate(mcc["processes"]):
            E = np.ascontiguousarray(E, np.float64)
            sig = np.ascontiguousarray(sig, np.float64)
            keep += [E, sig]
            p = c.processes[k]
            p.type, p.species, p.threshold_ev, p.n_points = typ, sp, thr, len(E)
            p.energy_ev = E.ctypes.data_as(L.C.POINTER(L.C.c_double))
            p.sigma_m2 = sig.ctypes.data_as(L.C.POINTER(L.C.c_double))
        c.ionization_electron_species = mcc.get("e_species", 0)
        c.ionization_ion_species = mcc.get("i_species", 1)
    c._keep = keep  # the tables must outlive the config
    return c


def argon_mcc(density: float, temperature: float = 300.0) -> dict:
    t = argon_tables()
    return {
        "mode": L.MCC_NULL_COLLISION, "density": density, "temperature": temperature, "gas_mass": M_AR,
        "processes": [
            (L.PROC_ELASTIC, 0, 0.0, t["E"], t["elastic"]),
            (L.PROC_EXCITATION, 0, 11.5, t["E"], t["excitation"]),
            (L.PROC_IONIZATION, 0, 15.76, t["E"], t["ionization"]),
            (L.PROC_CHARGE_EXCHANGE, 1, 0.0, t["E"], t["cx"]),
        ],
        "e_species": 0, "i_species": 1,
    }


def plasma(nx: int, L_dom: float, n_per_species: int, *, n0: float = 1e15, capacity_factor: float = 1.25,
           **kw) -> L.JobConfig:
    w = n0 * L_dom * L_dom / n_per_species
    cap = int(n_per_species * capacity_factor) + 1024
    return make_config(nx, L_dom, kw.pop("dt", 1e-11), [(-QE, ME, w, cap), (QE, M_AR, w, cap)], **kw)


def plain_small(**kw) -> L.JobConfig:
    kw.setdefault("tol", 1e-6)
    kw.setdefault("warm_start", 1)
    return plasma(129, 0.01, 100_000, **kw)


# Over-relaxation of the red-black smoother for the 1e-9 workloads (the reference's solver is
# red-black SOR, Multigrid.cu:246-265).  Measured V-cycle contraction of V(2,2) on the FP64
# oracle: 0.052 at omega 1 (Gauss-Seidel), 0.019 at 1.15, 0.025 at 1.25; on B200 the 1025^2
# MCC step then takes 4 V-cycles instead of 5 (0.95 against 1.05 ms per step).
MG_OMEGA_1E9 = 1.15


def mcc_mixed(n_per_species: int = 10_000_000, **kw) -> L.JobConfig:
    kw.setdefault("tol", 1e-9)
    kw.setdefault("warm_start", 1)
    kw.setdefault("omega", MG_OMEGA_1E9)
    kw.setdefault("mcc", argon_mcc(3.2e21))
    return plasma(1025, 0.05, n_per_species, **kw)


def large(n_per_species: int = 100_000_000, deposit: int = L.DEPOSIT_F32, **kw) -> L.JobConfig:
    kw.setdefault("tol", 1e-9)
    kw.setdefault("warm_start", 1)
    kw.setdefault("omega", MG_OMEGA_1E9)
    kw.setdefault("mcc", argon_mcc(3.2e21))
    return plasma(4097, 0.05 * 4, n_per_species, deposit=deposit, **kw)


WORKLOADS = {
    "plain_small": dict(builder=plain_small, n=100_000, Te=2.0, Ti=0.03),
    "mcc_mixed": dict(builder=mcc_mixed, n=10_000_000, Te=3.0, Ti=0.03),
    "large": dict(builder=large, n=100_000_000, Te=2.0, Ti=0.03),
}


def maxwellian_state(n: int, L_dom: float, T_ev: float, mass: float, seed: int, device=None):
    """Uniform positions in [0, L)^2 and Maxwellian (vx, vy, vz) at temperature T_ev.
    numpy (host) when device is None, else torch tensors generated on that CUDA device."""
    vth = math.sqrt(T_ev * QE / mass)
    if device is None:
        rng = np.random.default_rng(seed)
        x = rng.random(n) * L_dom
        y = rng.random(n) * L_dom
        v = rng.standard_normal((3, n)) * vth
        return x, y, v[0].copy(), v[1].copy(), v[2].copy()
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    x = torch.rand(n, generator=g, device=device, dtype=torch.float64) * L_dom
    y = torch.rand(n, generator=g, device=device, dtype=torch.float64) * L_dom
    v = torch.randn(3, n, generator=g, device=device, dtype=torch.float64) * vth
    return x, y, v[0].contiguous(), v[1].contiguous(), v[2].contiguous()


def load_plasma(job, n_per_species: int, L_dom: float, Te: float, Ti: float, seed: int = 1234, device=None):
    """Electrons (species 0) and Ar+ (species 1), uniform, Maxwellian."""
    e = maxwellian_state(n_per_species, L_dom, Te, ME, seed, device)
    i = maxwellian_state(n_per_species, L_dom, Ti, M_AR, seed + 1, device)
    job.load_species(0, *e)
    job.load_species(1, *i)
    return e, i
