"""Cross-section tables from files, for the null-collision MCC.

`read_cross_section` has the semantics of the reference's reader (mcc.cu:17-41): a text file
of `energy sigma` pairs (eV, m^2), one per line; empty lines and lines starting with '#' are
skipped; a line whose first two fields do not parse as numbers is skipped; anything after
the second field is ignored; a file that cannot be opened gives two empty lists (the
reference prints an error and returns empty vectors).  The LXCat-style files the reference
ships (its csf/ directory) have this layout on non-uniform energy grids.

The engine holds every table in FP32 on the device; `process_table` rounds a table once to
FP32, so the engine and any FP64 check of it interpolate the same values.
"""
from __future__ import annotations

import sys

import numpy as np

from . import _lib as L
from . import configs as cf


def _number(tok: str):
    try:
        return float(tok)
    except ValueError:
        return None


def read_cross_section(filename) -> tuple[list[float], list[float]]:
    energies: list[float] = []
    sigmas: list[float] = []
    try:
        fh = open(filename, "r")
    except OSError:
        print(f"Error: cannot open cross-section file: {filename}", file=sys.stderr)
        return energies, sigmas
    with fh:
        for line in fh:
            line = line.rstrip("\r\n")
            if not line or line[0] == "#":
                continue
            tok = line.split()
            if len(tok) < 2:
                continue
            e, s = _number(tok[0]), _number(tok[1])
            if e is None or s is None:
                continue
            energies.append(e)
            sigmas.append(s)
    return energies, sigmas


def process_table(energies, sigmas) -> tuple[np.ndarray, np.ndarray]:
    """(E, sigma) as FP64 arrays holding FP32-representable values, checked for the engine's
    table rules (at least 2 points, energies strictly increasing)."""
    e = np.asarray(energies, np.float64).astype(np.float32).astype(np.float64)
    s = np.asarray(sigmas, np.float64).astype(np.float32).astype(np.float64)
    if e.shape != s.shape or e.ndim != 1 or len(e) < 2:
        raise ValueError("a cross-section table needs at least two (energy, sigma) points")
    if not np.all(np.diff(e) > 0):
        raise ValueError("cross-section energies must increase strictly")
    return np.ascontiguousarray(e), np.ascontiguousarray(s)


def argon_file_mcc(density: float, elastic, ionization, *, excitation=None, charge_exchange=None,
                   temperature: float = 300.0) -> dict:
    """Null-collision MCC for electrons and Ar+ in argon with the electron elastic and
    ionisation cross sections given as (E, sigma) tables (e.g. read from the reference's
    csf/Ar.txt and csf/Ar+.txt).  Excitation and ion charge exchange default to the
    synthetic tables of the benchmark configurations (11.5 eV threshold; 5e-19 m^2)."""
    syn = cf.argon_tables()
    el = process_table(*elastic)
    iz = process_table(*ionization)
    ex = process_table(*excitation) if excitation is not None else (syn["E"], syn["excitation"])
    cx = process_table(*charge_exchange) if charge_exchange is not None else (syn["E"], syn["cx"])
    return {
        "mode": L.MCC_NULL_COLLISION, "density": density, "temperature": temperature, "gas_mass": cf.M_AR,
        "processes": [
            (L.PROC_ELASTIC, 0, 0.0, el[0], el[1]),
            (L.PROC_EXCITATION, 0, 11.5, ex[0], ex[1]),
            (L.PROC_IONIZATION, 0, 15.76, iz[0], iz[1]),
            (L.PROC_CHARGE_EXCHANGE, 1, 0.0, cx[0], cx[1]),
        ],
        "e_species": 0, "i_species": 1,
    }
