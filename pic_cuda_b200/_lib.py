"""ctypes binding of the C ABI in include/pic_b200.h (libpic_b200.so, built in-tree).

The structs below mirror the C declarations field by field; `check_abi()` compares their
sizes with the library's own sizeof values.  Loading fails loudly when the library is
missing: there is no Python or CPU fallback for any compute path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpic_b200.so"

PIC_OK, PIC_ERR_ARG, PIC_ERR_OOM, PIC_ERR_CUDA, PIC_ERR_NOT_CONVERGED = 0, 1, 2, 3, 4
PIC_ERR_TIMEOUT, PIC_ERR_CAPACITY, PIC_ERR_STATE, PIC_ERR_NO_DEVICE = 5, 6, 7, 8
MAX_SPECIES, MAX_WALLS, MAX_PROCESSES = 4, 64, 8
UNITS_REF, UNITS_SI = 0, 1
WALLS_NONE, WALLS_BOX, WALLS_SEGMENTS, WALLS_BOX_AND_SEGMENTS = 0, 1, 2, 3
DEPOSIT_F32, DEPOSIT_I64 = 0, 1
MCC_NONE, MCC_NULL_COLLISION, MCC_REF_ELASTIC2D = 0, 1, 2
PROC_ELASTIC, PROC_EXCITATION, PROC_IONIZATION, PROC_CHARGE_EXCHANGE = 1, 2, 3, 4
PHASE_KICK, PHASE_MCC, PHASE_DRIFT, PHASE_WALLS, PHASE_DEPOSIT = 1, 2, 4, 8, 16
GRID_RHO, GRID_PHI, GRID_EX, GRID_EY = 0, 1, 2, 3
MEM_HOST, MEM_DEVICE = 0, 1
OPT_MG_LEVELS_KERNEL, OPT_MG_CLUSTER_TOP, OPT_MG_COARSE_TOP, OPT_MOVER_CTAS_PER_SM, OPT_MG_WIDE_TILES = 1, 2, 3, 4, 5
NODE_FLUID, NODE_DIRICHLET, NODE_SOLID = 0, 1, 2
EMB_COARSEN_ANY, EMB_PROLONG_BILINEAR = 1, 2


class SpeciesConfig(C.Structure):
    _fields_ = [("charge", C.c_double), ("mass", C.c_double), ("weight", C.c_double), ("capacity", C.c_int64)]


class ProcessConfig(C.Structure):
    _fields_ = [("type", C.c_int), ("species", C.c_int), ("threshold_ev", C.c_double), ("n_points", C.c_int),
                ("energy_ev", C.POINTER(C.c_double)), ("sigma_m2", C.POINTER(C.c_double))]


class JobConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("Lx", C.c_double), ("Ly", C.c_double), ("dt", C.c_double),
        ("units", C.c_int), ("n_species", C.c_int), ("species", SpeciesConfig * MAX_SPECIES),
        ("mg_levels", C.c_int), ("nu_pre", C.c_int), ("nu_post", C.c_int), ("nu_coarse", C.c_int),
        ("omega", C.c_double), ("tol", C.c_double), ("max_cycles", C.c_int),
        ("wall_mode", C.c_int), ("n_walls", C.c_int), ("walls", (C.c_double * 4) * MAX_WALLS),
        ("deposit_mode", C.c_int), ("sort_every", C.c_int),
        ("mcc_mode", C.c_int), ("gas_density", C.c_double), ("gas_temperature", C.c_double),
        ("gas_mass", C.c_double), ("n_processes", C.c_int), ("processes", ProcessConfig * MAX_PROCESSES),
        ("ionization_electron_species", C.c_int), ("ionization_ion_species", C.c_int), ("seed", C.c_uint64),
        ("mg_warm_start", C.c_int),
    ]


class Diagnostics(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("count", C.c_int64 * MAX_SPECIES), ("absorbed", C.c_int64 * MAX_SPECIES),
        ("collisions", (C.c_int64 * MAX_PROCESSES) * MAX_SPECIES), ("ionizations", C.c_int64),
        ("vcycles", C.c_int32), ("converged", C.c_int32), ("relres", C.c_double), ("total_charge", C.c_double),
        ("kinetic_energy", C.c_double * MAX_SPECIES), ("status", C.c_uint32),
        ("next_pid", C.c_uint32),
    ]


class EngineStats(C.Structure):
    _fields_ = [("kernel_launches", C.c_int64), ("steps", C.c_int64), ("vcycles", C.c_int64),
                ("mover_launches", C.c_int64), ("mover_ms", C.c_double), ("phase_ms", C.c_double * 4)]


class PicError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


_lib = None

# name -> (restype, argtypes)
_VP, _D, _I, _I64 = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_int64
_SIGS = {
    "pic_engine_create": (_I, [_I, _I64, C.POINTER(_VP)]),
    "pic_engine_destroy": (_I, [_VP]),
    "pic_engine_bytes_needed": (_I, [C.POINTER(JobConfig), C.POINTER(_I64)]),
    "pic_engine_num_jobs": (_I, [_VP, C.POINTER(_I)]),
    "pic_engine_reserve": (_I, [_VP, _I64]),
    "pic_job_create": (_I, [_VP, C.POINTER(JobConfig), C.POINTER(_I)]),
    "pic_job_destroy": (_I, [_VP, _I]),
    "pic_job_load_species": (_I, [_VP, _I, _I, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _I]),
    "pic_job_export_species": (_I, [_VP, _I, _I, _I64, _VP, _VP, _VP, _VP, _VP, _VP, C.POINTER(_I64), _I]),
    "pic_job_export_species_raw": (_I, [_VP, _I, _I, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, C.POINTER(_I64)]),
    "pic_step": (_I, [_VP, _I, _VP]),
    "pic_step_graph": (_I, [_VP, _I, _VP]),
    "pic_sync": (_I, [_VP]),
    "pic_engine_profile": (_I, [_VP, _I]),
    "pic_engine_get_stats": (_I, [_VP, C.POINTER(EngineStats), _I]),
    "pic_job_diagnostics": (_I, [_VP, _I, C.POINTER(Diagnostics)]),
    "pic_job_run_phases": (_I, [_VP, _I, _I, _I64, _VP]),
    "pic_job_compact": (_I, [_VP, _I, _VP]),
    "pic_job_zero_rho": (_I, [_VP, _I, _VP]),
    "pic_job_solve_field": (_I, [_VP, _I, _VP]),
    "pic_job_sort": (_I, [_VP, _I, _VP]),
    "pic_job_get_grid": (_I, [_VP, _I, _I, _VP, _I]),
    "pic_job_set_grid": (_I, [_VP, _I, _I, _VP, _I]),
    "pic_job_get_hits": (_I, [_VP, _I, _I, _I64, C.POINTER(_I64), C.POINTER(_I64)]),
    "pic_solve_multigrid_f64": (_I, [_VP, _VP, _I, _I, _I, C.c_double, C.c_double, _I, _I, _I, C.c_double, _I,
                                     _VP, C.POINTER(_I), _D]),
    "pic_efield_f64": (_I, [_VP, _VP, _I, _I, C.c_double, C.c_double, _VP]),
    "pic_job_snapshot_positions": (_I, [_VP, _I, _I, _I64, _VP, C.POINTER(_I64), _I]),
    "pic_solve_embedded_f64": (_I, [_VP, _VP, _VP, _VP, _I, _I, _I, C.c_double, _I, _I, _I, C.c_double, _I, _VP,
                                    C.POINTER(_I), _D]),
    "pic_engine_set_option": (_I, [_VP, _I, _I64]),
    "pic_engine_get_option": (_I, [_VP, _I, C.POINTER(_I64)]),
    "pic_job_set_sort_every": (_I, [_VP, _I, _I]),
    "pic_solve_multigrid_f64_static": (_I, [_VP, _VP, _I, _I, _I, C.c_double, C.c_double, _I, _I, _I, C.c_double,
                                            _I, _VP, C.POINTER(_I), _D]),
    "pic_last_error": (C.c_char_p, []),
    "pic_version": (_I, []),
    "pic_abi_sizes": (_I, [C.POINTER(_I64)]),
    "pic_philox4x32_10": (None, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
}


def lib():
    """The loaded engine library (raises if it is missing: no fallback exists)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m pic_cuda_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(code: int, where: str) -> None:
    if code != PIC_OK:
        raise PicError(code, where, (lib().pic_last_error() or b"").decode())


def check_abi() -> None:
    out = (C.c_int64 * 4)()
    lib().pic_abi_sizes(out)
    mine = [C.sizeof(JobConfig), C.sizeof(Diagnostics), C.sizeof(SpeciesConfig), C.sizeof(ProcessConfig)]
    if list(out) != mine:
        raise RuntimeError(f"ctypes struct sizes {mine} differ from the library's {list(out)}")


def philox4x32_10(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().pic_philox4x32_10(c, k, o)
    return list(o)
