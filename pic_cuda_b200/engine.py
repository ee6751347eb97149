"""Python host API over the C ABI: Engine (device tables + stepping) and Job (one simulation).

Arrays passed in may be numpy arrays (host memory) or CUDA torch tensors (device memory);
the engine converts them to its FP32 cell-relative layout on the device.  Every compute
call goes to libpic_b200.so; nothing here computes physics on the host.
"""
from __future__ import annotations

import ctypes as C
from typing import Any

import numpy as np

from . import _lib as L


def _is_torch_cuda(a: Any) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _as_ptr(a: Any, dtype, n: int | None = None):
    """(pointer, memory kind, keep-alive) for a host numpy array or a CUDA torch tensor."""
    if a is None:
        return None, L.MEM_HOST, None
    if _is_torch_cuda(a):
        import torch
        tdt = {np.float64: torch.float64, np.float32: torch.float32, np.uint32: torch.int32,
               np.int64: torch.int64}[dtype]
        t = a.contiguous()
        if t.dtype != tdt:
            t = t.to(tdt)
        return C.c_void_p(t.data_ptr()), L.MEM_DEVICE, t
    if hasattr(a, "numpy") and not isinstance(a, np.ndarray):  # CPU torch tensor (maybe pinned)
        if a.is_contiguous() and str(a.dtype).endswith({np.float64: "float64", np.float32: "float32",
                                                            np.uint32: "int32", np.int64: "int64"}[dtype]):
            return C.c_void_p(a.data_ptr()), L.MEM_HOST, a
        a = a.numpy()
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data_as(C.c_void_p), L.MEM_HOST, arr


class Job:
    def __init__(self, engine: "Engine", job_id: int, cfg: L.JobConfig, keep: Any = None):
        self.engine = engine
        self.id = job_id
        self.cfg = cfg
        self._keep = keep
        self.nx, self.ny = cfg.nx, cfg.ny

    # -- particles
    def load_species(self, species: int, x, y, vx, vy, vz=None, pid=None) -> None:
        n = len(x)
        px, mem, kx = _as_ptr(x, np.float64)
        py, _, ky = _as_ptr(y, np.float64)
        pvx, _, kvx = _as_ptr(vx, np.float64)
        pvy, _, kvy = _as_ptr(vy, np.float64)
        pvz, _, kvz = _as_ptr(vz, np.float64)
        ppid, _, kp = _as_ptr(pid, np.uint32)
        L.check(L.lib().pic_job_load_species(self.engine.h, self.id, species, n, px, py, pvx, pvy, pvz, ppid, mem),
                "pic_job_load_species")

    def count(self, species: int) -> int:
        return int(self.diagnostics()["count"][species])

    def export_species(self, species: int) -> dict:
        cap = int(self.cfg.species[species].capacity)
        out = {k: np.empty(cap, np.float64) for k in ("x", "y", "vx", "vy", "vz")}
        out["pid"] = np.empty(cap, np.uint32)
        n = C.c_int64()
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        L.check(L.lib().pic_job_export_species(self.engine.h, self.id, species, cap, ptr(out["x"]), ptr(out["y"]),
                                               ptr(out["vx"]), ptr(out["vy"]), ptr(out["vz"]), ptr(out["pid"]),
                                               C.byref(n), L.MEM_HOST), "pic_job_export_species")
        return {k: v[: n.value] for k, v in out.items()}

    def export_raw(self, species: int) -> dict:
        """FP32 cell-relative layout as CUDA torch tensors (no host round trip)."""
        import torch
        cap = int(self.cfg.species[species].capacity)
        dev = torch.device("cuda", self.engine.device)
        out = {k: torch.empty(cap, dtype=torch.float32, device=dev) for k in ("fx", "fy", "vx", "vy", "vz")}
        out["cell"] = torch.empty(cap, dtype=torch.int32, device=dev)
        out["pid"] = torch.empty(cap, dtype=torch.int32, device=dev)
        n = C.c_int64()
        p = lambda t: C.c_void_p(t.data_ptr())
        L.check(L.lib().pic_job_export_species_raw(self.engine.h, self.id, species, cap, p(out["cell"]), p(out["fx"]),
                                                   p(out["fy"]), p(out["vx"]), p(out["vy"]), p(out["vz"]),
                                                   p(out["pid"]), C.byref(n)), "pic_job_export_species_raw")
        return {k: v[: n.value] for k, v in out.items()}

    def snapshot_positions(self, species: int, device: bool = False):
        """Interleaved FP32 (x, y) of every particle, shape (n, 2): the headless counterpart of
        the reference's vertex-buffer fill (kernels.cu:268-274).  device=True returns a CUDA
        torch tensor filled on the device, else a numpy array."""
        cap = int(self.cfg.species[species].capacity)
        n = C.c_int64()
        if device:
            import torch
            out = torch.empty((cap, 2), dtype=torch.float32, device=torch.device("cuda", self.engine.device))
            ptr, mem = C.c_void_p(out.data_ptr()), L.MEM_DEVICE
        else:
            out = np.empty((cap, 2), np.float32)
            ptr, mem = out.ctypes.data_as(C.c_void_p), L.MEM_HOST
        L.check(L.lib().pic_job_snapshot_positions(self.engine.h, self.id, species, cap, ptr, C.byref(n), mem),
                "pic_job_snapshot_positions")
        return out[: n.value]

    def write_snapshot(self, path) -> None:
        """Positions of every species and the job's diagnostics to one .npz file (the headless
        replacement of the reference's viewer frame)."""
        data = {f"xy{s}": self.snapshot_positions(s) for s in range(int(self.cfg.n_species))}
        d = self.diagnostics()
        for k, v in d.items():
            data[f"diag_{k}"] = np.asarray(v)
        np.savez_compressed(path, **data)

    def hits(self, species: int) -> np.ndarray:
        cap = int(self.cfg.species[species].capacity)
        buf = np.empty(max(cap, 1), np.int64)
        n = C.c_int64()
        L.check(L.lib().pic_job_get_hits(self.engine.h, self.id, species, cap,
                                         buf.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(n)), "pic_job_get_hits")
        return buf[: n.value].copy()

    # -- grids
    def get_grid(self, which: int) -> np.ndarray:
        out = np.empty(self.nx * self.ny, np.float64)
        L.check(L.lib().pic_job_get_grid(self.engine.h, self.id, which, out.ctypes.data_as(C.c_void_p), L.MEM_HOST),
                "pic_job_get_grid")
        return out.reshape(self.ny, self.nx)

    def set_grid(self, which: int, arr) -> None:
        a = np.ascontiguousarray(arr, np.float64).reshape(-1)
        L.check(L.lib().pic_job_set_grid(self.engine.h, self.id, which, a.ctypes.data_as(C.c_void_p), L.MEM_HOST),
                "pic_job_set_grid")

    # -- phases
    def run_phases(self, flags: int, step: int = 0) -> None:
        L.check(L.lib().pic_job_run_phases(self.engine.h, self.id, flags, step, None), "pic_job_run_phases")

    def set_sort_every(self, n: int) -> None:
        L.check(L.lib().pic_job_set_sort_every(self.engine.h, self.id, n), "pic_job_set_sort_every")

    def compact(self) -> None:
        L.check(L.lib().pic_job_compact(self.engine.h, self.id, None), "pic_job_compact")

    def zero_rho(self) -> None:
        L.check(L.lib().pic_job_zero_rho(self.engine.h, self.id, None), "pic_job_zero_rho")

    def solve_field(self) -> None:
        L.check(L.lib().pic_job_solve_field(self.engine.h, self.id, None), "pic_job_solve_field")

    def sort(self) -> None:
        L.check(L.lib().pic_job_sort(self.engine.h, self.id, None), "pic_job_sort")

    def diagnostics(self) -> dict:
        d = L.Diagnostics()
        L.check(L.lib().pic_job_diagnostics(self.engine.h, self.id, C.byref(d)), "pic_job_diagnostics")
        ns = self.cfg.n_species
        return {
            "step": d.step, "count": [d.count[s] for s in range(ns)], "absorbed": [d.absorbed[s] for s in range(ns)],
            "collisions": [[d.collisions[s][p] for p in range(L.MAX_PROCESSES)] for s in range(ns)],
            "ionizations": d.ionizations, "vcycles": d.vcycles, "converged": bool(d.converged), "relres": d.relres,
            "total_charge": d.total_charge, "kinetic_energy": [d.kinetic_energy[s] for s in range(ns)],
            "status": d.status, "next_pid": d.next_pid,
        }

    def destroy(self) -> None:
        if self.id is not None:
            L.check(L.lib().pic_job_destroy(self.engine.h, self.id), "pic_job_destroy")
            self.id = None


class Engine:
    def __init__(self, device: int = 0, pool_bytes: int = 0):
        self.device = device
        self.h = C.c_void_p()
        L.check(L.lib().pic_engine_create(device, pool_bytes, C.byref(self.h)), "pic_engine_create")

    def add_job(self, cfg: L.JobConfig, keep: Any = None) -> Job:
        jid = C.c_int()
        L.check(L.lib().pic_job_create(self.h, C.byref(cfg), C.byref(jid)), "pic_job_create")
        return Job(self, jid.value, cfg, keep if keep is not None else getattr(cfg, "_keep", None))

    def step(self, n: int = 1, stream=None) -> None:
        L.check(L.lib().pic_step(self.h, n, stream), "pic_step")

    def step_graph(self, n: int = 1, stream=None) -> None:
        L.check(L.lib().pic_step_graph(self.h, n, stream), "pic_step_graph")

    def reserve(self, nbytes: int) -> None:
        """Map nbytes of device memory into the job pool now (pic_engine_reserve), so that
        later job creation does not grow the pool."""
        L.check(L.lib().pic_engine_reserve(self.h, int(nbytes)), "pic_engine_reserve")

    def set_option(self, option: int, value: int) -> None:
        L.check(L.lib().pic_engine_set_option(self.h, option, value), "pic_engine_set_option")

    def get_option(self, option: int) -> int:
        v = L.C.c_int64()
        L.check(L.lib().pic_engine_get_option(self.h, option, L.C.byref(v)), "pic_engine_get_option")
        return v.value

    def sync(self) -> None:
        L.check(L.lib().pic_sync(self.h), "pic_sync")

    def profile(self, enable: bool = True) -> None:
        L.check(L.lib().pic_engine_profile(self.h, 1 if enable else 0), "pic_engine_profile")

    def stats(self, reset: bool = False) -> dict:
        st = L.EngineStats()
        L.check(L.lib().pic_engine_get_stats(self.h, C.byref(st), 1 if reset else 0), "pic_engine_get_stats")
        d = {k: getattr(st, k) for k, _ in st._fields_ if k != "phase_ms"}
        d["phase_ms"] = dict(zip(("sort", "particles", "compact", "field"), list(st.phase_ms)))
        return d

    def close(self) -> None:
        if self.h:
            L.lib().pic_engine_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bytes_needed(cfg: L.JobConfig) -> int:
    b = C.c_int64()
    L.check(L.lib().pic_engine_bytes_needed(C.byref(cfg), C.byref(b)), "pic_engine_bytes_needed")
    return b.value


def check_device_arrays(arrays, shape, device=None):
    """Validate the arrays of a stateless solver call on the host, before anything launches.

    arrays: (name, tensor or None, torch dtype, optional) tuples.  Every given array must be a
    contiguous CUDA tensor of `shape` and its dtype, and all of them must sit on one device
    (the first array's, or `device`).  Returns that device.  Raises ValueError otherwise: a
    kernel handed a host pointer, a wrong-sized buffer or another GPU's memory would read out
    of bounds or over the peer link."""
    dev = device
    for name, a, dt, optional in arrays:
        if a is None:
            if optional:
                continue
            raise ValueError(f"{name}: an array is required")
        if not (getattr(a, "is_cuda", False) and a.dtype == dt and a.is_contiguous()
                and tuple(a.shape) == tuple(shape)):
            raise ValueError(f"{name}: a contiguous CUDA {dt} tensor of shape {tuple(shape)} is required")
        if dev is None:
            dev = a.device
        elif a.device != dev:
            raise ValueError(f"{name}: on {a.device}, but the call runs on {dev}; all arrays must share one device")
    return dev


def _stream_ptr(stream):
    if stream is None:
        return None
    return C.c_void_p(getattr(stream, "cuda_stream", stream))


def solve_multigrid_f64(phi, rho, nx: int, ny: int, levels: int, h: float, omega: float = 1.25, nu_pre: int = 3,
                        nu_post: int = 3, nu_coarse: int = 20, tol: float = 1e-5, max_cycles: int = 50, stream=None,
                        static: bool = False):
    """solve_multigrid (Multigrid.cu:573) on CUDA torch tensors (FP64, (ny, nx), in place on
    phi), on the arrays' device.  static=True calls pic_solve_multigrid_f64_static (no device
    allocation; grids up to PIC_STATIC_MG_MAX_SIDE nodes per side).  Returns (cycles,
    relative residual, converged)."""
    import torch
    dev = check_device_arrays([("phi", phi, torch.float64, False), ("rho", rho, torch.float64, False)], (ny, nx))
    fn = L.lib().pic_solve_multigrid_f64_static if static else L.lib().pic_solve_multigrid_f64
    cyc = C.c_int()
    rel = C.c_double()
    with torch.cuda.device(dev):
        rc = fn(C.c_void_p(phi.data_ptr()), C.c_void_p(rho.data_ptr()), nx, ny, levels, h, omega, nu_pre, nu_post,
                nu_coarse, tol, max_cycles, _stream_ptr(stream), C.byref(cyc), C.byref(rel))
    if rc not in (L.PIC_OK, L.PIC_ERR_NOT_CONVERGED):
        L.check(rc, "pic_solve_multigrid_f64_static" if static else "pic_solve_multigrid_f64")
    return cyc.value, rel.value, rc == L.PIC_OK


def solve_embedded_f64(phi, rhs, mask, phi_bc, levels: int, h: float, nu_pre: int = 2, nu_post: int = 2,
                       options: int = 0, tol: float = 1e-10, max_cycles: int = 100, stream=None):
    """Embedded-boundary multigrid (Multigrid_embedded.cu:110-188) on CUDA torch tensors:
    phi, rhs, phi_bc FP64 and mask uint8 (PIC_NODE_*), all (ny, nx) and on one device; phi in
    place; phi_bc may be None.  Runs on the arrays' device.  Returns (cycles, relative
    residual, converged)."""
    import torch
    if not hasattr(phi, "shape") or len(phi.shape) != 2:
        raise ValueError("phi: a 2-D CUDA float64 tensor is required")
    ny, nx = phi.shape
    dev = check_device_arrays([("phi", phi, torch.float64, False), ("rhs", rhs, torch.float64, False),
                               ("mask", mask, torch.uint8, False), ("phi_bc", phi_bc, torch.float64, True)],
                              (ny, nx))
    cyc = C.c_int()
    rel = C.c_double()
    bc = C.c_void_p(phi_bc.data_ptr()) if phi_bc is not None else None
    with torch.cuda.device(dev):
        rc = L.lib().pic_solve_embedded_f64(C.c_void_p(phi.data_ptr()), C.c_void_p(rhs.data_ptr()),
                                            C.c_void_p(mask.data_ptr()), bc, nx, ny, levels, h, nu_pre, nu_post,
                                            options, tol, max_cycles, _stream_ptr(stream), C.byref(cyc),
                                            C.byref(rel))
    if rc not in (L.PIC_OK, L.PIC_ERR_NOT_CONVERGED):
        L.check(rc, "pic_solve_embedded_f64")
    return cyc.value, rel.value, rc == L.PIC_OK
