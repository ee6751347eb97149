"""Builds tests/compat/compat_driver.cpp (a program written against the reference's headers,
linked to libpic_b200.so) and exchanges record files with it."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "compat" / "compat_driver.cpp"
LIBDIR = ROOT / "pic_cuda_b200"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def build_driver(out_dir: Path) -> Path:
    """Compiles the driver as a user of the reference's API would: its sources, the
    include/compat headers and -lpic_b200."""
    exe = Path(out_dir) / "compat_driver"
    cmd = [nvcc(), "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-I", str(ROOT / "include"), "-o", str(exe),
           str(SRC), "-L", str(LIBDIR), "-lpic_b200", "-Xlinker", f"-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError("driver build failed:\n" + r.stdout + r.stderr)
    return exe


def write_records(path: Path, arrays) -> None:
    with open(path, "wb") as f:
        for a in arrays:
            b = np.ascontiguousarray(a).tobytes()
            f.write(np.int64(len(b)).tobytes())
            f.write(b)


def read_records(path: Path, dtypes) -> list[np.ndarray]:
    out = []
    with open(path, "rb") as f:
        for dt in dtypes:
            nb = int(np.frombuffer(f.read(8), np.int64)[0])
            out.append(np.frombuffer(f.read(nb), dt).copy())
    return out


def run(exe: Path, mode: str, tmp: Path, arrays, dtypes, *extra: str, timeout: int = 300) -> list[np.ndarray]:
    fi, fo = Path(tmp) / f"{mode}.in", Path(tmp) / f"{mode}.out"
    write_records(fi, arrays)
    r = subprocess.run([str(exe), mode, str(fi), str(fo), *extra], capture_output=True, text=True, timeout=timeout)
    if r.returncode:
        raise RuntimeError(f"compat_driver {mode} failed ({r.returncode}):\n{r.stdout}{r.stderr}")
    return read_records(fo, dtypes)
