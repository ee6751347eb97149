"""The C-ABI library loads and exports what include/pic_b200.h declares (CPU only: no compute
calls that need a device)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    txt = (ROOT / "include" / "pic_b200.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(pic_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from pic_cuda_b200 import _lib
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), name
    # the ctypes binding covers every declared entry point
    assert set(names) <= set(_lib.exported_symbols())


def test_struct_layout_matches_library():
    from pic_cuda_b200 import _lib
    _lib.check_abi()


def test_host_philox_matches_oracle(orc):
    from pic_cuda_b200 import _lib
    for ctr, key in [([1, 2, 3, 4], [5, 6]), ([0xDEADBEEF, 7, 0, 1], [1234, 0])]:
        assert _lib.philox4x32_10(ctr, key) == orc.philox(ctr, key)


def test_engine_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    from pic_cuda_b200 import _lib
    from pic_cuda_b200.engine import Engine
    try:
        Engine(0)
    except _lib.PicError as e:
        assert e.code == _lib.PIC_ERR_NO_DEVICE
    else:
        raise AssertionError("engine creation must fail without a device")


def test_config_validation_is_host_side():
    from pic_cuda_b200 import _lib, configs
    from pic_cuda_b200.engine import bytes_needed
    cfg = configs.plain_small()
    b = bytes_needed(cfg)
    assert b > 129 * 129 * 20
    cfg.nx = cfg.ny = 100  # not 2^k+1
    try:
        bytes_needed(cfg)
    except _lib.PicError as e:
        assert e.code == _lib.PIC_ERR_ARG
    else:
        raise AssertionError("bad grid accepted")


COMPAT_SYMBOLS = [
    "Grid2D::Grid2D(int, int, double, double)", "Grid2D::~Grid2D()", "Grid2D::debugGrid()",
    "Particles2D::Particles2D(int)", "Particles2D::~Particles2D()", "Particles2D::add_species(double, double)",
    "Particles2D::change_species(int, double, double)", "Particles2D::debugParticles(int)",
    "Particles2D::removeCollidedParticles()", "Boundaries2D::~Boundaries2D()",
    "Boundaries2D::add_wall(double, double, double, double)", "Boundaries2D::compile_walls()",
    "solve_multigrid(double*, double*, int, int, int, double, double)",
    "elasticCollisions(Particles2D&, double, double, cross_sections&)",
    "updateSimulationCUDA(Particles2D&, Grid2D&, Boundaries2D&, int&, double, int, SimulationTiming&)",
]


def test_library_exports_reference_host_api():
    """The drop-in classes and functions of include/compat are defined in libpic_b200.so."""
    import subprocess
    from pic_cuda_b200 import _lib
    so = _lib.lib()._name
    out = subprocess.run(["nm", "-DC", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    for sym in COMPAT_SYMBOLS:
        assert sym in out, sym
    assert "read_cross_section(" in out


def test_program_written_against_reference_headers_links(tmp_path):
    """A program using the reference's API (set-up of main.cu, updateSimulationCUDA,
    removeCollidedParticles, elasticCollisions, solve_multigrid) compiles against
    include/compat and links to libpic_b200.so."""
    import compat_io
    exe = compat_io.build_driver(tmp_path)
    assert exe.exists()


def test_embedded_solver_checks_its_arrays_on_the_host():
    """solve_embedded_f64 rejects host, mistyped or misshaped arrays before any device call."""
    import pytest
    import torch
    from pic_cuda_b200.engine import solve_embedded_f64
    a = torch.zeros((9, 9), dtype=torch.float64)
    m = torch.zeros((9, 9), dtype=torch.uint8)
    with pytest.raises(ValueError):
        solve_embedded_f64(a, a, m, None, 2, 0.1)            # host tensors
    with pytest.raises(ValueError):
        solve_embedded_f64(a, a, m.to(torch.int32), None, 2, 0.1)


class _FakeCudaTensor:
    """Stands in for a CUDA tensor on a given device index (no GPU is touched)."""

    def __init__(self, index, shape, dtype):
        import torch
        self.is_cuda = True
        self.device = torch.device("cuda", index)
        self.shape = shape
        self.dtype = dtype

    def is_contiguous(self):
        return True

    def data_ptr(self):
        raise AssertionError("a pointer was taken: the call got past validation")


def test_solver_bindings_reject_arrays_on_different_devices():
    """Arrays spread over two GPUs are rejected on the host, before a pointer is taken or a
    kernel launched (a kernel on one device would otherwise read the other's memory)."""
    import pytest
    import torch
    from pic_cuda_b200.engine import check_device_arrays, solve_embedded_f64, solve_multigrid_f64
    f64, u8 = torch.float64, torch.uint8
    a0, a1 = _FakeCudaTensor(0, (9, 9), f64), _FakeCudaTensor(1, (9, 9), f64)
    m0 = _FakeCudaTensor(0, (9, 9), u8)
    with pytest.raises(ValueError, match="one device"):
        solve_embedded_f64(a0, a1, m0, None, 2, 0.1)
    with pytest.raises(ValueError, match="one device"):
        solve_embedded_f64(a0, a0, m0, a1, 2, 0.1)
    with pytest.raises(ValueError, match="one device"):
        solve_multigrid_f64(a0, a1, 9, 9, 0, 0.1)
    with pytest.raises(ValueError, match="one device"):
        solve_multigrid_f64(a1, a0, 9, 9, 0, 0.1, static=True)
    with pytest.raises(ValueError):
        solve_multigrid_f64(a0, a0, 17, 17, 0, 0.1)               # shape does not match nx, ny
    with pytest.raises(ValueError):
        solve_multigrid_f64(a0, torch.zeros((9, 9), dtype=f64), 9, 9, 0, 0.1)  # host array
    assert check_device_arrays([("a", a1, f64, False), ("b", a1, f64, False)], (9, 9)) == torch.device("cuda", 1)
