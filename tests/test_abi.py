"""The C-ABI library loads and exports every entry point its header
declares (CPU only: no compute call is made without a GPU)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


def _declared(header):
    with open(os.path.join(ROOT, "include", header)) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:solv_gpu|fv_gpu)_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    from programs_b200.solver import EXPORTS, lib
    L = lib()
    names = _declared("solv_gpu.h")
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) <= set(EXPORTS) | set(names)


def test_every_fv_symbol_is_exported():
    from programs_b200.solver import lib
    L = lib()
    names = _declared("fv_gpu.h")
    assert len(names) == 9
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_no_device_path():
    import torch
    from programs_b200.solver import GpuSolver, SolverError, lib
    L = lib()
    assert L.solv_gpu_status_string(0) == b"ok"
    assert L.solv_gpu_status_string(4) == b"bad input"
    with open(os.path.join(ROOT, "include", "solv_gpu.h")) as f:
        header = f.read()
    codes = [int(v) for v in re.findall(r"#define SOLV_GPU_[A-Z_]+ (\d+) +/\*", header)]
    assert len(codes) >= 8
    for code in codes:
        assert L.solv_gpu_status_string(code) != b"unknown status", code
    assert L.solv_gpu_status_string(99) == b"unknown status"
    if not torch.cuda.is_available():
        with pytest.raises(SolverError):
            GpuSolver(0)


def test_fortran_interface_module_names_match():
    """The iso_c_binding module binds exactly the exported C names."""
    f90 = open(os.path.join(ROOT, "programs_b200", "fortran", "solv_gpu_m.f90")).read()
    bound = set(re.findall(r"bind\s*\(\s*c\s*,\s*name\s*=\s*['\"](\w+)['\"]", f90, flags=re.I))
    from programs_b200.solver import lib
    L = lib()
    assert bound and all(hasattr(L, n) for n in bound)
