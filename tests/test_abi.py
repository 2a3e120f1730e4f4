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
    assert len(names) == 12
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


def _c_params(header_src, name):
    m = re.search(r"\b" + name + r"\s*\(([^;{]*)\)\s*;", header_src, flags=re.S)
    assert m, name
    body = m.group(1).strip()
    return [] if body in ("", "void") else [p.strip() for p in body.split(",")]


def _f_dummies(f90_src):
    """bound C name -> [(dummy, attributes line)] for each interface body."""
    out = {}
    for m in re.finditer(r"function\s+\w+\s*\(([^)]*)\)\s*&?\s*bind\s*\(\s*c\s*,\s*name\s*=\s*'(\w+)'\s*\)"
                         r"(.*?)end\s+function", f90_src, flags=re.S | re.I):
        names = [a.strip() for a in m.group(1).replace("&", " ").split(",") if a.strip()]
        decls = [l.strip() for l in m.group(3).splitlines() if "::" in l]
        attrs = {}
        for d in decls:
            spec, vars_ = d.split("::", 1)
            for v in vars_.split(","):
                attrs[v.strip()] = spec.strip().lower()
        out[m.group(2)] = [(n, attrs.get(n, "")) for n in names]
    return out


def test_fortran_interfaces_match_the_c_declarations():
    """Arity and passing convention of every binding: C scalars by value;
    a C data pointer is an array passed by reference, or an address
    (c_ptr / c_intptr_t handle) passed by value; a pointer to a pointer is
    an address passed by value, or a handle variable passed by reference."""
    with open(os.path.join(ROOT, "include", "solv_gpu.h")) as f:
        header = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    with open(os.path.join(ROOT, "programs_b200", "fortran", "solv_gpu_m.f90")) as f:
        binds = _f_dummies(f.read())
    assert binds
    for cname, dummies in binds.items():
        params = _c_params(header, cname)
        assert len(params) == len(dummies), (cname, params, dummies)
        for cp, (dn, spec) in zip(params, dummies):
            stars = cp.count("*")
            by_value = "value" in spec
            address = "type(c_ptr)" in spec or "c_intptr_t" in spec
            if stars == 0:
                assert by_value and not address, (cname, cp, spec)
            elif stars == 1:
                assert (not by_value and "dimension" in spec) or (by_value and address), \
                    (cname, cp, spec)
            else:
                assert (by_value and "type(c_ptr)" in spec) or \
                    (not by_value and "c_intptr_t" in spec), (cname, cp, spec)


def test_fortran_by_reference_shims_report_through_status():
    """The gfortran-convention entry points (every argument by reference,
    the handle an integer(8) holding the context address) return their
    code in `status`: a null handle or a missing argument is BAD_INPUT,
    and without a device create reports DEVICE_ERROR and a zero handle."""
    import ctypes
    import torch
    from programs_b200.solver import lib
    L = lib()
    i64, i32, f64 = ctypes.c_int64, ctypes.c_int, ctypes.c_double
    st = i32(-1)
    h0 = i64(0)
    one, zero = i32(1), i32(0)
    red = f64(1e-10)
    buf = (ctypes.c_double * 8)()
    L.solv_gpu_cg_(ctypes.byref(h0), ctypes.byref(zero), ctypes.byref(red), ctypes.byref(one),
                   ctypes.byref(one), buf, buf, buf, ctypes.byref(zero), ctypes.byref(st))
    assert st.value == 4
    st.value = -1
    L.solv_gpu_bicg_(ctypes.byref(h0), None, ctypes.byref(red), ctypes.byref(one),
                     ctypes.byref(one), buf, buf, buf, ctypes.byref(zero), ctypes.byref(st))
    assert st.value == 4
    st.value = -1
    L.solv_gpu_destroy_(ctypes.byref(h0), ctypes.byref(st))
    assert st.value == 4
    if not torch.cuda.is_available():
        h = i64(12345)
        st.value = -1
        L.solv_gpu_create_(ctypes.byref(h), ctypes.byref(zero), ctypes.byref(st))
        assert st.value == 5 and h.value == 0


def test_ctypes_stubs_match_the_header_arity():
    """Every ctypes stub the Python layer declares (solver.py, fv.py,
    mesh.py) takes as many arguments as the C declaration it binds."""
    from programs_b200 import fv, mesh, solver
    L = solver.lib()
    fv._typed()
    M = mesh._lib()
    checked = 0
    for lib_, header in ((L, "solv_gpu.h"), (L, "fv_gpu.h"),
                         (M, os.path.join("..", "programs_b200", "csrc", "fvmesh.h"))):
        with open(os.path.join(ROOT, "include", header)) as f:
            src = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
        for name in set(re.findall(r"\b((?:solv_gpu|fv_gpu|fvm)_\w+)\s*\(", src)):
            fn = getattr(lib_, name, None)
            types = getattr(fn, "argtypes", None) if fn is not None else None
            if types is None:
                continue
            assert len(types) == len(_c_params(src, name)), name
            checked += 1
    assert checked >= 60, checked
