"""The C ABI: header <-> ctypes mirror, exported symbols, host-only calls."""
import ctypes
import math
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "erebus_b200.h")


def header_structs():
    h = open(HEADER).read()
    out = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", h, re.S):
        body = re.sub(r"/\*.*?\*/", "", m.group(2), flags=re.S)
        names = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            rest = decl.split(None, 1)[1]
            for v in rest.split(","):
                v = v.strip().lstrip("*")
                names.append(re.sub(r"\[\d+\]", "", v))
        out[m.group(1)] = names
    return out


def header_functions():
    h = open(HEADER).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    return sorted(set(re.findall(r"\b(erebus_\w+)\s*\(", h)))


def test_ctypes_mirror_matches_header(pkg):
    hs = header_structs()
    for name in ["ErebusParams", "ErebusMarkersHost", "ErebusGridHost", "ErebusSumsHost",
                 "ErebusSolveStats", "ErebusStepStats", "ErebusSolverOptions"]:
        cls = getattr(pkg, name)
        assert [f[0] for f in cls._fields_] == hs[name], name


def test_library_exports_every_declared_symbol(pkg, built_lib):
    for fn in header_functions():
        assert hasattr(built_lib, fn), fn


def test_default_params_match_python(pkg, built_lib):
    p = pkg.ErebusParams()
    assert built_lib.erebus_default_params(ctypes.byref(p), 15, 15) == 0
    q = pkg.default_params(15, 15)
    for name, _ in p._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if hasattr(a, "__len__"):
            a, b = list(a), list(b)
            assert all((x == y) or (math.isnan(x) and math.isnan(y)) for x, y in zip(a, b)), name
        else:
            assert a == b, name


def test_check_params_rejects_bad_sets(pkg, built_lib):
    p = pkg.default_params(15, 15)
    assert built_lib.erebus_check_params(ctypes.byref(p)) == 0
    p.Ny = 17   # non-square
    assert built_lib.erebus_check_params(ctypes.byref(p)) == 1
    p = pkg.default_params(15, 15)
    p.marker_property_mode = 3
    assert built_lib.erebus_check_params(ctypes.byref(p)) == 1
    p = pkg.default_params(15, 15)
    p.dsubgrids = 1.0    # subgrid diffusion is part of the device path
    assert built_lib.erebus_check_params(ctypes.byref(p)) == 0
    p.dsubgridt = -1.0   # but a negative diffusion coefficient is not a valid set
    assert built_lib.erebus_check_params(ctypes.byref(p)) == 1


def test_create_fails_loudly_without_device(pkg, built_lib):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a CUDA device is present")
    st = pkg.make_state("planetesimal_41")
    with pytest.raises(pkg.ErebusError) as e:
        pkg.Simulation(st)
    assert e.value.code == 7   # EREBUS_ENODEVICE


def test_grid_layout_matches_library(pkg, built_lib):
    """The host grid block (HostState) and the device slab share one layout,
    so erebus_step_host copies the grid in one transfer."""
    import ctypes

    from erebus_b200.abi import GRID_FIELDS
    from erebus_b200.host import grid_layout
    p = pkg.config_params("planetesimal_141")
    off = (ctypes.c_int64 * len(GRID_FIELDS))()
    total = ctypes.c_int64()
    built_lib.erebus_grid_layout.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    assert built_lib.erebus_grid_layout(ctypes.byref(p), off, ctypes.byref(total)) == 0
    mine, tot = grid_layout(p)
    assert [mine[k] for k in GRID_FIELDS] == list(off) and tot == total.value
    st = pkg.HostState(p)
    base = st.grid[GRID_FIELDS[0]].ctypes.data
    assert all(st.grid[k].ctypes.data == base + mine[k] for k in GRID_FIELDS)
