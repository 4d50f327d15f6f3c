"""The Julia package (erebus.jl_b200/julia) against the C ABI, checked by
parsing: Julia is not installed here, so the binding cannot run, but its
contract with the library can be verified.

- src/structs.jl is what gen_structs.py generates from the ctypes mirror
  (which tests/test_abi.py checks field by field against the header);
- every `ccall((:erebus_..., liberebus)` names a function the header declares
  and the built library exports, and every function the header declares is
  wrapped;
- the CLI's lists of the reference's setup results cover exactly the grid
  and marker arrays of the ABI structs, and the save_state list matches the
  reference's argument count (98 with the five scalars);
- brackets balance in each file.
"""
import importlib.util
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "erebus.jl_b200", "julia")
HEADER = os.path.join(ROOT, "include", "erebus_b200.h")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_structs",
                                                  os.path.join(JL, "gen_structs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _read(*p):
    with open(os.path.join(JL, *p)) as f:
        return f.read()


def _header_functions():
    src = open(HEADER).read()
    return set(re.findall(r"^(?:int|const char \*)\s*(erebus_\w+)\(", src, re.M))


def test_structs_generated_from_abi():
    assert _read("src", "structs.jl") == _gen().render()


def test_ccalls_match_header_and_library(built_lib):
    jl = _read("src", "ErebusB200.jl")
    called = set(re.findall(r"ccall\(\(:(erebus_\w+),\s*liberebus\)", jl))
    declared = _header_functions()
    assert called <= declared, called - declared
    assert declared <= called, declared - called
    for name in called:
        assert hasattr(built_lib, name), name


def _tuple(src, name):
    m = re.search(r"const %s = \(\s*(.*?)\n\)" % name, src, re.S)
    return re.findall(r":(\w+)", m.group(1))


def test_cli_lists_cover_the_abi():
    from erebus_b200 import abi
    cli = _read("run_simulation_b200.jl")
    grid = _tuple(cli, "GRID_SETUP") + _tuple(cli, "GRID_HELPERS")
    assert len(grid) == len(set(grid))
    assert set(grid) == set(abi.GRID_FIELDS)
    markers = set(_tuple(cli, "MARKER_SETUP") + _tuple(cli, "MARKER_HELPERS"))
    assert set(abi.MARKER_FIELDS) - markers == {"etasolidm_m"}   # library extension
    assert set(_tuple(cli, "DEFINE_MARKERS_ARGS")) <= markers
    save = _tuple(cli, "SAVE_STATE_ARRAYS")
    assert len(save) + 5 == 98
    assert set(save) <= set(grid) | markers


@pytest.mark.parametrize("path", [("src", "ErebusB200.jl"), ("src", "structs.jl"),
                                  ("run_simulation_b200.jl",)])
def test_brackets_balance(path):
    src = re.sub(r'"(?:[^"\\]|\\.)*"', '""', _read(*path))        # strings
    src = re.sub(r"#.*", "", src)                                   # comments
    for o, c in ("()", "[]", "{}"):
        assert src.count(o) == src.count(c), (path, o)
