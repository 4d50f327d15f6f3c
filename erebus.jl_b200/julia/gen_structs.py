"""Writes src/structs.jl, the Julia mirrors of the C ABI's structs, from the
ctypes mirror (erebus_b200/abi.py, itself checked field by field against
include/erebus_b200.h by tests/test_abi.py).

    python erebus.jl_b200/julia/gen_structs.py

Every struct becomes an isbits `struct` with the C field order and types, so
`Ref(x)` passes it to `ccall` as the C struct.  Fixed arrays (double[3])
become NTuple{3, Float64}; pointers become Ptr{T}.
"""
import ctypes
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
OUT = os.path.join(HERE, "src", "structs.jl")

SCALARS = {ctypes.c_int32: "Int32", ctypes.c_int64: "Int64", ctypes.c_uint64: "UInt64",
           ctypes.c_double: "Float64", ctypes.c_uint8: "UInt8", ctypes.c_int: "Cint"}


def _abi():
    spec = importlib.util.spec_from_file_location("erebus_abi", os.path.join(PKG, "abi.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def julia_type(ct):
    if ct in SCALARS:
        return SCALARS[ct]
    if hasattr(ct, "_length_"):
        return "NTuple{%d, %s}" % (ct._length_, julia_type(ct._type_))
    if hasattr(ct, "_type_") and issubclass(ct, ctypes._Pointer):
        return "Ptr{%s}" % julia_type(ct._type_)
    raise TypeError("no Julia mirror for %r" % ct)


STRUCTS = ["ErebusParams", "ErebusMarkersHost", "ErebusGridHost", "ErebusSumsHost",
           "ErebusSolveStats", "ErebusStepStats", "ErebusFactorStats", "ErebusAdjointStats",
           "ErebusSolverOptions"]


def render():
    abi = _abi()
    out = ["# Generated by gen_structs.py from the ctypes mirror of",
           "# include/erebus_b200.h; do not edit by hand.", ""]
    for name in STRUCTS:
        cls = getattr(abi, name)
        out.append("struct %s" % name)
        for fname, ct in cls._fields_:
            out.append("    %s::%s" % (fname, julia_type(ct)))
        out.append("end")
        out.append("")
    out.append("const MARKER_FIELDS = (%s)" %
               ", ".join(":%s" % f for f, _ in abi.ErebusMarkersHost._fields_))
    out.append("const GRID_FIELDS = (%s)" %
               ", ".join(":%s" % f for f, _ in abi.ErebusGridHost._fields_))
    out.append("const SUM_FIELDS = (%s)" %
               ", ".join(":%s" % f for f, _ in abi.ErebusSumsHost._fields_))
    out.append("")
    return "\n".join(out)


if __name__ == "__main__":
    with open(OUT, "w") as f:
        f.write(render())
    sys.stdout.write("wrote %s\n" % OUT)
