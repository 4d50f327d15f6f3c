"""Snapshot files: save_state (src/Erebus.jl:5718-5960).

The reference writes output_<timestep, 5 digits>.jld2 with jldsave every
savematstep timesteps (src/Erebus.jl:7106).  JLD2 is an HDF5 dialect and no
HDF5 writer is available to this package, so the same record is written as
output_<timestep, 5 digits>.npz: one array per key, the reference's key names
and order (src/Erebus.jl:5820-5955), node arrays (Ny, Nx) / (Ny1, Nx1) in
column-major order as in Julia, YNY* as bool and the marker arrays trimmed
to marknum.
"""
import os

import numpy as np

from .host import BOOL_GRID

# scalar keys in jldsave order (src/Erebus.jl:5822-5854); the value is the
# parameter or geometry attribute it comes from
SCALAR_KEYS = [
    ("Δtreaction", "dtreaction"), ("reaction_rate_coeff_mode", "reaction_rate_coeff_mode"),
    ("marker_property_mode", "marker_property_mode"), ("timesum", None), ("marknum", None),
    ("phim0", "phim0"), ("XWsolidm_init", "XWsolidm_init"), ("ratio_al", "ratio_al"),
    ("t_half_al", "t_half_al"), ("dsubgrids", "dsubgrids"), ("dsubgridt", "dsubgridt"),
    ("hr_al", "hr_al"), ("hr_fe", "hr_fe"), ("rplanet", "rplanet"), ("rcrust", "rcrust"),
    ("psurface", "psurface"), ("xsize", "xsize"), ("ysize", "ysize"),
]
GEOMETRY_KEYS = ["xcenter", "ycenter", "Nx", "Ny", "Nx1", "Ny1", "Nxm", "Nym", "dx", "dy",
                 "dxm", "dym"]
COORDINATE_KEYS = ["x", "y", "xvx", "yvx", "xvy", "yvy", "xp", "yp", "xxm", "yym"]
GRID_KEYS = [
    "ETA", "ETA0", "GGG", "EXY", "SXY", "SXY0", "wyx", "COH", "TEN", "FRI", "YNY",
    "RHOX", "RHOFX", "KX", "PHIX", "vx", "vxf", "RX", "qxD", "gx",
    "RHOY", "RHOFY", "KY", "PHIY", "vy", "vyf", "RY", "qyD", "gy",
    "RHO", "RHOCP", "ALPHA", "ALPHAF", "HR", "HA", "HS", "ETAP", "GGGP", "EXX", "SXX",
    "SXX0", "tk1", "tk2", "vxp", "vyp", "vxpf", "vypf", "pr", "pf", "ps", "pr0", "pf0",
    "ps0", "ETAPHI", "BETAPHI", "PHI", "APHI", "FI", "ETA5", "ETA00", "YNY5", "YNY00",
    "YNY_inv_ETA", "DSXY", "EII", "SII", "DSXX", "DMP", "DHP", "XWS",
]
MARKER_KEYS = [
    "XWsolidm0", "xm", "ym", "tm", "tkm", "sxxm", "sxym", "etavpm", "phim", "rhototalm",
    "rhocptotalm", "etatotalm", "hrtotalm", "ktotalm", "tkm_rhocptotalm",
    "etafluidcur_inv_kphim", "inv_gggtotalm", "fricttotalm", "cohestotalm", "tenstotalm",
    "rhofluidcur", "alphasolidcur", "alphafluidcur",
]


def _range(start, step, n):
    """Elements of the Julia range start:step:stop of length n."""
    return start + step * np.arange(n, dtype=np.float64)


def coordinates(g):
    """Node and marker-grid coordinates (src/constants.jl:40-47, 116-119)."""
    return {
        "x": _range(0.0, g.dx, g.Nx),
        "y": _range(0.0, g.dy, g.Ny),
        "xvx": _range(0.0, g.dx, g.Ny1),        # 0:dx:xsize+dy, Ny1 entries
        "yvx": _range(-g.dy / 2, g.dy, g.Nx1),
        "xvy": _range(-g.dx / 2, g.dx, g.Nx1),
        "yvy": _range(0.0, g.dy, g.Ny1),
        "xp": _range(-g.dx / 2, g.dx, g.Nx1),
        "yp": _range(-g.dy / 2, g.dy, g.Ny1),
        "xxm": _range(g.dxm / 2, g.dxm, g.Nxm),
        "yym": _range(g.dym / 2, g.dym, g.Nxm),  # SVector{Nxm} as in the reference
    }


def state_record(timestep, st):
    """The key -> array mapping save_state writes for HostState `st`."""
    p, g = st.p, st.g
    rec = {"timestep": np.int64(timestep), "dt": np.float64(st.dt)}
    for key, attr in SCALAR_KEYS:
        if key == "timesum":
            rec[key] = np.float64(st.timesum)
        elif key == "marknum":
            rec[key] = np.int64(st.marknum)
        else:
            rec[key] = np.asarray(getattr(p, attr))
    for key in GEOMETRY_KEYS:
        rec[key] = np.asarray(getattr(g, key))
    rec.update(coordinates(g))
    for key in GRID_KEYS:
        a = st.grid[key]
        rec[key] = a.astype(bool) if key in BOOL_GRID else a
    for key in MARKER_KEYS:
        rec[key] = st.m[key][: st.marknum]
    return rec


def output_file(output_path, timestep):
    return os.path.join(output_path, "output_%05d.npz" % timestep)


def save_state(output_path, timestep, st):
    """Writes output_<timestep>.npz for HostState `st` (save_state,
    src/Erebus.jl:5718-5960); returns the file name."""
    fid = output_file(output_path, timestep)
    np.savez(fid, **state_record(timestep, st))
    return fid


def load_state(fid):
    """The record of one snapshot file as {key: array}."""
    with np.load(fid) as z:
        return {k: z[k] for k in z.files}
