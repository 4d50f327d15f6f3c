"""Comparison helpers shared by the GPU parity tests (test infrastructure)."""
import numpy as np

SOLUTION_FIELDS = ["vx", "vy", "pr", "pf", "qxD", "qyD", "tk2"]


def rel_linf(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    d = np.abs(a - b)
    scale = np.max(np.abs(b)) if b.size else 0.0
    return float(np.max(d) / scale) if scale > 0 else float(np.max(d) if d.size else 0.0)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


def assert_step_parity(sg, so, gs, ostats, pos_tol=1e-10, field_tol=1e-8, res_tol=1e-10,
                       dt_tol=1e-10, what=""):
    """One timestep of the device (state sg, ErebusStepStats gs) against the
    oracle (state so, its stats dict): the iteration counts and marker
    population exactly, dt to `dt_tol` relative, marker positions to
    `pos_tol` relative (max norm), marker temperature, porosity and water
    content to `field_tol`, the solution fields to `field_tol` relative L2,
    and every solve's final scaled residual to `res_tol`."""
    assert gs.titer == ostats["titer"], (what, gs.titer, ostats["titer"])
    assert gs.iplast_total == ostats["iplast_total"], (what, gs.iplast_total,
                                                      ostats["iplast_total"])
    assert gs.marknum == ostats["marknum"] == sg.marknum, (what, gs.marknum, ostats["marknum"])
    assert abs(gs.dt - ostats["dt"]) <= dt_tol * ostats["dt"], (what, gs.dt, ostats["dt"])
    assert gs.worst_rel_residual <= res_tol, (what, gs.worst_rel_residual)
    n = so.marknum
    for k in ["xm", "ym"]:
        e = rel_linf(sg.m[k][:n], so.m[k][:n])
        assert e <= pos_tol, (what, k, e)
    for k in ["tkm", "phim", "XWsolidm0"]:
        e = rel_linf(sg.m[k][:n], so.m[k][:n])
        assert e <= field_tol, (what, k, e)
    np.testing.assert_array_equal(sg.m["tm"][:n], so.m["tm"][:n], err_msg=what)
    for k in SOLUTION_FIELDS:
        e = rel_l2(sg.grid[k], so.grid[k])
        assert e <= field_tol, (what, k, e)
