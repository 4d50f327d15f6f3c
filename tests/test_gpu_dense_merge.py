"""GPU: the marker-order merges bit for bit against the oracle where nodes
gather more markers than one warp holds in shared memory (256).

Such nodes take the one-thread walk on lane 0 inside the warp-per-node merge
kernel.  With 9 x 9 markers per cell every interior node has ~324 markers, so
all interior nodes take it; with 8 x 8 an interior node has exactly 256 at
the start, and after a timestep has moved the markers some nodes hold more
and some fewer, so both paths run in the same launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SUMS = ["ETA0SUM", "ETASUM", "GGGSUM", "SXYSUM", "COHSUM", "TENSUM", "FRISUM", "WTSUM",
        "RHOXSUM", "KXSUM", "PHIXSUM", "RXSUM", "WTXSUM", "RHOYSUM", "RYSUM", "WTYSUM",
        "RHOSUM", "RHOCPSUM", "ALPHASUM", "HRSUM", "GGGPSUM", "SXXSUM", "TKSUM", "PHISUM",
        "WTPSUM"]
NODES = ["ETA0", "ETA", "GGG", "SXY0", "COH", "TEN", "FRI", "YNY", "RHOX", "RHOFX", "KX",
         "PHIX", "RX", "RHOY", "KY", "RY", "RHO", "RHOCP", "ALPHA", "HR", "GGGP", "SXX0",
         "tk1", "PHI", "BETAPHI"]


def max_markers_per_node(st):
    """Largest number of markers in the four cells around a basic node."""
    p, n = st.p, st.marknum
    dx, dy = p.xsize / (p.Nx - 1), p.ysize / (p.Ny - 1)
    j = np.clip((st.m["xm"][:n] // dx).astype(int), 0, p.Nx - 2)
    i = np.clip((st.m["ym"][:n] // dy).astype(int), 0, p.Ny - 2)
    cells = np.zeros((p.Ny + 1, p.Nx + 1), np.int64)
    np.add.at(cells, (i + 1, j + 1), 1)
    nodes = cells[:-1, :-1] + cells[1:, :-1] + cells[:-1, 1:] + cells[1:, 1:]
    return int(nodes.max())


def rel_linf(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def dense_state(pkg, oracle, mpc, advance):
    from erebus_b200.params import config_params
    p = config_params("planetesimal_41")
    p.Nx = p.Ny = 21
    p.Nxmc = p.Nymc = mpc
    st = pkg.make_state(p)
    if advance:
        oracle.Oracle(st).step(1)
    assert max_markers_per_node(st) > 256   # some nodes take the one-thread walk
    return st


@pytest.mark.parametrize("mpc,advance", [(9, False), (8, True)])
def test_dense_markers_to_nodes_bitexact(pkg, oracle, built_lib, mpc, advance):
    st = dense_state(pkg, oracle, mpc, advance)
    so, sg = st.copy(), st.copy()
    o, sim = oracle.Oracle(so), pkg.Simulation(sg)
    try:
        o.markers_to_nodes(so.timesum)
        sim.markers_to_nodes(sg.timesum)
        sim.download()
        sums = sim.download_sums()
        for k in SUMS:
            np.testing.assert_array_equal(sums[k], so.sums[k], err_msg=k)
        for k in NODES:
            np.testing.assert_array_equal(sg.grid[k], so.grid[k], err_msg=k)
    finally:
        sim.close()


def test_dense_step_parity(pkg, oracle, built_lib):
    """A whole timestep (reaction and melt merges included) on the 8 x 8
    state, against the oracle to the tolerances of the plain parity tests."""
    st = dense_state(pkg, oracle, 8, True)
    so, sg = st.copy(), st.copy()
    o, sim = oracle.Oracle(so), pkg.Simulation(sg)
    try:
        so_stats = o.step(2)
        gs = sim.step(2)
        sim.download()
        assert gs.titer == so_stats["titer"]
        assert gs.marknum == so_stats["marknum"] == sg.marknum
        n = so.marknum
        np.testing.assert_array_equal(sg.m["tm"][:n], so.m["tm"][:n])
        for k in ("xm", "ym"):
            assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-10, k
        for k in ("tkm", "phim", "XWsolidm0"):
            assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-8, k
        for k in ("vx", "vy", "pr", "pf", "tk2"):
            assert rel_l2(sg.grid[k], so.grid[k]) <= 1e-8, k
    finally:
        sim.close()
