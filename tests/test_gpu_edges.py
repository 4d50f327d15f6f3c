"""GPU edge cases of the boundary: an empty marker set, markers beyond the
domain, and marker capacity exhausted by replenishment."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_no_markers_leaves_nodes(pkg, oracle, built_lib):
    """marknum 0: every weight sum is zero, so the node fields keep their
    previous (stale) values, as in compute_*_node_properties! (E:1991,
    E:2049, E:2173); the oracle agrees."""
    st = pkg.make_state("planetesimal_41")
    rng = np.random.default_rng(1)
    for k in ("ETA", "RHOX", "RHO", "tk1"):
        st.grid[k][:] = rng.random(st.grid[k].shape)
    st.marknum = 0
    so, sg = st.copy(), st.copy()
    sim = pkg.Simulation(sg)
    sim.markers_to_nodes(sg.timesum)
    sim.download()
    sim.close()
    oracle.Oracle(so).markers_to_nodes(so.timesum)
    for k in ("ETA", "RHOX", "RHO"):
        np.testing.assert_array_equal(sg.grid[k], so.grid[k], err_msg=k)
        np.testing.assert_array_equal(sg.grid[k], st.grid[k], err_msg=k)


def test_markers_outside_domain(pkg, oracle, built_lib):
    """Markers up to a cell beyond every edge clamp to the border cells
    (fix, E:1456) and scatter there, bit for bit as the oracle."""
    st = pkg.make_state("planetesimal_41")
    n = st.marknum
    g = st.g
    rng = np.random.default_rng(2)
    k = rng.choice(n, 500, replace=False)
    st.m["xm"][k] = rng.uniform(-g.dx, st.p.xsize + g.dx, k.size)
    st.m["ym"][k] = rng.uniform(-g.dy, st.p.ysize + g.dy, k.size)
    so, sg = st.copy(), st.copy()
    sim = pkg.Simulation(sg)
    sim.markers_to_nodes(sg.timesum)
    sim.download()
    sums = sim.download_sums()
    sim.close()
    oracle.Oracle(so).markers_to_nodes(so.timesum)
    for name in ("WTSUM", "WTXSUM", "WTYSUM", "WTPSUM", "RHOSUM", "ETASUM"):
        np.testing.assert_array_equal(sums[name], so.sums[name], err_msg=name)


def test_capacity_exhausted(pkg, built_lib):
    """Replenishment that needs more markers than the capacity fails with
    EREBUS_ECAPACITY rather than truncating."""
    st = pkg.make_state("planetesimal_41")
    n = st.marknum
    # empty a block of cells so replenishment must add markers
    g = st.g
    keep = ~((st.m["xm"][:n] > 20 * g.dx) & (st.m["xm"][:n] < 24 * g.dx))
    for k in st.m:
        st.m[k][: keep.sum()] = st.m[k][:n][keep]
    st.marknum = int(keep.sum())
    sim = pkg.Simulation(st, capacity=st.marknum)
    with pytest.raises(pkg.ErebusError) as e:
        sim.replenish(1)
    assert e.value.code == 4     # EREBUS_ECAPACITY
    sim.close()
