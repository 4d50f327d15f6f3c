"""GPU parity: every phase of the timestep, called through the C ABI, against
the CPU oracle on the same seeded inputs.

Tolerances: marker->node sums and node properties are compared bit for bit
(the device scatter keeps the reference's serial summation order); marker
gathers and stencils to 1e-12 relative (transcendental functions of the
device math library may differ from the host's by an ulp); linear-system
solutions to 1e-8 relative L2 per field (the oracle's SuperLU and the
device LU are different factorisations of the same system); marker
positions after RK4 to 1e-10 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = "planetesimal_41"


def rel_linf(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    d = np.abs(a - b)
    scale = np.max(np.abs(b)) if b.size else 0.0
    return float(np.max(d) / scale) if scale > 0 else float(np.max(d))


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


@pytest.fixture(scope="module")
def advanced(pkg, oracle):
    """A state advanced two oracle timesteps (non-zero stresses, moved and
    replenished markers, non-trivial pressures)."""
    st = pkg.make_state(CFG)
    o = oracle.Oracle(st)
    for ts in (1, 2):
        o.step(ts)
    return st


def _pair(pkg, oracle, st):
    so, sg = st.copy(), st.copy()
    return so, oracle.Oracle(so), sg, pkg.Simulation(sg)


def test_markers_to_nodes_bitexact(pkg, oracle, built_lib, advanced):
    so, o, sg, sim = _pair(pkg, oracle, advanced)
    o.markers_to_nodes(so.timesum)
    sim.markers_to_nodes(sg.timesum)
    sim.download()
    sums = sim.download_sums()
    for k in ["ETA0SUM", "ETASUM", "GGGSUM", "SXYSUM", "COHSUM", "TENSUM", "FRISUM",
              "WTSUM", "RHOXSUM", "KXSUM", "PHIXSUM", "RXSUM", "WTXSUM", "RHOYSUM",
              "RYSUM", "WTYSUM", "RHOSUM", "RHOCPSUM", "ALPHASUM", "HRSUM", "GGGPSUM",
              "SXXSUM", "TKSUM", "PHISUM", "WTPSUM"]:
        np.testing.assert_array_equal(sums[k], so.sums[k], err_msg=k)
    for k in ["ETA0", "ETA", "GGG", "SXY0", "COH", "TEN", "FRI", "YNY", "RHOX", "RHOFX",
              "KX", "PHIX", "RX", "RHOY", "KY", "RY", "RHO", "RHOCP", "ALPHA", "HR",
              "GGGP", "SXX0", "tk1", "PHI", "BETAPHI"]:
        np.testing.assert_array_equal(sg.grid[k], so.grid[k], err_msg=k)
    for k in ["rhototalm", "rhocptotalm", "etatotalm", "ktotalm", "tkm_rhocptotalm"]:
        n = so.marknum
        assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-14, k
    sim.close()


def test_gravity(pkg, oracle, built_lib, advanced):
    so, o, sg, sim = _pair(pkg, oracle, advanced)
    o.markers_to_nodes(so.timesum)
    sim.markers_to_nodes(sg.timesum)
    o.gravity()
    st = sim.gravity()
    sim.download()
    assert st.rel_residual <= 1e-10
    for k in ["FI", "gx", "gy"]:
        assert rel_l2(sg.grid[k], so.grid[k]) <= 1e-8, k
    sim.close()


def test_hydromech_assembly_matches_oracle(pkg, oracle, built_lib, advanced):
    import scipy.sparse as sp
    so, o, sg, sim = _pair(pkg, oracle, advanced)
    for s_ in (so,):
        pass
    o.markers_to_nodes(so.timesum)
    sim.markers_to_nodes(sg.timesum)
    o.gravity()
    sim.gravity()
    sim.download()
    # same grid state on both sides for the assembly check
    so.grid.update({k: v.copy(order="F") for k, v in sg.grid.items()})
    o._refresh()
    oracle.lib().oracle_bulk_viscosity(o.pP, o.pG)
    dt = 1.0e11
    A, b = o.hydromech_system(dt)
    rows, cols, vals, R = sim.export_hydromech(dt)
    n = A.shape[0]
    Ag = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    d = (Ag - A).tocoo()
    scale = np.maximum(abs(A).max(axis=1).toarray().ravel(), 1e-300)
    assert np.all(np.abs(d.data) <= 1e-12 * scale[d.row]), "Stokes-Darcy matrix"
    assert rel_linf(R, b) <= 1e-12
    sim.close()


def test_one_step_parity(pkg, oracle, built_lib, advanced):
    so, o, sg, sim = _pair(pkg, oracle, advanced)
    so_stats = o.step(3)
    gs = sim.step(3)
    sim.download()
    assert gs.titer == so_stats["titer"]
    assert gs.iplast_total == so_stats["iplast_total"]
    assert gs.marknum == so_stats["marknum"] == sg.marknum
    assert abs(gs.dt - so_stats["dt"]) <= 1e-10 * so_stats["dt"]
    assert gs.worst_rel_residual <= 1e-10
    n = so.marknum
    for k in ["xm", "ym"]:
        assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-10, k
    for k in ["tkm", "phim", "XWsolidm0"]:
        assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-8, k
    np.testing.assert_array_equal(sg.m["tm"][:n], so.m["tm"][:n])
    for k in ["vx", "vy", "pr", "pf", "qxD", "qyD", "tk2"]:
        assert rel_l2(sg.grid[k], so.grid[k]) <= 1e-8, k
    # the pressures traced back along the velocities (backtrace_pressures_rk4!,
    # E:5284-5496) and the P nodes' melt composition (E:1929-1939)
    for k in ["pr0", "pf0", "ps0", "XWS"]:
        assert rel_l2(sg.grid[k], so.grid[k]) <= 1e-8, k
    sim.close()


def test_first_steps_from_initial_state(pkg, oracle, built_lib):
    """Timesteps 1-3 from the initial marker set (timestep-1 special cases:
    tk2 == 0 in the reaction, BETAPHI = 0, the pressure copies)."""
    st = pkg.make_state(CFG)
    so, sg = st.copy(), st.copy()
    o = oracle.Oracle(so)
    sim = pkg.Simulation(sg)
    for ts in (1, 2, 3):
        a = o.step(ts)
        b = sim.step(ts)
        assert b.titer == a["titer"], ts
        assert b.marknum == a["marknum"], ts
    sim.download()
    n = so.marknum
    assert rel_linf(sg.m["xm"][:n], so.m["xm"][:n]) <= 1e-10
    assert rel_linf(sg.m["ym"][:n], so.m["ym"][:n]) <= 1e-10
    assert rel_linf(sg.m["tkm"][:n], so.m["tkm"][:n]) <= 1e-8
    assert rel_l2(sg.grid["tk2"], so.grid["tk2"]) <= 1e-8
    sim.close()


def test_replenish_matches_oracle(pkg, oracle, built_lib, advanced):
    """Markers displaced so that anchors empty out: the new markers, their
    order and copied fields match the oracle exactly."""
    st = advanced.copy()
    g = st.g
    n = st.marknum
    rng = np.random.default_rng(7)
    # push a band of markers out of the body centre region
    sel = np.where(np.abs(st.m["xm"][:n] - g.xcenter) < 3 * g.dxm)[0]
    st.m["xm"][sel] += rng.choice([-1.0, 1.0], size=sel.size) * 4 * g.dxm
    so, sg = st.copy(), st.copy()
    o = oracle.Oracle(so)
    sim = pkg.Simulation(sg)
    nn = o.L.oracle_replenish(o.pP, o.pM, so.marknum, so.capacity,
                              oracle._a(o.mdis), oracle._a(o.mnum), 5)
    so.marknum = int(nn)
    ng = sim.replenish(5)
    sim.download()
    assert ng == nn and ng > n
    for k in ["xm", "ym", "tm", "tkm", "phim", "sxxm", "etavpm"]:
        np.testing.assert_array_equal(sg.m[k][:ng], so.m[k][:ng], err_msg=k)
    sim.close()


def test_subgrid_diffusion_step(pkg, oracle, built_lib):
    """A timestep with subgrid stress and temperature diffusion switched on
    (dsubgrids, dsubgridt > 0; the reference's defaults are 0): the marker
    stresses, temperatures and positions and the stress and temperature
    changes on the nodes agree with the oracle as in the other step tests."""
    st = pkg.make_state(CFG)
    st.p.dsubgrids = 1e-21      # relaxation factors of order one at dt ~ 1e11 s
    st.p.dsubgridt = 1e-3
    o = oracle.Oracle(st)
    o.step(1)
    so, o, sg, sim = _pair(pkg, oracle, st)
    so_stats = o.step(2)
    gs = sim.step(2)
    sim.download()
    sim.close()
    assert gs.titer == so_stats["titer"]
    n = so.marknum
    assert sg.marknum == n
    for k in ["xm", "ym"]:
        assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-10, k
    for k in ["sxxm", "sxym", "tkm"]:
        assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-8, k
    for k in ["DSXX", "DSXY", "DT", "tk2"]:
        assert rel_l2(sg.grid[k], so.grid[k]) <= 1e-8, k


@pytest.mark.parametrize("mode,rmode", [(1, 1), (1, 2), (9, 3)])
def test_material_and_reaction_modes(pkg, oracle, built_lib, mode, rmode):
    """Temperature-dependent material laws (marker_property_mode 1:
    Hobbs/Touloukian heat capacity and conductivities, E:2272-2358) and the
    reaction-time modes 2 and 3 (E:2386-2389): two timesteps from the
    initial state against the oracle."""
    st = pkg.make_state(CFG)
    st.p.marker_property_mode = mode
    st.p.reaction_rate_coeff_mode = rmode
    so, o, sg, sim = _pair(pkg, oracle, st)
    for ts in (1, 2):
        a = o.step(ts)
        b = sim.step(ts)
        assert a["titer"] == b.titer, ts
    sim.download()
    sim.close()
    n = so.marknum
    assert sg.marknum == n
    for k in ["xm", "ym"]:
        assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-10, k
    for k in ["tkm", "phim", "XWsolidm0"]:
        assert rel_linf(sg.m[k][:n], so.m[k][:n]) <= 1e-8, k
    # (DMP is left out: near equilibrium (1 - RV) / dt is rounding noise of
    # order 1e-27 on both sides, E:2667)
    for k in ["vx", "pr", "pf", "tk2"]:
        assert rel_l2(sg.grid[k], so.grid[k]) <= 1e-8, k
