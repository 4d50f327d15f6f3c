"""The oracle's node->marker updates, melt composition, thermodynamic transfer
and pressure back-trace against re-expressions of the reference's own tests.

Each test restates one testset of test/runtests.jl (cited T:<line>): the
reference checks each function against a loop-by-loop "verification" taken
from the MATLAB codes the model comes from (HTM-planetary.m,
HTM-hydration.m, madcph.p), with rtol 1e-9.  Here the same verification is
written in Python and applied to the C restatement (oracle/erebus_oracle.c)
on inputs drawn, as the reference draws them, from the ranges its testsets
state; the grid is that of src/test_constants.jl (15 x 15 basic nodes over
14 km, four markers per cell).

The marker updates of simulation_loop (E:6945-7019) run in the oracle as one
pass, oracle_nodes_to_markers: viscosity (update_marker_viscosity!, E:774),
stress (update_marker_stress!, E:4354), temperature
(update_marker_temperature!, E:4782), porosity (update_marker_porosity!,
E:4822) and the melt composition on the P nodes
(update_p_nodes_melt_composition!, E:1929).  One call with independent
random inputs for each update checks all five against their testsets.
"""
import ctypes

import numpy as np
import pytest

from test_oracle_reference import G, L, P, _a, _interp_v, _ref  # noqa: F401

RTOL = 1e-9


def _fix(xx, yy, x0, y0, dx, dy, jlo, jhi, ilo, ihi):
    """Index of the upper-left node (1-based, clamped) and the four weights
    (i,j), (i+1,j), (i,j+1), (i+1,j+1) of the verifications."""
    j = np.clip(np.trunc((xx - x0) / dx).astype(np.int64) + 1, jlo, jhi)
    i = np.clip(np.trunc((yy - y0) / dy).astype(np.int64) + 1, ilo, ihi)
    dxmj = xx - (x0 + (j - 1) * dx)
    dymi = yy - (y0 + (i - 1) * dy)
    w = np.stack([(1 - dxmj / dx) * (1 - dymi / dy), (1 - dxmj / dx) * (dymi / dy),
                  (dxmj / dx) * (1 - dymi / dy), (dxmj / dx) * (dymi / dy)])
    return i, j, w


def _gather(A, i, j, w):
    return (A[i - 1, j - 1] * w[0] + A[i, j - 1] * w[1] + A[i - 1, j] * w[2] +
            A[i, j] * w[3])


def _markers_in(rng, G, n, margin_x, margin_y):
    """Markers drawn on a 0.1 m lattice from one cell outside the box
    (rand(rgen, -dx:0.1:x[end]+dx, marknum) in the reference tests)."""
    lo_x, hi_x = -margin_x, G.xsize + margin_x
    lo_y, hi_y = -margin_y, G.ysize + margin_y
    xm = lo_x + 0.1 * rng.integers(0, int(round((hi_x - lo_x) / 0.1)) + 1, n)
    ym = lo_y + 0.1 * rng.integers(0, int(round((hi_y - lo_y) / 0.1)) + 1, n)
    return xm, ym


def _nodes_to_markers(L, P, pkg, st, dt, timestep):
    rc = L.oracle_nodes_to_markers(_ref(P), _ref(st.markers_struct()), st.marknum,
                                   _ref(st.grid_struct()), _ref(st.sums_struct()), dt,
                                   timestep)
    assert rc == 0


@pytest.mark.parametrize("timestep", [1, 2])
def test_node_to_marker_updates(L, P, G, pkg, timestep):
    """update_marker_viscosity! (T:841-910), update_marker_stress!
    (T:5201-5270), update_marker_temperature! (T:5554-5600, timesteps 1 and
    2), update_marker_porosity! (T:5602-5653) and
    update_p_nodes_melt_composition! (T:3356-3422)."""
    rng = np.random.default_rng(841 + timestep)
    n = G.start_marknum
    st = pkg.HostState(P, capacity=n)
    st.marknum = n
    m, g = st.m, st.grid
    Ny, Nx, dx, dy = G.Ny, G.Nx, G.dx, G.dy
    # viscosity inputs (T:841-852)
    xv, yv = _markers_in(rng, G, n, dx, dy)
    tm = rng.integers(1, 4, n)
    tkm = P.tmfluidphase - 100 + 0.1 * rng.integers(
        0, int(round((P.tmsolidphase + 100 - (P.tmfluidphase - 100)) / 0.1)) + 1, n)
    etasolidm = np.array(list(P.etasolidm))
    etasolidmm = np.array(list(P.etasolidmm))
    ETA = rng.random((Ny, Nx))
    YNY = rng.random((Ny, Nx)) < 0.5
    # The viscosity, stress, temperature and porosity updates all read the
    # marker positions; the reference draws them separately per testset, and
    # every update uses only its own inputs, so one set of positions serves.
    m["xm"][:n], m["ym"][:n], m["tm"][:n] = xv, yv, tm
    m["tkm"][:n] = tkm
    m["etatotalm"][:n] = etasolidm[tm - 1]
    g["ETA"][...] = ETA
    g["YNY"][...] = YNY
    g["YNY_inv_ETA"][...] = YNY / ETA
    # stress inputs (T:5201-5210)
    sxxm, sxym = rng.random(n), rng.random(n)
    m["sxxm"][:n], m["sxym"][:n] = sxxm, sxym
    g["DSXX"][...] = rng.random((Ny + 1, Nx + 1))
    g["DSXY"][...] = rng.random((Ny, Nx))
    # temperature inputs (T:5557-5562)
    g["DT"][...] = rng.random((Ny + 1, Nx + 1))
    g["tk2"][...] = rng.random((Ny + 1, Nx + 1))
    # porosity inputs (T:5604-5612); the pass starts with phim = phinewm
    phim = rng.random(n)
    m["phinewm"][:n] = phim
    g["APHI"][...] = rng.random((Ny + 1, Nx + 1))
    dtm = P.dt_longest
    # melt composition input (T:3356-3369): XWsolidm0 = XWsolidm at the pass
    xw = rng.random(n)
    m["XWsolidm"][:n] = xw

    _nodes_to_markers(L, P, pkg, st, dtm, timestep)

    # viscosity (HTM-planetary.m line 1321ff)
    i, j, w = _fix(xv, yv, G.x[0], G.y[0], dx, dy, 1, Nx - 1, 1, Ny - 1)
    es = np.where(tkm > P.tmsolidphase, etasolidmm[tm - 1], etasolidm[tm - 1])
    etot = np.where(tm < 3, es, etasolidm[tm - 1])
    anyy = YNY[i - 1, j - 1] | YNY[i, j - 1] | YNY[i - 1, j] | YNY[i, j]
    with np.errstate(divide="ignore"):
        ev = 1.0 / _gather(YNY / ETA, i, j, w)
    etavpm_ver = np.where(anyy, np.where(ev >= etot, etot, ev), etot)
    np.testing.assert_allclose(m["etavpm"][:n], etavpm_ver, rtol=RTOL)
    # stress (HTM-planetary.m line 1495ff): P grid clamped to 2..N-1
    ip, jp, wp = _fix(xv, yv, G.xp[0], G.yp[0], dx, dy, 2, Nx - 1, 2, Ny - 1)
    np.testing.assert_allclose(m["sxxm"][:n], sxxm + _gather(g["DSXX"], ip, jp, wp),
                               rtol=RTOL)
    ib, jb, wb = _fix(xv, yv, G.x[0], G.y[0], dx, dy, 1, Nx - 1, 1, Ny - 1)
    np.testing.assert_allclose(m["sxym"][:n], sxym + _gather(g["DSXY"], ib, jb, wb),
                               rtol=RTOL)
    # temperature (HTM-planetary.m line 1805ff)
    i, j, w = _fix(xv, yv, G.xp[0], G.yp[0], dx, dy, 1, Nx, 1, Ny)
    tk_ver = _gather(g["tk2"], i, j, w) if timestep == 1 else tkm + _gather(g["DT"], i, j, w)
    np.testing.assert_allclose(m["tkm"][:n], tk_ver, rtol=RTOL)
    # porosity (rocks only; clamped to [phimin, phimax])
    aphim = _gather(g["APHI"], i, j, w)
    with np.errstate(over="ignore"):     # exp(APHI * dt_longest) overflows to Inf, as in
        ph = phim / ((1 - phim) * np.exp(aphim * dtm) + phim)   # the reference test
    ph = np.clip(ph, P.phimin, P.phimax)
    np.testing.assert_allclose(m["phim"][:n], np.where(tm < 3, ph, phim), rtol=RTOL)
    # melt composition on the P nodes (i2visHTM_hydration.m line 1547ff)
    xws = np.zeros((Ny + 1, Nx + 1))
    wts = np.zeros((Ny + 1, Nx + 1))
    for k, (di, dj) in enumerate(((0, 0), (1, 0), (0, 1), (1, 1))):
        np.add.at(xws, (i - 1 + di, j - 1 + dj), xw * w[k])
        np.add.at(wts, (i - 1 + di, j - 1 + dj), w[k])
    ver = np.where(wts > 0, xws / np.where(wts > 0, wts, 1.0), 0.0)
    np.testing.assert_allclose(g["XWS"], ver, rtol=RTOL)


def test_melt_composition_hook(L, P, G, pkg):
    """update_p_nodes_melt_composition! alone (T:3356-3422), markers over
    the P grid's extent plus one cell."""
    rng = np.random.default_rng(3356)
    n = G.start_marknum
    st = pkg.HostState(P, capacity=n)
    st.marknum = n
    xm, ym = _markers_in(rng, G, n, G.dx, G.dy)
    st.m["xm"][:n], st.m["ym"][:n] = xm, ym
    x0 = rng.random(n)
    st.m["XWsolidm0"][:n] = x0
    st.grid["XWS"][...] = rng.random(st.grid["XWS"].shape)
    L.oracle_melt_composition(_ref(P), _ref(st.markers_struct()), n,
                              _ref(st.grid_struct()), _ref(st.sums_struct()))
    i, j, w = _fix(xm, ym, G.xp[0], G.yp[0], G.dx, G.dy, 1, G.Nx, 1, G.Ny)
    xws = np.zeros((G.Ny1, G.Nx1))
    wts = np.zeros((G.Ny1, G.Nx1))
    for k, (di, dj) in enumerate(((0, 0), (1, 0), (0, 1), (1, 1))):
        np.add.at(xws, (i - 1 + di, j - 1 + dj), x0 * w[k])
        np.add.at(wts, (i - 1 + di, j - 1 + dj), w[k])
    ver = np.where(wts > 0, xws / np.where(wts > 0, wts, 1.0), 0.0)
    np.testing.assert_allclose(st.grid["XWS"], ver, rtol=RTOL)


def test_thermodynamic_xfer(L, P, G, pkg):
    """compute_thermodynamic_xfer! (T:3265-3354): marker values scattered to
    the P nodes (interpolate_add_to_grid!), then DMP = DMPSUM / WTPSUM and
    DHP = DHPSUM / WTPSUM where WTPSUM > 0, zero elsewhere."""
    rng = np.random.default_rng(3265)
    n = G.start_marknum
    xm, ym = _markers_in(rng, G, n, G.dx, G.dy)
    prop = rng.random((2, n)) * 1e3
    i, j, w = _fix(xm, ym, G.xp[0], G.yp[0], G.dx, G.dy, 1, G.Nx, 1, G.Ny)
    st = pkg.HostState(P, capacity=1)
    s = st.sums
    sums = {"DMPSUM": np.zeros((G.Ny1, G.Nx1)), "DHPSUM": np.zeros((G.Ny1, G.Nx1)),
            "WTPSUM": np.zeros((G.Ny1, G.Nx1))}
    # serial marker order, as interpolate_add_to_grid! adds
    for mk in range(n):
        for k, (di, dj) in enumerate(((0, 0), (1, 0), (0, 1), (1, 1))):
            r, c = i[mk] - 1 + di, j[mk] - 1 + dj
            sums["DMPSUM"][r, c] += prop[0, mk] * w[k, mk]
            sums["DHPSUM"][r, c] += prop[1, mk] * w[k, mk]
            sums["WTPSUM"][r, c] += w[k, mk]
    for k, v in sums.items():
        s[k][...] = v
    st.grid["DMP"][...] = rng.random((G.Ny1, G.Nx1))
    st.grid["DHP"][...] = rng.random((G.Ny1, G.Nx1))
    L.oracle_thermodynamic_xfer(_ref(P), _ref(st.sums_struct()), _ref(st.grid_struct()))
    wt = sums["WTPSUM"]
    safe = np.where(wt > 0, wt, 1.0)
    np.testing.assert_allclose(st.grid["DMP"], np.where(wt > 0, sums["DMPSUM"] / safe, 0.0),
                               rtol=RTOL)
    np.testing.assert_allclose(st.grid["DHP"], np.where(wt > 0, sums["DHPSUM"] / safe, 0.0),
                               rtol=RTOL)


def _backtrace_ver(G, vx, vy, p, dtm):
    """madcph.p line 2363ff as T:6133-6258 states it: every interior P node
    traced back over dtm with RK4 through the corrected velocity
    interpolation, then p sampled there bilinearly."""
    out = p.copy()
    for jj in range(2, G.Nx + 1):
        for ii in range(2, G.Ny + 1):
            xA, yA = G.xp[jj - 1], G.yp[ii - 1]
            xc, yc = xA, yA
            vxm, vym = [0.0] * 4, [0.0] * 4
            for rk in range(4):
                vxm[rk] = _interp_v(G, vx, xc, yc, True)
                vym[rk] = _interp_v(G, vy, xc, yc, False)
                if rk in (0, 1):
                    xc, yc = xA - dtm / 2 * vxm[rk], yA - dtm / 2 * vym[rk]
                elif rk == 2:
                    xc, yc = xA - dtm * vxm[rk], yA - dtm * vym[rk]
            vxe = 1 / 6 * (vxm[0] + 2 * vxm[1] + 2 * vxm[2] + vxm[3])
            vye = 1 / 6 * (vym[0] + 2 * vym[1] + 2 * vym[2] + vym[3])
            xc, yc = xA - dtm * vxe, yA - dtm * vye
            i, j, w = _fix(np.array([xc]), np.array([yc]), G.xp[0], G.yp[0], G.dx, G.dy,
                           1, G.Nx, 1, G.Ny)
            out[ii - 1, jj - 1] = _gather(p, i, j, w)[0]
    return out


def test_backtrace_pressures(L, P, G, pkg):
    """backtrace_pressures_rk4! (T:6112-6395): pr0 and ps0 traced with the
    solid velocity, pf0 with the fluid velocity; the boundary ring keeps the
    copies of pr, ps and pf."""
    rng = np.random.default_rng(6112)
    st = pkg.HostState(P, capacity=1)
    g = st.grid
    shp = (G.Ny1, G.Nx1)
    for k in ("vx", "vy", "vxf", "vyf"):
        g[k][...] = rng.random(shp) * 2e-9 - 1e-9
    for k in ("pr", "pf", "ps", "pr0", "pf0", "ps0"):
        g[k][...] = rng.random(shp) * 1e6
    pr, pf, ps = g["pr"].copy(), g["pf"].copy(), g["ps"].copy()
    dtm = 0.9
    assert L.oracle_backtrace_pressures(_ref(P), _ref(st.grid_struct()), dtm) == 0
    # the displacements are far below a cell here (as in the reference test);
    # the next test traces across cells
    np.testing.assert_allclose(g["pr0"], _backtrace_ver(G, g["vx"], g["vy"], pr, dtm),
                               rtol=RTOL)
    np.testing.assert_allclose(g["ps0"], _backtrace_ver(G, g["vx"], g["vy"], ps, dtm),
                               rtol=RTOL)
    np.testing.assert_allclose(g["pf0"], _backtrace_ver(G, g["vxf"], g["vyf"], pf, dtm),
                               rtol=RTOL)


def test_backtrace_pressures_long_trace(L, P, G, pkg):
    """The same verification with displacements of up to about two cells, so
    that the traced points cross cells, reach the corrected interpolation's
    both branches and leave the grid at its edges (clamped)."""
    rng = np.random.default_rng(6113)
    st = pkg.HostState(P, capacity=1)
    g = st.grid
    shp = (G.Ny1, G.Nx1)
    dtm = 1e11
    vmax = 2.0 * G.dx / dtm
    for k in ("vx", "vy", "vxf", "vyf"):
        g[k][...] = (rng.random(shp) * 2 - 1) * vmax
    for k in ("pr", "pf", "ps"):
        g[k][...] = rng.random(shp) * 1e6
    pr, pf, ps = g["pr"].copy(), g["pf"].copy(), g["ps"].copy()
    assert L.oracle_backtrace_pressures(_ref(P), _ref(st.grid_struct()), dtm) == 0
    np.testing.assert_allclose(g["pr0"], _backtrace_ver(G, g["vx"], g["vy"], pr, dtm),
                               rtol=RTOL)
    np.testing.assert_allclose(g["ps0"], _backtrace_ver(G, g["vx"], g["vy"], ps, dtm),
                               rtol=RTOL)
    np.testing.assert_allclose(g["pf0"], _backtrace_ver(G, g["vxf"], g["vyf"], pf, dtm),
                               rtol=RTOL)
