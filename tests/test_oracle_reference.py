"""The oracle against re-expressions of the reference's own unit tests.

Julia is not available here, so the reference cannot be run to produce golden
outputs.  Its test suite (test/runtests.jl, cited T:<line>) checks each
function of the hot path against a "verification" computed with the
independent, loop-by-loop formulation of the MATLAB codes the model comes from
(HTM-planetary.m, HTM-hydration.m).  Each test below restates one of those
verifications in Python and applies it to the C restatement (the oracle,
oracle/erebus_oracle.c), with the reference test's tolerance unless stated:

- exact (==) where the reference tests with ==, and for the marker->node sums,
  which the oracle accumulates in the reference's serial order;
- rtol 1e-9 (1e-12 for the gravity matrix, 1e-4 for the RK4 temperature, 1e-6
  for the reaction) where the reference tests with those.

The reference compares whole matrices with `isapprox`, a norm-wise test; the
assembly tests here compare each entry against the largest entry of its row,
which is stricter.  The grid is that of src/test_constants.jl (15 x 15 basic
nodes over 14 km, four markers per cell).  Inputs are drawn from a seeded
numpy generator in the ranges the reference tests draw them from.
"""
import ctypes
import math

import numpy as np
import pytest

RTOL = 1e-9


@pytest.fixture(scope="module")
def L(oracle):
    return oracle.lib()


@pytest.fixture(scope="module")
def P(pkg):
    return pkg.params.default_params(15, 15)


@pytest.fixture(scope="module")
def G(P):
    """Grid geometry of src/test_constants.jl (C:15-124)."""
    class Geo:
        pass
    g = Geo()
    g.Nx, g.Ny = P.Nx, P.Ny
    g.Nx1, g.Ny1 = P.Nx + 1, P.Ny + 1
    g.xsize, g.ysize = P.xsize, P.ysize
    g.dx = P.xsize / (P.Nx - 1)
    g.dy = P.ysize / (P.Ny - 1)
    g.x = np.array([k * g.dx for k in range(g.Nx)])
    g.y = np.array([k * g.dy for k in range(g.Ny)])
    g.xvx = np.array([k * g.dx for k in range(g.Nx1)])
    g.yvx = np.array([-g.dy / 2 + k * g.dy for k in range(g.Ny1)])
    g.xvy = np.array([-g.dx / 2 + k * g.dx for k in range(g.Nx1)])
    g.yvy = np.array([k * g.dy for k in range(g.Ny1)])
    g.xp = np.array([-g.dx / 2 + k * g.dx for k in range(g.Nx1)])
    g.yp = np.array([-g.dy / 2 + k * g.dy for k in range(g.Ny1)])
    g.Nxm = (P.Nx - 1) * P.Nxmc
    g.Nym = (P.Ny - 1) * P.Nymc
    g.dxm = P.xsize / g.Nxm
    g.dym = P.ysize / g.Nym
    g.xxm = np.array([g.dxm / 2 + k * g.dxm for k in range(g.Nxm)])
    g.yym = np.array([g.dym / 2 + k * g.dym for k in range(g.Nym)])
    g.start_marknum = g.Nxm * g.Nym
    return g


def _ref(x):
    return ctypes.byref(x)


def _a(arr):
    return arr.ctypes.data_as(ctypes.c_void_p)


# (axis x, axis y, jmax, imax) of the four grids, with the clamp ranges of
# C:66-101 (jmin = imin = 1)
def _grids(G):
    return {0: (G.x, G.y, G.Nx - 1, G.Ny - 1),      # basic
            1: (G.xvx, G.yvx, G.Nx - 1, G.Ny),      # Vx
            2: (G.xvy, G.yvy, G.Nx, G.Ny - 1),      # Vy
            3: (G.xp, G.yp, G.Nx, G.Ny)}            # P


def _fix_ver(xx, yy, xa, ya, dx, dy, jmax, imax):
    """HTM-planetary.m line 395ff as T:1132-1152 states it (with / dx)."""
    j = int(math.trunc((xx - xa[0]) / dx)) + 1
    i = int(math.trunc((yy - ya[0]) / dy)) + 1
    j = 1 if j < 1 else (jmax if j > jmax else j)
    i = 1 if i < 1 else (imax if i > imax else i)
    return i, j


def _weights_ver(xm, ym, xa, ya, dx, dy, jmax, imax):
    """fix_basic of T:1393-1413, vectorised (1-based i, j)."""
    j = np.trunc((xm - xa[0]) / dx).astype(np.int64) + 1
    i = np.trunc((ym - ya[0]) / dy).astype(np.int64) + 1
    j = np.clip(j, 1, jmax)
    i = np.clip(i, 1, imax)
    dxmj = xm - xa[j - 1]
    dymi = ym - ya[i - 1]
    w = np.stack([(1 - dxmj / dx) * (1 - dymi / dy), (1 - dxmj / dx) * (dymi / dy),
                  (dxmj / dx) * (1 - dymi / dy), (dxmj / dx) * (dymi / dy)])
    return i, j, w


# ---------------------------------------------------------------------------
# fix / fix_weights (T:1127-1252, T:1597-1794)
# ---------------------------------------------------------------------------
def test_fix_all_grids(L, P, G):
    """T:1127-1252: every point of a dx/3 lattice from one cell outside the
    domain to one cell beyond it, on all four grids."""
    i_, j_ = ctypes.c_int(), ctypes.c_int()
    ny = int(round((G.ysize + 2 * G.dy) / (G.dy / 3)))
    nx = int(round((G.xsize + 2 * G.dx) / (G.dx / 3)))
    checked = 0
    for grid, (xa, ya, jmax, imax) in _grids(G).items():
        for a in range(ny + 1):
            yy = -G.dy + a * (G.dy / 3)
            for b in range(nx + 1):
                xx = -G.dx + b * (G.dx / 3)
                L.oracle_fix_grid(_ref(P), grid, xx, yy, _ref(i_), _ref(j_))
                assert (i_.value, j_.value) == _fix_ver(xx, yy, xa, ya, G.dx, G.dy,
                                                        jmax, imax), (grid, xx, yy)
                checked += 1
    assert checked == 4 * (nx + 1) * (ny + 1)


def test_fix_weights_corners_and_random(L, P, G):
    """T:1389-1596 (domain corners) and T:1597-1794 (10,000 random markers on a
    0.1 m lattice from the origin to one cell beyond the domain)."""
    rng = np.random.default_rng(1389)
    n = 10_000
    xm = rng.integers(0, int((G.x[-1] + G.dx) / 0.1) + 1, n) * 0.1
    ym = rng.integers(0, int((G.y[-1] + G.dy) / 0.1) + 1, n) * 0.1
    corners_x = np.array([-G.x[0], G.x[0], G.x[-1], G.x[-1]])
    corners_y = np.array([-G.y[0], G.y[-1], G.y[0], G.y[-1]])
    xm = np.concatenate([corners_x, xm])
    ym = np.concatenate([corners_y, ym])
    i_, j_ = ctypes.c_int(), ctypes.c_int()
    w = (ctypes.c_double * 4)()
    for grid, (xa, ya, jmax, imax) in _grids(G).items():
        iv, jv, wv = _weights_ver(xm, ym, xa, ya, G.dx, G.dy, jmax, imax)
        for m in range(xm.size):
            L.oracle_weights_grid(_ref(P), grid, xm[m], ym[m], _ref(i_), _ref(j_), w)
            assert (i_.value, j_.value) == (iv[m], jv[m]), (grid, m)
            np.testing.assert_allclose(np.array(w[:]), wv[:, m], rtol=RTOL,
                                       atol=1e-15, err_msg="grid %d m %d" % (grid, m))


# ---------------------------------------------------------------------------
# pointwise laws (T:939-1126, T:3424-3499)
# ---------------------------------------------------------------------------
def test_total_ktotal_kphi(L, P):
    rng = np.random.default_rng(939)
    assert L.oracle_total(0, 0, 0) == 0
    assert L.oracle_total(1, 0, 0) == 1
    assert L.oracle_total(0, 1, 0) == 0
    assert L.oracle_total(0, 0, 1) == 0
    assert L.oracle_total(1, 2, 0.5) == 1.5
    phim0 = P.phim0
    for _ in range(1000):
        s, f, phi = rng.random(3)
        assert L.oracle_total(s, f, phi) == pytest.approx(s * (1 - phi) + f * phi, rel=RTOL)
        # T:981-989 (HTM-planetary.m line 1761)
        a = s * (3 * phi - 2) + f * (1 - 3 * phi)
        kver = (s * f / 2 + a ** 2 / 16) ** 0.5 - a / 4
        assert L.oracle_ktotal(s, f, phi) == pytest.approx(kver, rel=RTOL)
        # T:1001-1008 (HTM-planetary.m line 333: eta_f / k(phi))
        k0, ph, etaf = rng.random(3)
        kphi = k0 * (ph / phim0) ** 3 / ((1 - ph) / (1 - phim0)) ** 2
        assert L.oracle_etaf_inv_kphi(_ref(P), k0, ph, etaf) == pytest.approx(
            etaf / kphi, rel=RTOL)


def test_radiogenic_heating(L, P, pkg):
    """T:1029-1060."""
    Q = lambda f, ratio, E, tau, t: f * ratio * E * math.exp(-t / tau) / tau
    assert L.oracle_Q_radiogenic(1., 2., 3., 4., 5.) == Q(1., 2., 3., 4., 5.)
    assert L.oracle_Q_radiogenic(1., 2., 3., 4., 0.) == Q(1., 2., 3., 4., 0.)
    hrs, hrf = (ctypes.c_double * 3)(), (ctypes.c_double * 3)()
    tau_al = P.t_half_al / math.log(2.0)
    tau_fe = P.t_half_fe / math.log(2.0)
    for al, fe in [(0, 0), (1, 0), (0, 1)]:
        p = pkg.params.default_params(15, 15)
        p.hr_al, p.hr_fe = al, fe
        L.oracle_radioactive_heating(_ref(p), 1000.0, hrs, hrf)
        u = [0.0, 0.0, 0.0]
        v = [0.0, 0.0, 0.0]
        if al:
            q = L.oracle_Q_radiogenic(p.f_al, p.ratio_al, p.E_al, tau_al, 1000.0)
            u = [q * p.rhosolidm[0], q * p.rhosolidm[1], 0.0]
        if fe:
            q = L.oracle_Q_radiogenic(p.f_fe, p.ratio_fe, p.E_fe, tau_fe, 1000.0)
            v = [q * p.rhofluidm[0], 0.0, 0.0]
        assert list(hrs) == u and list(hrf) == v, (al, fe)


def test_gibbs_enthalpy_reaction_constant(L, P):
    """T:1062-1125 (i2visHTM_hydration.m lines 612ff, 614ff, 623ff)."""
    rng = np.random.default_rng(1062)
    dVWD = P.MD / P.rhoDs + P.MH2O / P.rhoH2Of - (P.MD + P.MH2O) / P.rhoWs   # C:258
    for _ in range(200):
        phi = rng.random()
        XW0 = rng.random()
        tk, pf, XD0 = rng.random(3)
        dtr = L.oracle_dtreaction(_ref(P), tk, phi)
        for dt in (0.5 * dtr, 1.5 * dtr):
            g0 = P.dHWD - tk * P.dSWD + dVWD * pf + 8.314 * tk * math.log(XD0 / XW0)
            ver = g0 * (1 - dt / dtr) if dt < dtr else 0.0
            assert L.oracle_gibbs(_ref(P), tk, pf, XD0, XW0, dt, dtr) == pytest.approx(
                ver, rel=RTOL)
        Xs0 = rng.random()
        assert L.oracle_rel_enthalpy(_ref(P), Xs0, XW0) == pytest.approx(
            -Xs0 * XW0 * P.dHWD / (P.MD + P.MH2O), rel=RTOL)
        dG = rng.random()
        K = math.exp(-(P.dHWD - tk * P.dSWD + dVWD * pf - dG) / 8.314 / tk)
        assert L.oracle_reaction_constant(_ref(P), tk, pf, dG) == pytest.approx(K, rel=RTOL)


TS = lambda P: [170.0, P.tmfluidphase - 10.0, P.tmfluidphase - 3.0, P.tmfluidphase,
                P.tmfluidphase + 3.0, P.tmfluidphase + 10.0, 370.0, 470.0]


def test_fluid_and_solid_conductivity_heat_capacity(L, P, pkg):
    """T:3424-3479 (Hobbs's laws for marker_property_mode 1, constants
    otherwise)."""
    tm, Lf = P.tmfluidphase, P.Lf

    def rhocp_hobbs(T):
        if T >= 410:
            return P.rhoH2Of * (-4.67e4 + 333 * T - 0.731 * T ** 2 + 5.4e-4 * T ** 3)
        if T >= tm + 5:
            return P.rhoH2Of * 4200
        if T >= tm:
            return P.rhoH2Of * (4200.0 + 0.1 * Lf)
        if T >= tm - 5:
            return P.rhoH2Ofi * (7.67 * T + 0.1 * Lf)
        return P.rhoH2Ofi * 7.67 * T

    def kf_hobbs(T):
        if T >= 410:
            return -0.142 + 4.12e-3 * T - 5.01e-6 * T ** 2
        if T >= tm:
            return -0.581 + 6.34e-3 * T - 7.93e-6 * T ** 2
        return 0.465 + 488.0 / T

    p1 = pkg.params.default_params(15, 15)
    p1.marker_property_mode = 1
    p9 = pkg.params.default_params(15, 15)
    p9.marker_property_mode = 9
    for T in TS(P):
        assert L.oracle_rhocpfluid(_ref(p1), T) == pytest.approx(rhocp_hobbs(T), rel=RTOL)
        assert L.oracle_rhocpfluid(_ref(p9), T) == pytest.approx(P.rhocpfluidm[0], rel=RTOL)
        assert L.oracle_ksolid(_ref(p1), T) == pytest.approx(0.73 + 1293.0 / (T + 77.0),
                                                             rel=RTOL)
        assert L.oracle_ksolid(_ref(p9), T) == pytest.approx(P.ksolidm[0], rel=RTOL)
        assert L.oracle_kfluid(_ref(p1), T) == pytest.approx(kf_hobbs(T), rel=RTOL)
        assert L.oracle_kfluid(_ref(p9), T) == pytest.approx(P.kfluidm[0], rel=RTOL)


def test_reaction_time(L, P, pkg):
    """T:3481-3498, the four reaction-rate modes."""
    phi = 0.37
    ps = {}
    for mode in (1, 2, 3, 9):
        ps[mode] = pkg.params.default_params(15, 15)
        ps[mode].reaction_rate_coeff_mode = mode
    lcr = P.log_completion_rate
    for T in TS(P):
        assert L.oracle_dtreaction(_ref(ps[1]), T, phi) == pytest.approx(
            -lcr / (P.A_I * phi) * math.exp(P.b_I * (T - P.c_I) ** 2), rel=1e-12)
        assert L.oracle_dtreaction(_ref(ps[2]), T, phi) == pytest.approx(
            -lcr / (P.Sxo_B * phi) * 2.0 ** (-(T - P.To_B) / P.Tscl_B), rel=1e-12)
        assert L.oracle_dtreaction(_ref(ps[3]), T, phi) == pytest.approx(
            -lcr / (P.Sxo_T * phi * math.exp(P.Ea_T / P.RG * (1 / P.To_T - 1 / T))),
            rel=1e-12)
        assert L.oracle_dtreaction(_ref(ps[9]), T, phi) == P.dtreaction


def test_insulating_boundary(L, pkg):
    """T:3500-3510 on every array size from 3x3 to 10x10."""
    rng = np.random.default_rng(3500)
    for j in range(3, 11):
        for i in range(3, 11):
            p = pkg.params.default_params(j - 1, i - 1)     # Ny1 = i, Nx1 = j
            t = np.asfortranarray(rng.random((i, j)))
            L.oracle_insulating_bc(_ref(p), _a(t))
            assert np.array_equal(t[0, 1:j - 1], t[1, 1:j - 1])
            assert np.array_equal(t[i - 1, 1:j - 1], t[i - 2, 1:j - 1])
            assert np.array_equal(t[:, 0], t[:, 1])
            assert np.array_equal(t[:, j - 1], t[:, j - 2])


# ---------------------------------------------------------------------------
# marker -> node sums and node properties (T:2113-2629, T:2630-3264)
# ---------------------------------------------------------------------------
def _random_markers(pkg, P, G, rng, n):
    """Markers as setup_marker_properties(randomized=true) draws them (E:426):
    positions on a 0.1 m lattice from one cell outside the domain to one
    cell beyond it, properties uniform in [0, 1)."""
    st = pkg.HostState(P, capacity=n)
    for k, v in st.m.items():
        if k == "tm":
            v[:] = rng.integers(1, 4, n)
        else:
            v[:] = rng.random(n)
    st.m["xm"][:] = -G.dx + rng.integers(0, int((G.xsize + 2 * G.dx) / 0.1) + 1, n) * 0.1
    st.m["ym"][:] = -G.dy + rng.integers(0, int((G.ysize + 2 * G.dy) / 0.1) + 1, n) * 0.1
    st.m["inv_gggtotalm"][:] = 1.0 / (1e10 * (0.5 + rng.random(n)))
    st.marknum = n
    return st


SCATTER = {   # grid -> [(sum, marker property or None for the weight)]
    0: [("ETA0SUM", "etatotalm"), ("ETASUM", "etavpm"), ("GGGSUM", "inv_gggtotalm"),
        ("SXYSUM", "sxym"), ("COHSUM", "cohestotalm"), ("TENSUM", "tenstotalm"),
        ("FRISUM", "fricttotalm"), ("WTSUM", None)],
    1: [("RHOXSUM", "rhototalm"), ("RHOFXSUM", "rhofluidcur"), ("KXSUM", "ktotalm"),
        ("PHIXSUM", "phim"), ("RXSUM", "etafluidcur_inv_kphim"), ("WTXSUM", None)],
    2: [("RHOYSUM", "rhototalm"), ("RHOFYSUM", "rhofluidcur"), ("KYSUM", "ktotalm"),
        ("PHIYSUM", "phim"), ("RYSUM", "etafluidcur_inv_kphim"), ("WTYSUM", None)],
    3: [("GGGPSUM", "inv_gggtotalm"), ("SXXSUM", "sxxm"), ("RHOSUM", "rhototalm"),
        ("RHOCPSUM", "rhocptotalm"), ("ALPHASUM", "alphasolidcur"),
        ("ALPHAFSUM", "alphafluidcur"), ("HRSUM", "hrtotalm"), ("PHISUM", "phim"),
        ("TKSUM", "tkm_rhocptotalm"), ("WTPSUM", None)],
}


def _scatter_ver(G, st):
    """marker_to_{basic,vx,vy,P}_nodes! verification (T:2113-2629): weights of
    HTM-planetary.m line 373ff, accumulated node by node in marker order."""
    n = st.marknum
    out = {}
    for grid, (xa, ya, jmax, imax) in _grids(G).items():
        i, j, w = _weights_ver(st.m["xm"][:n], st.m["ym"][:n], xa, ya, G.dx, G.dy,
                               jmax, imax)
        shape = (G.Ny, G.Nx) if grid == 0 else (G.Ny1, G.Nx1)
        for name, prop in SCATTER[grid]:
            v = np.ones(n) if prop is None else st.m[prop][:n]
            acc = np.zeros(shape, order="F")
            # interpolate_add_to_grid! order: (i,j), (i+1,j), (i,j+1), (i+1,j+1)
            # per marker; np.add.at is unbuffered and keeps that order.
            ii = np.stack([i, i + 1, i, i + 1], axis=1).ravel() - 1
            jj = np.stack([j, j, j + 1, j + 1], axis=1).ravel() - 1
            vals = (v[:, None] * w.T).ravel()
            np.add.at(acc, (ii, jj), vals)
            out[name] = acc
    return out


def test_scatter_sums_exact(L, P, G, pkg):
    """Marker->node sums on all four grids, bit for bit (T:2113-2629 test the
    sums with ==)."""
    rng = np.random.default_rng(2113)
    st = _random_markers(pkg, P, G, rng, G.start_marknum)
    S = st.sums_struct()
    L.oracle_scatter_only(_ref(P), _ref(st.markers_struct()), st.marknum, _ref(S))
    ver = _scatter_ver(G, st)
    for name, acc in ver.items():
        np.testing.assert_array_equal(st.sums[name], acc, err_msg=name)


def test_node_properties(L, P, G, pkg):
    """compute_{basic,vx,vy,p}_node_properties! (T:2630-3264): node values are
    the weighted means of the sums (shear moduli harmonic), YNY where the
    visco-plastic mean is below the viscous one; rtol 1e-9."""
    rng = np.random.default_rng(2630)
    st = _random_markers(pkg, P, G, rng, G.start_marknum)
    # a few empty nodes, as the reference's randomised layouts have
    keep = ~((st.m["xm"] > 3 * G.dx) & (st.m["xm"] < 5 * G.dx)
             & (st.m["ym"] > 3 * G.dy) & (st.m["ym"] < 5 * G.dy))
    for k in st.m:
        st.m[k][: keep.sum()] = st.m[k][: st.marknum][keep]
    st.marknum = int(keep.sum())
    S = st.sums_struct()
    L.oracle_scatter_only(_ref(P), _ref(st.markers_struct()), st.marknum, _ref(S))
    sums = {k: v.copy() for k, v in st.sums.items()}
    L.oracle_node_properties(_ref(P), _ref(S), _ref(st.grid_struct()))
    g = st.grid

    def mean(num, wt):
        out = np.zeros_like(num)
        nz = wt > 0
        out[nz] = num[nz] / wt[nz]
        return out, nz

    wt = sums["WTSUM"]
    ETA0, nz = mean(sums["ETA0SUM"], wt)
    ETA, _ = mean(sums["ETASUM"], wt)
    assert (~nz).sum() > 0
    checks = {"ETA0": ETA0, "ETA": ETA, "SXY0": mean(sums["SXYSUM"], wt)[0],
              "COH": mean(sums["COHSUM"], wt)[0], "TEN": mean(sums["TENSUM"], wt)[0],
              "FRI": mean(sums["FRISUM"], wt)[0]}
    GGG = np.zeros_like(wt)
    GGG[nz] = 1.0 / (sums["GGGSUM"][nz] / wt[nz])
    checks["GGG"] = GGG
    for k, wname in (("X", "WTXSUM"), ("Y", "WTYSUM")):
        w = sums[wname]
        for f in ("RHO%s", "RHOF%s", "K%s", "PHI%s", "R%s"):
            checks[f % k] = mean(sums[(f % k) + "SUM"], w)[0]
    w = sums["WTPSUM"]
    for f in ("RHO", "RHOCP", "ALPHA", "ALPHAF", "HR", "PHI"):
        checks[f] = mean(sums[f + "SUM"], w)[0]
    checks["SXX0"] = mean(sums["SXXSUM"], w)[0]
    nzp = w > 0
    GGGP = np.zeros_like(w)
    GGGP[nzp] = 1.0 / (sums["GGGPSUM"][nzp] / w[nzp])
    checks["GGGP"] = GGGP
    tk1 = np.zeros_like(w)
    tk1[nzp] = sums["TKSUM"][nzp] / sums["RHOCPSUM"][nzp]
    checks["tk1"] = tk1
    BETAPHI = np.zeros_like(w)
    BETAPHI[nzp] = checks["PHI"][nzp] / GGGP[nzp]
    checks["BETAPHI"] = BETAPHI
    for k, v in checks.items():
        np.testing.assert_allclose(g[k], v, rtol=RTOL, atol=0, err_msg=k)
    np.testing.assert_array_equal(g["YNY"].astype(bool), nz & (ETA < ETA0))


# ---------------------------------------------------------------------------
# thermochemical reaction (T:3512-3731)
# ---------------------------------------------------------------------------
def test_thermochemical_reaction(L, P, G, pkg):
    """perform_thermochemical_reaction! against HTM-hydration.m line 558ff
    (T:3512-3731), timestep 1, iteration 3, dt = 0.9 x the constant reaction
    time; rtol 1e-6 as there."""
    rng = np.random.default_rng(3512)
    n = G.start_marknum
    st = pkg.HostState(P, capacity=n)
    m = st.m
    m["tm"][:] = rng.integers(1, 4, n)
    m["xm"][:] = -G.dx + rng.integers(0, int((G.xsize + 2 * G.dx) / 0.1) + 1, n) * 0.1
    m["ym"][:] = -G.dy + rng.integers(0, int((G.ysize + 2 * G.dy) / 0.1) + 1, n) * 0.1
    for k in ("XWsolidm0", "XWsolidm", "phim", "phinewm"):
        m[k][:] = rng.random(n)
    m["pfm0"][:] = 2700 + rng.integers(0, 6001, n) * 0.1
    st.marknum = n
    g = st.grid
    g["pf"][:] = 2700 + rng.integers(0, 6001, g["pf"].shape) * 0.1
    g["tk2"][:] = 263 + rng.integers(0, 471, g["tk2"].shape) * 0.1
    for k in ("DMP", "DHP"):
        g[k][:] = rng.random(g[k].shape)
    for k in ("DMPSUM", "DHPSUM", "WTPSUM"):
        st.sums[k][:] = rng.random(st.sums[k].shape)
    dt = 0.9 * P.dtreaction
    ver = {k: m[k][:n].copy() for k in ("XWsolidm0", "XWsolidm", "phim", "phinewm", "pfm0")}
    pf, tk2 = g["pf"].copy(), g["tk2"].copy()
    L.oracle_thermochemical_reaction(_ref(P), _ref(st.markers_struct()), n,
                                     _ref(st.grid_struct()), _ref(st.sums_struct()),
                                     dt, 1, 3)
    VDs, VWs = P.MD / P.rhoDs, (P.MD + P.MH2O) / P.rhoWs
    VH2Of, VH2Ofi = P.MH2O / P.rhoH2Of, P.MH2O / P.rhoH2Ofi
    dVWD = VDs + VH2Of - VWs                                               # C:258
    DMPSUM = np.zeros((G.Ny1, G.Nx1))
    DHPSUM = np.zeros((G.Ny1, G.Nx1))
    WTPSUM = np.zeros((G.Ny1, G.Nx1))
    dx, dy = G.dx, G.dy
    for k in range(n):
        if m["tm"][k] >= 3:
            continue
        x, y = m["xm"][k], m["ym"][k]
        i, j = _fix_ver(x, y, G.xp, G.yp, dx, dy, G.Nx, G.Ny)
        dxmj, dymi = x - G.xp[j - 1], y - G.yp[i - 1]
        w = [(1 - dxmj / dx) * (1 - dymi / dy), (1 - dxmj / dx) * (dymi / dy),
             (dxmj / dx) * (1 - dymi / dy), (dxmj / dx) * (dymi / dy)]
        cells = [(i - 1, j - 1), (i, j - 1), (i - 1, j), (i, j)]
        pfn = sum(pf[c] * wc for c, wc in zip(cells, w))
        tkn = sum(tk2[c] * wc for c, wc in zip(cells, w))
        pfn = max(pfn, 0)
        pfn = pfn * (1 - P.pfcoeff) + ver["pfm0"][k] * P.pfcoeff      # titer > 2
        ver["pfm0"][k] = pfn
        VH2O = VH2Of if tkn > P.tmfluidphase else VH2Ofi
        XW0 = ver["XWsolidm0"][k]
        ph = ver["phim"][k]
        XD0 = 1 - XW0
        Xf0 = ph * (XW0 * VWs + XD0 * VDs) / ((1 - ph) * VH2O + ph * (XW0 * VWs + XD0 * VDs))
        Xs0 = 1 - Xf0
        XH2O = (XW0 * Xs0 + Xf0) / (1 + XW0 * Xs0)
        XDt = 1 - XH2O
        rhos0 = (P.MD + P.MH2O * XW0) / (VWs * XW0 + VDs * XD0)
        rhof = P.rhoH2Of if tkn > P.tmfluidphase else P.rhoH2Ofi
        H0 = -Xs0 * XW0 * P.dHWD / (P.MD + P.MH2O)
        dG0 = P.dHWD - tkn * P.dSWD + dVWD * pfn + 8.314 * tkn * math.log(XD0 / XW0)
        dtr = L.oracle_dtreaction(_ref(P), tkn, ph)
        dG = dG0 * (1 - dt / dtr) if dt < dtr else 0
        K = math.exp(-(P.dHWD - tkn * P.dSWD + dVWD * pfn - dG) / 8.314 / tkn)
        XW1 = 1 / (K + 1)
        XD1 = 1 - XW1
        Xs1 = XDt / (1 - XDt * XW1)
        Xf1 = 1 - Xs1
        if not (0 < Xf1 < 1):
            continue
        phn = Xf1 * VH2O / (Xf1 * VH2O + Xs1 * (XW1 * VWs + XD1 * VDs))
        rhos = (P.MD + P.MH2O * XW1) / (VWs * XW1 + VDs * XD1)
        H1 = -Xs1 * XW1 * P.dHWD / (P.MD + P.MH2O)
        RV = (rhos * (1 - phn) + rhof * phn) / (rhos0 * (1 - ph) + rhof * ph)
        Gm = (rhos0 * RV * (1 - ph) - rhos * (1 - phn)) / dt
        DMm = (1 - RV) / dt
        DHm = Gm * (H1 - H0)
        ver["XWsolidm"][k] = XW1
        ver["phinewm"][k] = phn
        ver["XWsolidm0"][k] = XW1                  # timestep 1
        ver["phim"][k] = phn
        for c, wc in zip(cells, w):
            DMPSUM[c] += DMm * wc
            DHPSUM[c] += DHm * wc
            WTPSUM[c] += wc
    nz = WTPSUM > 0
    DMP = np.zeros_like(DMPSUM)
    DHP = np.zeros_like(DHPSUM)
    DMP[nz] = DMPSUM[nz] / WTPSUM[nz]
    DHP[nz] = DHPSUM[nz] / WTPSUM[nz]
    np.testing.assert_allclose(g["DMP"], DMP, rtol=1e-6, atol=1e-6 * np.abs(DMP).max())
    np.testing.assert_allclose(g["DHP"], DHP, rtol=1e-6, atol=1e-6 * np.abs(DHP).max())
    for k, v in ver.items():
        np.testing.assert_allclose(m[k][:n], v, rtol=1e-6, err_msg=k)


# ---------------------------------------------------------------------------
# linear systems (T:3733-3922, T:4094-4449, T:5377-5458)
# ---------------------------------------------------------------------------
def _dense(L_fn, P, st, dim, nmax, *extra):
    rows = np.zeros(nmax, np.int64)
    cols = np.zeros(nmax, np.int64)
    vals = np.zeros(nmax)
    R = np.zeros(dim)
    n = L_fn(_ref(P), _ref(st.grid_struct()), *extra, _a(rows), _a(cols), _a(vals), _a(R))
    A = np.zeros((dim, dim))
    np.add.at(A, (rows[:n], cols[:n]), vals[:n])
    return A, R


def _assert_rows_close(A, A_ver, rtol, what):
    scale = np.maximum(np.abs(A).max(axis=1), np.abs(A_ver).max(axis=1))
    bad = np.abs(A - A_ver) > rtol * scale[:, None]
    if bad.any():
        r, c = np.argwhere(bad)[0]
        raise AssertionError("%s: %d entries differ, first at (%d, %d): %r vs %r"
                             % (what, bad.sum(), r, c, A[r, c], A_ver[r, c]))
    # and the reference's own norm-wise isapprox
    assert np.linalg.norm(A - A_ver) <= rtol * max(np.linalg.norm(A), np.linalg.norm(A_ver))


def _gravity_ver(P, G, RHO):
    """HTM-planetary.m line 680ff (T:3757-3789)."""
    n = G.Nx1 * G.Ny1
    A = np.zeros((n, n))
    R = np.zeros(n)
    dx, dy = G.dx, G.dy
    for j in range(1, G.Nx1 + 1):
        for i in range(1, G.Ny1 + 1):
            gk = (j - 1) * G.Ny1 + i - 1
            rnode = ((G.xp[j - 1] - G.xsize / 2) ** 2 + (G.yp[i - 1] - G.ysize / 2) ** 2) ** 0.5
            if rnode > G.xsize / 2 or i == 1 or i == G.Ny1 or j == 1 or j == G.Nx1:
                A[gk, gk] = 1
                R[gk] = 0
            else:
                A[gk, gk - G.Ny1] = 1 / dx ** 2
                A[gk, gk - 1] = 1 / dy ** 2
                A[gk, gk] = -2 / dx ** 2 - 2 / dy ** 2
                A[gk, gk + 1] = 1 / dy ** 2
                A[gk, gk + G.Ny1] = 1 / dx ** 2
                R[gk] = 2 / 3 * 4 * P.G * math.pi * RHO[i - 1, j - 1]
    return A, R


def _potential_to_g(G, FI):
    gx = np.zeros((G.Ny1, G.Nx1))
    gy = np.zeros((G.Ny1, G.Nx1))
    gx[:, :G.Nx] = -(FI[:, 1:] - FI[:, :-1]) / G.dx
    gy[:G.Ny, :] = -(FI[1:, :] - FI[:-1, :]) / G.dy
    return gx, gy


def test_gravity_assembly_solve_process(L, P, G, pkg, oracle):
    """assemble_gravitational_lse! (T:3828-3880, rtol 1e-12),
    compute_gravity_solution! (T:3733-3826) and
    process_gravitational_solution! (T:3882-3921), rtol 1e-9."""
    rng = np.random.default_rng(3733)
    st = pkg.HostState(P, capacity=1)
    st.grid["RHO"][:] = rng.random((G.Ny1, G.Nx1)) * 7e3
    n = G.Nx1 * G.Ny1
    A, R = _dense(L.oracle_assemble_gravity, P, st, n, 5 * n)
    A_ver, R_ver = _gravity_ver(P, G, st.grid["RHO"])
    _assert_rows_close(A, A_ver, 1e-12, "gravity matrix")
    np.testing.assert_allclose(R, R_ver, rtol=1e-12, atol=0)
    # the solution, through the oracle's solve and processing
    o = oracle.Oracle(st)
    o.gravity()
    FI_ver = np.linalg.solve(A_ver, R_ver).reshape((G.Ny1, G.Nx1), order="F")
    gx_ver, gy_ver = _potential_to_g(G, FI_ver)
    sl = (slice(0, G.Ny), slice(0, G.Nx))
    for name, ver in (("FI", FI_ver), ("gx", gx_ver), ("gy", gy_ver)):
        np.testing.assert_allclose(st.grid[name][sl], ver[sl], rtol=RTOL,
                                   atol=1e-12 * np.abs(ver).max(), err_msg=name)
    # process alone, on a random solution vector
    SP = rng.random(n)
    L.oracle_process_gravity(_ref(P), _a(SP), _ref(st.grid_struct()))
    FI = SP.reshape((G.Ny1, G.Nx1), order="F")
    gx_ver, gy_ver = _potential_to_g(G, FI)
    np.testing.assert_array_equal(st.grid["FI"], FI)
    np.testing.assert_allclose(st.grid["gx"][sl], gx_ver[sl], rtol=RTOL)
    np.testing.assert_allclose(st.grid["gy"][sl], gy_ver[sl], rtol=RTOL)


def test_bulk_viscosity(L, P, G, pkg):
    """recompute_bulk_viscosity! against HTM-planetary.m line 771ff
    (T:3923-3951)."""
    rng = np.random.default_rng(3923)
    st = pkg.HostState(P, capacity=1)
    ETA = rng.random((G.Ny, G.Nx))
    PHI = rng.random((G.Ny1, G.Nx1))
    st.grid["ETA"][:] = ETA
    st.grid["PHI"][:] = PHI
    L.oracle_bulk_viscosity(_ref(P), _ref(st.grid_struct()))
    ETAP = np.zeros((G.Ny1, G.Nx1))
    ETAPHI = np.zeros((G.Ny1, G.Nx1))
    for i in range(2, G.Ny + 1):
        for j in range(2, G.Nx + 1):
            ETAP[i - 1, j - 1] = 1 / ((1 / ETA[i - 2, j - 2] + 1 / ETA[i - 1, j - 2]
                                       + 1 / ETA[i - 2, j - 1] + 1 / ETA[i - 1, j - 1]) / 4)
            ETAPHI[i - 1, j - 1] = P.etaphikoef * ETAP[i - 1, j - 1] / PHI[i - 1, j - 1]
    sl = (slice(0, G.Ny), slice(0, G.Nx))
    np.testing.assert_allclose(st.grid["ETAP"][sl], ETAP[sl], rtol=RTOL)
    np.testing.assert_allclose(st.grid["ETAPHI"][sl], ETAPHI[sl], rtol=RTOL)


def _hydro_ver(P, G, f, dt):
    """Stokes-Darcy matrix and right-hand side of HTM-planetary.m line 779ff and
    HTM-hydration.m line 707ff, as T:4146-4443 state them."""
    Nx, Ny, Nx1, Ny1, dx, dy = G.Nx, G.Ny, G.Nx1, G.Ny1, G.dx, G.dy
    n = 6 * Nx1 * Ny1
    A = np.zeros((n, n))
    R = np.zeros(n)
    K = P.Kcont
    vxleft, vxright = P.strainrate * P.xsize / 2, -P.strainrate * P.xsize / 2
    vytop, vybottom = -P.strainrate * P.ysize / 2, P.strainrate * P.ysize / 2
    ETA, ETAP, GGG, GGGP = f["ETA"], f["ETAP"], f["GGG"], f["GGGP"]
    SXY0, SXX0, RHOX, RHOY = f["SXY0"], f["SXX0"], f["RHOX"], f["RHOY"]
    gx, gy = f["gx"], f["gy"]

    def E(a, i, j):
        return a[i - 1, j - 1]

    def visc(e, gg, i, j):
        return E(e, i, j) * E(gg, i, j) * dt / (E(gg, i, j) * dt + E(e, i, j))

    def old(s, e, gg, i, j):
        return E(s, i, j) * E(e, i, j) / (E(gg, i, j) * dt + E(e, i, j))

    def pbound(i, j):
        return ((i == 2 and 2 <= j <= Nx) or (i == Ny and 2 <= j <= Nx)
                or (j == 2 and 2 <= i <= Ny) or (j == Nx and 2 <= i <= Ny))

    for j in range(1, Nx1 + 1):
        for i in range(1, Ny1 + 1):
            kvx = ((j - 1) * Ny1 + i - 1) * 6
            kvy, kpm, kqx, kqy, kpf = kvx + 1, kvx + 2, kvx + 3, kvx + 4, kvx + 5
            # x-Stokes
            if i == 1 or i == Ny1 or j == 1 or j == Nx or j == Nx1:
                if j == Nx1:
                    A[kvx, kvx] = 1
                    R[kvx] = 0
                if j == 1:
                    A[kvx, kvx] = 1
                    R[kvx] = vxleft
                if j == Nx:
                    A[kvx, kvx] = 1
                    R[kvx] = vxright
                if i == 1 and 1 < j < Nx:
                    A[kvx, kvx] = 1
                    A[kvx, kvx + 6] = P.bctop
                    R[kvx] = 0
                if i == Ny1 and 1 < j < Nx:
                    A[kvx, kvx] = 1
                    A[kvx, kvx - 6] = P.bcbottom
                    R[kvx] = 0
            else:
                E1, E2 = visc(ETA, GGG, i - 1, j), visc(ETA, GGG, i, j)
                EP1, EP2 = visc(ETAP, GGGP, i, j), visc(ETAP, GGGP, i, j + 1)
                S1, S2 = old(SXY0, ETA, GGG, i - 1, j), old(SXY0, ETA, GGG, i, j)
                X1, X2 = old(SXX0, ETAP, GGGP, i, j), old(SXX0, ETAP, GGGP, i, j + 1)
                dRdx = (E(RHOX, i, j + 1) - E(RHOX, i, j - 1)) / 2 / dx
                dRdy = (E(RHOX, i + 1, j) - E(RHOX, i - 1, j)) / 2 / dy
                g_ = E(gx, i, j)
                A[kvx, kvx - Ny1 * 6] = EP1 / dx ** 2
                A[kvx, kvx - 6] = E1 / dy ** 2
                A[kvx, kvx] = -(EP1 + EP2) / dx ** 2 - (E1 + E2) / dy ** 2 - dRdx * g_ * dt
                A[kvx, kvx + 6] = E2 / dy ** 2
                A[kvx, kvx + Ny1 * 6] = EP2 / dx ** 2
                A[kvx, kvy] = EP1 / dx / dy - E2 / dx / dy - dRdy * g_ * dt / 4
                A[kvx, kvy + Ny1 * 6] = -EP2 / dx / dy + E2 / dx / dy - dRdy * g_ * dt / 4
                A[kvx, kvy - 6] = -EP1 / dx / dy + E1 / dx / dy - dRdy * g_ * dt / 4
                A[kvx, kvy + Ny1 * 6 - 6] = EP2 / dx / dy - E1 / dx / dy - dRdy * g_ * dt / 4
                A[kvx, kpm] = K / dx
                A[kvx, kpm + Ny1 * 6] = -K / dx
                R[kvx] = -E(RHOX, i, j) * g_ - (S2 - S1) / dy - (X2 - X1) / dx
            # y-Stokes
            if j == 1 or j == Nx1 or i == 1 or i == Ny or i == Ny1:
                if i == Ny1:
                    A[kvy, kvy] = 1
                    R[kvy] = 0
                if i == 1:
                    A[kvy, kvy] = 1
                    R[kvy] = vytop
                if i == Ny:
                    A[kvy, kvy] = 1
                    R[kvy] = vybottom
                if j == 1 and 1 < i < Ny:
                    A[kvy, kvy] = 1
                    A[kvy, kvy + 6 * Ny1] = P.bcleft
                    R[kvy] = 0
                if j == Nx1 and 1 < i < Ny:
                    A[kvy, kvy] = 1
                    A[kvy, kvy - 6 * Ny1] = P.bcright
                    R[kvy] = 0
            else:
                E1, E2 = visc(ETA, GGG, i, j - 1), visc(ETA, GGG, i, j)
                EP1, EP2 = visc(ETAP, GGGP, i, j), visc(ETAP, GGGP, i + 1, j)
                S1, S2 = old(SXY0, ETA, GGG, i, j - 1), old(SXY0, ETA, GGG, i, j)
                Y1 = -old(SXX0, ETAP, GGGP, i, j)
                Y2 = -old(SXX0, ETAP, GGGP, i + 1, j)
                dRdx = (E(RHOY, i, j + 1) - E(RHOY, i, j - 1)) / 2 / dx
                dRdy = (E(RHOY, i + 1, j) - E(RHOY, i - 1, j)) / 2 / dy
                g_ = E(gy, i, j)
                A[kvy, kvy - Ny1 * 6] = E1 / dx ** 2
                A[kvy, kvy - 6] = EP1 / dy ** 2
                A[kvy, kvy] = -(EP1 + EP2) / dy ** 2 - (E1 + E2) / dx ** 2 - dRdy * g_ * dt
                A[kvy, kvy + 6] = EP2 / dy ** 2
                A[kvy, kvy + Ny1 * 6] = E2 / dx ** 2
                A[kvy, kvx] = EP1 / dx / dy - E2 / dx / dy - dRdx * g_ * dt / 4
                A[kvy, kvx + 6] = -EP2 / dx / dy + E2 / dx / dy - dRdx * g_ * dt / 4
                A[kvy, kvx - Ny1 * 6] = -EP1 / dx / dy + E1 / dx / dy - dRdx * g_ * dt / 4
                A[kvy, kvx + 6 - Ny1 * 6] = EP2 / dx / dy - E1 / dx / dy - dRdx * g_ * dt / 4
                A[kvy, kpm] = K / dy
                A[kvy, kpm + 6] = -K / dy
                R[kvy] = -E(RHOY, i, j) * g_ - (S2 - S1) / dx - (Y2 - Y1) / dy
            # total-pressure continuity
            c = K / (1 - E(f["PHI"], i, j)) * (1 / E(f["ETAPHI"], i, j)
                                              + E(f["BETAPHI"], i, j) / dt)
            rc = ((E(f["pr0"], i, j) - E(f["pf0"], i, j)) / (1 - E(f["PHI"], i, j))
                  * E(f["BETAPHI"], i, j) / dt)
            outer = i == 1 or j == 1 or i == Ny1 or j == Nx1
            if outer or pbound(i, j):
                A[kpm, kpm] = 1
                R[kpm] = 0
                if pbound(i, j):
                    A[kpm, kpm] = 1 * K
                    R[kpm] = P.psurface
            else:
                A[kpm, kvx - Ny1 * 6] = -1 / dx
                A[kpm, kvx] = 1 / dx
                A[kpm, kvy - 6] = -1 / dy
                A[kpm, kvy] = 1 / dy
                A[kpm, kpm] = c
                A[kpm, kpf] = -c
                R[kpm] = rc + E(f["DMP"], i, j)
            # x-Darcy
            if i == 1 or i == Ny1 or j == 1 or j == Nx or j == Nx1:
                A[kqx, kqx] = 1
                R[kqx] = 0
                if i == 1 and 1 < j < Nx:
                    A[kqx, kqx + 6] = P.bcftop
                if i == Ny1 and 1 < j < Nx:
                    A[kqx, kqx - 6] = P.bcfbottom
            else:
                A[kqx, kqx] = E(f["RX"], i, j)
                A[kqx, kpf] = -K / dx
                A[kqx, kpf + Ny1 * 6] = K / dx
                R[kqx] = E(f["RHOFX"], i, j) * E(gx, i, j)
            # y-Darcy
            if j == 1 or j == Nx1 or i == 1 or i == Ny or i == Ny1:
                A[kqy, kqy] = 1
                R[kqy] = 0
                if j == 1 and 1 < i < Ny:
                    A[kqy, kqy + 6 * Ny1] = P.bcfleft
                if j == Nx1 and 1 < i < Ny:
                    A[kqy, kqy - 6 * Ny1] = P.bcfright
            else:
                A[kqy, kqy] = E(f["RY"], i, j)
                A[kqy, kpf] = -K / dy
                A[kqy, kpf + 6] = K / dy
                R[kqy] = E(f["RHOFY"], i, j) * E(gy, i, j)
            # fluid-pressure continuity; the "real" boundary rows of the fluid
            # pressure exclude the corners of the j = 2 and j = Nx columns
            real_f = ((i == 2 and 2 <= j <= Nx) or (i == Ny and 2 <= j <= Nx)
                      or (j == 2 and 2 < i < Ny) or (j == Nx and 2 < i < Ny))
            if outer or pbound(i, j):
                A[kpf, kpf] = 1
                R[kpf] = 0
                if real_f:
                    A[kpf, kpf] = 1 * K
                    R[kpf] = P.psurface
            else:
                A[kpf, kqx - Ny1 * 6] = -1 / dx
                A[kpf, kqx] = 1 / dx
                A[kpf, kqy - 6] = -1 / dy
                A[kpf, kqy] = 1 / dy
                A[kpf, kpm] = -c
                A[kpf, kpf] = c
                R[kpf] = -rc
    return A, R


def test_hydromechanical_assembly(L, P, G, pkg):
    """assemble_hydromechanical_lse! (T:4094-4449) on random node fields in
    the reference test's ranges, dt = dt_longest."""
    rng = np.random.default_rng(4094)
    st = pkg.HostState(P, capacity=1)
    g = st.grid
    ranges = {"ETA": 1e16, "ETAP": 1e16, "GGG": 1e10, "GGGP": 1e10, "SXY0": 1e4,
              "SXX0": 1e4, "RHOX": 1e4, "RHOY": 1e4, "RHOFX": 1e4, "RHOFY": 1e4,
              "RX": 1e39, "RY": 1e39, "ETAPHI": 1e15, "BETAPHI": 1e-10, "PHI": 1.0,
              "gx": 1.0, "gy": 1.0, "pr0": 1e5, "pf0": 1e5, "DMP": 1e5}
    for k, s in ranges.items():
        g[k][:] = rng.random(g[k].shape) * s
    dt = P.dt_longest
    n = 6 * G.Nx1 * G.Ny1
    A, R = _dense(L.oracle_assemble_hydromech, P, st, n, 12 * n, dt)
    A_ver, R_ver = _hydro_ver(P, G, g, dt)
    _assert_rows_close(A, A_ver, RTOL, "Stokes-Darcy matrix")
    np.testing.assert_allclose(R, R_ver, rtol=RTOL, atol=RTOL * np.abs(R_ver).max())


def _thermal_ver(P, G, f, dt):
    """HTM-planetary.m line 1618ff (T:5393-5454)."""
    Nx1, Ny1, dx, dy = G.Nx1, G.Ny1, G.dx, G.dy
    n = Nx1 * Ny1
    A = np.zeros((n, n))
    R = np.zeros(n)

    def E(a, i, j):
        return f[a][i - 1, j - 1]

    for j in range(1, Nx1 + 1):
        for i in range(1, Ny1 + 1):
            gk = (j - 1) * Ny1 + i - 1
            if i == 1 or i == Ny1 or j == 1 or j == Nx1:
                if i == 1 and 1 < j < Nx1:
                    A[gk, gk], A[gk, gk + 1], R[gk] = 1, -1, 0
                if i == Ny1 and 1 < j < Nx1:
                    A[gk, gk], A[gk, gk - 1], R[gk] = 1, -1, 0
                if j == 1:
                    A[gk, gk], A[gk, gk + Ny1], R[gk] = 1, -1, 0
                if j == Nx1:
                    A[gk, gk], A[gk, gk - Ny1], R[gk] = 1, -1, 0
            else:
                Kx1, Kx2 = E("KX", i, j - 1), E("KX", i, j)
                Ky1, Ky2 = E("KY", i - 1, j), E("KY", i, j)
                A[gk, gk - Ny1] = -Kx1 / dx ** 2
                A[gk, gk - 1] = -Ky1 / dy ** 2
                A[gk, gk] = E("RHOCP", i, j) / dt + (Kx1 + Kx2) / dx ** 2 + (Ky1 + Ky2) / dy ** 2
                A[gk, gk + 1] = -Ky2 / dy ** 2
                A[gk, gk + Ny1] = -Kx2 / dx ** 2
                R[gk] = (E("RHOCP", i, j) / dt * E("tk1", i, j) + E("HR", i, j)
                         + E("HA", i, j) + E("HS", i, j) + E("DHP", i, j))
    return A, R


def test_thermal_assembly(L, P, G, pkg):
    """assemble_thermal_lse! (T:5377-5458)."""
    rng = np.random.default_rng(5377)
    st = pkg.HostState(P, capacity=1)
    dt = rng.random()
    for k in ("tk1", "RHOCP", "KX", "KY", "HR", "HA", "HS", "DHP"):
        st.grid[k][:] = rng.random(st.grid[k].shape)
    n = G.Nx1 * G.Ny1
    A, R = _dense(L.oracle_assemble_thermal, P, st, n, 6 * n, dt)
    A_ver, R_ver = _thermal_ver(P, G, st.grid, dt)
    _assert_rows_close(A, A_ver, RTOL, "thermal matrix")
    np.testing.assert_allclose(R, R_ver, rtol=RTOL, atol=0)


# ---------------------------------------------------------------------------
# velocities, rotation, RK4 (T:5655-6110)
# ---------------------------------------------------------------------------
def test_velocities_and_rotation(L, P, G, pkg):
    """compute_velocities! (HTM-planetary.m line 1879ff, T:5655-5739) and
    compute_rotation_rate! (line 1942ff, T:5741-5757)."""
    rng = np.random.default_rng(5655)
    st = pkg.HostState(P, capacity=1)
    g = st.grid
    for k in ("vx", "vy", "vxf", "vyf"):
        g[k][:] = rng.random(g[k].shape)
    L.oracle_velocities(_ref(P), _ref(st.grid_struct()))
    L.oracle_rotation_rate(_ref(P), _ref(st.grid_struct()))
    Nx, Ny = G.Nx, G.Ny
    vxleft, vxright = P.strainrate * P.xsize / 2, -P.strainrate * P.xsize / 2
    vytop, vybottom = -P.strainrate * P.ysize / 2, P.strainrate * P.ysize / 2

    def xnode(v, top, bottom):
        o = np.zeros((G.Ny1, G.Nx1))
        o[1:Ny, 1:Nx] = (v[1:Ny, 1:Nx] + v[1:Ny, 0:Nx - 1]) / 2
        o[0, 1:Nx - 1] = -top * o[1, 1:Nx - 1]
        o[Ny, 1:Nx - 1] = -bottom * o[Ny - 1, 1:Nx - 1]
        o[:, 0] = 2 * vxleft - o[:, 1]
        o[:, Nx] = 2 * vxright - o[:, Nx - 1]
        return o

    def ynode(v, left, right):
        o = np.zeros((G.Ny1, G.Nx1))
        o[1:Ny, 1:Nx] = (v[1:Ny, 1:Nx] + v[0:Ny - 1, 1:Nx]) / 2
        o[1:Ny - 1, 0] = -left * o[1:Ny - 1, 1]
        o[1:Ny - 1, Nx] = -right * o[1:Ny - 1, Nx - 1]
        o[0, :] = 2 * vytop - o[1, :]
        o[Ny, :] = 2 * vybottom - o[Ny - 1, :]
        return o

    np.testing.assert_allclose(g["vxp"], xnode(g["vx"], P.bctop, P.bcbottom), rtol=RTOL)
    np.testing.assert_allclose(g["vyp"], ynode(g["vy"], P.bcleft, P.bcright), rtol=RTOL)
    np.testing.assert_allclose(g["vxpf"], xnode(g["vxf"], P.bcftop, P.bcfbottom), rtol=RTOL)
    np.testing.assert_allclose(g["vypf"], ynode(g["vyf"], P.bcfleft, P.bcfright), rtol=RTOL)
    wyx = 0.5 * ((g["vy"][:Ny, 1:Nx + 1] - g["vy"][:Ny, :Nx]) / G.dx
                 - (g["vx"][1:Ny + 1, :Nx] - g["vx"][:Ny, :Nx]) / G.dy)
    np.testing.assert_allclose(g["wyx"], wyx, rtol=RTOL)


def _interp_v(G, v, x, y, along_x):
    """Second-order corrected velocity interpolation of HTM-planetary.m line
    1947ff (T:5870-5940), for one point."""
    dx, dy, Nx, Ny = G.dx, G.dy, G.Nx, G.Ny
    if along_x:
        i, j = _fix_ver(x, y, G.xvx, G.yvx, dx, dy, Nx - 1, Ny)
        dxmj, dymi = x - G.xvx[j - 1], y - G.yvx[i - 1]
        V = lambda a, b: v[a - 1, b - 1]
        v13 = V(i, j) * (1 - dxmj / dx) + V(i, j + 1) * dxmj / dx
        v24 = V(i + 1, j) * (1 - dxmj / dx) + V(i + 1, j + 1) * dxmj / dx
        q = (dxmj / dx - 0.5) ** 2 / 2
        if dxmj / dx >= 0.5:
            if j < Nx - 1:
                v13 += q * (V(i, j) - 2 * V(i, j + 1) + V(i, j + 2))
                v24 += q * (V(i + 1, j) - 2 * V(i + 1, j + 1) + V(i + 1, j + 2))
        elif j > 1:
            v13 += q * (V(i, j - 1) - 2 * V(i, j) + V(i, j + 1))
            v24 += q * (V(i + 1, j - 1) - 2 * V(i + 1, j) + V(i + 1, j + 1))
        return (1 - dymi / dy) * v13 + (dymi / dy) * v24
    i, j = _fix_ver(x, y, G.xvy, G.yvy, dx, dy, Nx, Ny - 1)
    dxmj, dymi = x - G.xvy[j - 1], y - G.yvy[i - 1]
    V = lambda a, b: v[a - 1, b - 1]
    v12 = V(i, j) * (1 - dymi / dy) + V(i + 1, j) * dymi / dy
    v34 = V(i, j + 1) * (1 - dymi / dy) + V(i + 1, j + 1) * dymi / dy
    q = (dymi / dy - 0.5) ** 2 / 2
    if dymi / dy >= 0.5:
        if i < Ny - 1:
            v12 += q * (V(i, j) - 2 * V(i + 1, j) + V(i + 2, j))
            v34 += q * (V(i, j + 1) - 2 * V(i + 1, j + 1) + V(i + 2, j + 1))
    elif i > 1:
        v12 += q * (V(i - 1, j) - 2 * V(i, j) + V(i + 1, j))
        v34 += q * (V(i - 1, j + 1) - 2 * V(i, j + 1) + V(i + 1, j + 1))
    return (1 - dxmj / dx) * v12 + (dxmj / dx) * v34


def _bilinear(G, a, x, y, grid):
    xa, ya, jmax, imax = _grids(G)[grid]
    i, j = _fix_ver(x, y, xa, ya, G.dx, G.dy, jmax, imax)
    dxmj, dymi = x - xa[j - 1], y - ya[i - 1]
    dx, dy = G.dx, G.dy
    wij = (1 - dxmj / dx) * (1 - dymi / dy)
    wi1j = (1 - dxmj / dx) * (dymi / dy)
    wij1 = (dxmj / dx) * (1 - dymi / dy)
    wi1j1 = (dxmj / dx) * (dymi / dy)
    return a[i - 1, j - 1] * wij + a[i, j - 1] * wi1j + a[i - 1, j] * wij1 + a[i, j] * wi1j1


def _rk4(G, vx, vy, x0, y0, h):
    vxs, vys = [], []
    x, y = x0, y0
    for rk in range(4):
        vxs.append(_interp_v(G, vx, x, y, True))
        vys.append(_interp_v(G, vy, x, y, False))
        c = (0.5, 0.5, 1.0, None)[rk]
        if c is not None:
            x, y = x0 + h * c * vxs[rk], y0 + h * c * vys[rk]
    vxe = (vxs[0] + 2 * vxs[1] + 2 * vxs[2] + vxs[3]) / 6
    vye = (vys[0] + 2 * vys[1] + 2 * vys[2] + vys[3]) / 6
    return vxe, vye


def test_move_markers_rk4(L, P, G, pkg):
    """move_markers_rk4! against HTM-planetary.m line 1947ff (T:5759-6110):
    positions rtol 1e-12, stresses exactly, temperature rtol 1e-4 (the
    reference's tolerances).  The markers sit on the regular marker lattice
    plus 10,000 more at the origin, as there."""
    rng = np.random.default_rng(5759)
    dtm = 0.9
    n = G.start_marknum + 10_000
    st = pkg.HostState(P, capacity=n)
    m = st.m
    k = np.arange(G.start_marknum)
    m["xm"][:G.start_marknum] = G.dxm / 2 + (k // G.Nym) * G.dxm
    m["ym"][:G.start_marknum] = G.dym / 2 + (k % G.Nym) * G.dym
    m["tm"][:] = rng.integers(1, 4, n)
    m["tkm"][:] = 263 + rng.integers(0, 471, n) * 0.1
    m["phim"][:] = P.phimin + rng.integers(0, int((P.phimax - P.phimin) / 1e-4), n) * 1e-4
    m["sxym"][:] = rng.random(n)
    m["sxxm"][:] = rng.random(n)
    st.marknum = n
    g = st.grid
    for key in ("vx", "vy", "vxf", "vyf"):
        g[key][:] = rng.random(g[key].shape)
    g["tk2"][:] = 263 + rng.integers(0, 471, g["tk2"].shape) * 0.1
    g["wyx"][:] = rng.random(g["wyx"].shape)
    before = {key: m[key][:n].copy() for key in ("xm", "ym", "tkm", "sxxm", "sxym")}
    L.oracle_move_markers_rk4(_ref(P), _ref(st.markers_struct()), n,
                              _ref(st.grid_struct()), dtm)
    rcs = np.asarray(list(P.rhocpsolidm))
    rcf = np.asarray(list(P.rhocpfluidm))
    for q in range(n):
        x0, y0 = before["xm"][q], before["ym"][q]
        tks0 = _bilinear(G, g["tk2"], x0, y0, 3)
        om = _bilinear(G, g["wyx"], x0, y0, 0)
        th = dtm * om
        sxx, sxy = before["sxxm"][q], before["sxym"][q]
        # Julia's x^2 with a literal exponent is x*x (Base.literal_pow)
        c, s = math.cos(th), math.sin(th)
        sxx_new = sxx * (c * c) - sxx * (s * s) - sxy * math.sin(2 * th)
        sxy_new = sxx * math.sin(2 * th) + sxy * math.cos(2 * th)
        assert m["sxxm"][q] == sxx_new and m["sxym"][q] == sxy_new, q
        vxe, vye = _rk4(G, g["vx"], g["vy"], x0, y0, dtm)
        x1, y1 = x0 + dtm * vxe, y0 + dtm * vye
        assert m["xm"][q] == pytest.approx(x1, rel=1e-12), q
        assert m["ym"][q] == pytest.approx(y1, rel=1e-12), q
        # backtrace with the fluid velocity to the fluid temperature
        vxe, vye = _rk4(G, g["vxf"], g["vyf"], x1, y1, -dtm)
        tkf0 = _bilinear(G, g["tk2"], x1 - dtm * vxe, y1 - dtm * vye, 3)
        t = int(m["tm"][q]) - 1
        ph, tk = m["phim"][q], before["tkm"][q]
        ver = (((1 - ph) * tk * rcs[t] + ph * (tk + tkf0 - tks0) * rcf[t])
               / ((1 - ph) * rcs[t] + ph * rcf[t]))
        assert m["tkm"][q] == pytest.approx(ver, rel=1e-4), q


# ---------------------------------------------------------------------------
# replenish (T:6396-6598)
# ---------------------------------------------------------------------------
def test_replenish(L, P, G, pkg):
    """replenish_markers! without jitter against HTM-planetary.m line 2491ff
    (T:6396-6598): the start_marknum markers fill only the top-left quarter,
    every empty marker-lattice node within five cells of a marker receives a
    copy of its nearest marker at the node itself; all properties exact."""
    rng = np.random.default_rng(6396)
    p = pkg.params.default_params(15, 15)
    p.random_markers = 0
    n = G.start_marknum
    cap = 4 * n
    st = pkg.HostState(p, capacity=cap)
    m = st.m
    for k, v in m.items():
        if k == "tm":
            v[:n] = rng.integers(1, 4, n)
        elif k != "etasolidm_m":
            v[:n] = rng.random(n)
    m["xm"][:n] = -G.dx + rng.integers(0, int((G.x[-1] / 2 + G.dx) / 0.1) + 1, n) * 0.1
    m["ym"][:n] = -G.dy + rng.integers(0, int((G.y[-1] / 2 + G.dy) / 0.1) + 1, n) * 0.1
    st.marknum = n
    before = {k: v[:n].copy() for k, v in m.items()}
    Nxm, Nym = G.Nxm, G.Nym
    mdis = np.zeros(Nxm * Nym)
    mnum = np.zeros(Nxm * Nym, np.int64)
    n_new = L.oracle_replenish(_ref(p), _ref(st.markers_struct()), n, cap, _a(mdis),
                               _a(mnum), 1)
    # verification
    md = np.full((Nym, Nxm), 1e30)
    mn = np.zeros((Nym, Nxm), np.int64)
    xm, ym = before["xm"], before["ym"]
    for q in range(n):
        i, j = _fix_ver(xm[q], ym[q], G.xxm, G.yym, G.dxm, G.dym, Nxm - 1, Nym - 1)
        for di, dj in ((0, 0), (1, 0), (0, 1), (1, 1)):
            a, b = i - 1 + di, j - 1 + dj
            d = ((xm[q] - G.xxm[b]) ** 2 + (ym[q] - G.yym[a]) ** 2) ** 0.5
            if d < md[a, b]:
                md[a, b] = d
                mn[a, b] = q + 1
    dii, djj = 5 * p.Nxmc, 5 * p.Nymc
    added = []
    for j in range(Nxm):
        for i in range(Nym):
            if mn[i, j] != 0:
                continue
            win = mn[max(i - dii, 0):i + dii + 1, max(j - djj, 0):j + djj + 1]
            cand = win.ravel(order="F")
            cand = cand[cand > 0]
            if cand.size == 0:
                continue
            d = ((xm[cand - 1] - G.xxm[j]) ** 2 + (ym[cand - 1] - G.yym[i]) ** 2) ** 0.5
            best = cand[int(np.argmin(d))]        # first strict minimum, loop order
            mn[i, j] = -best
            added.append((G.xxm[j], G.yym[i], best - 1))
    assert n_new == n + len(added)
    src = np.array([a[2] for a in added], np.int64)
    np.testing.assert_array_equal(m["xm"][n:n_new], [a[0] for a in added])
    np.testing.assert_array_equal(m["ym"][n:n_new], [a[1] for a in added])
    for k in ("tm", "tkm", "phim", "sxxm", "sxym", "etavpm", "phinewm", "pfm0",
              "XWsolidm", "XWsolidm0"):
        np.testing.assert_array_equal(m[k][:n], before[k], err_msg=k)
        np.testing.assert_array_equal(m[k][n:n_new], before[k][src], err_msg=k)


# ---------------------------------------------------------------------------
# subgrid diffusion (T:5033-5200, T:5460-5553)
# ---------------------------------------------------------------------------
def _subgrid_state(pkg, P, G, rng):
    n = G.start_marknum
    st = pkg.HostState(P, capacity=n)
    m = st.m
    m["xm"][:] = -G.dx + rng.integers(0, int((G.xsize + 2 * G.dx) / 0.1) + 1, n) * 0.1
    m["ym"][:] = -G.dy + rng.integers(0, int((G.ysize + 2 * G.dy) / 0.1) + 1, n) * 0.1
    m["tm"][:] = rng.integers(1, 4, n)
    for k in ("sxxm", "sxym", "tkm", "phim"):
        m[k][:] = rng.random(n)
    m["inv_gggtotalm"][:] = 1.0 / (1e10 * (0.5 + rng.random(n)))
    st.marknum = n
    for k in ("SXX0", "SXY0", "DSXX", "DSXY", "tk1", "DT"):
        st.grid[k][:] = rng.random(st.grid[k].shape)
    return st


def test_subgrid_stress_diffusion(L, G, pkg):
    """apply_subgrid_stress_diffusion! against HTM-planetary.m line 1374ff as
    T:5076-5198 states it, with dsubgrids = 1 (the reference's default 0
    makes it a no-op) and the reference's viscosity factor 1 (E:4276):
    relaxation time 1 / G per marker."""
    rng = np.random.default_rng(5033)
    p = pkg.params.default_params(15, 15)
    p.dsubgrids = 1.0
    st = _subgrid_state(pkg, p, G, rng)
    m, g = st.m, st.grid
    n = st.marknum
    dt = 1e-3
    sxx, sxy = m["sxxm"][:n].copy(), m["sxym"][:n].copy()
    DSXX, DSXY = g["DSXX"].copy(), g["DSXY"].copy()
    L.oracle_subgrid_stress(_ref(p), _ref(st.markers_struct()), n, _ref(st.grid_struct()),
                            _ref(st.sums_struct()), dt)
    SXXSUM = np.zeros((G.Ny1, G.Nx1)); WTPSUM = np.zeros((G.Ny1, G.Nx1))
    SXYSUM = np.zeros((G.Ny, G.Nx)); WTSUM = np.zeros((G.Ny, G.Nx))
    for q in range(n):
        ggg = 1.0 / m["inv_gggtotalm"][q]
        relax = math.exp(-p.dsubgrids * dt / (1.0 / ggg))
        for grid, val, S, W in ((3, sxx, SXXSUM, WTPSUM), (0, sxy, SXYSUM, WTSUM)):
            xa, ya, jmax, imax = _grids(G)[grid]
            i, j = _fix_ver(m["xm"][q], m["ym"][q], xa, ya, G.dx, G.dy, jmax, imax)
            dxmj, dymi = m["xm"][q] - xa[j - 1], m["ym"][q] - ya[i - 1]
            w = [(1 - dxmj / G.dx) * (1 - dymi / G.dy), (1 - dxmj / G.dx) * (dymi / G.dy),
                 (dxmj / G.dx) * (1 - dymi / G.dy), (dxmj / G.dx) * (dymi / G.dy)]
            src = g["SXX0"] if grid == 3 else g["SXY0"]
            cells = [(i - 1, j - 1), (i, j - 1), (i - 1, j), (i, j)]
            d0 = val[q] - sum(src[c] * wc for c, wc in zip(cells, w))
            dd = d0 * relax - d0
            val[q] += dd
            for c, wc in zip(cells, w):
                S[c] += dd * wc
                W[c] += wc
    inner = np.zeros_like(WTPSUM, bool)
    inner[1:G.Ny, 1:G.Nx] = True
    nz = inner & (WTPSUM > 0)
    DSXX[nz] -= SXXSUM[nz] / WTPSUM[nz]
    nzb = WTSUM > 0
    DSXY[nzb] -= SXYSUM[nzb] / WTSUM[nzb]
    np.testing.assert_allclose(m["sxxm"][:n], sxx, rtol=RTOL)
    np.testing.assert_allclose(m["sxym"][:n], sxy, rtol=RTOL)
    np.testing.assert_allclose(g["DSXX"], DSXX, rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(g["DSXY"], DSXY, rtol=RTOL, atol=1e-12)


def test_subgrid_temperature_diffusion(L, G, pkg):
    """apply_subgrid_temperature_diffusion! against HTM-planetary.m line
    1731ff as T:5480-5550 states it, with dsubgridt = 1 and constant
    material laws (mode 9)."""
    rng = np.random.default_rng(5460)
    p = pkg.params.default_params(15, 15)
    p.dsubgridt = 1.0
    st = _subgrid_state(pkg, p, G, rng)
    m, g = st.m, st.grid
    n = st.marknum
    dt = 1e7
    tk = m["tkm"][:n].copy()
    DT = g["DT"].copy()
    L.oracle_subgrid_temperature(_ref(p), _ref(st.markers_struct()), n,
                                 _ref(st.grid_struct()), _ref(st.sums_struct()), dt)
    TKSUM = np.zeros((G.Ny1, G.Nx1)); RCP = np.zeros((G.Ny1, G.Nx1))
    rs, rf = list(p.rhocpsolidm), list(p.rhocpfluidm)
    ks, kf = list(p.ksolidm), list(p.kfluidm)
    for q in range(n):
        i, j = _fix_ver(m["xm"][q], m["ym"][q], G.xp, G.yp, G.dx, G.dy, G.Nx, G.Ny)
        dxmj, dymi = m["xm"][q] - G.xp[j - 1], m["ym"][q] - G.yp[i - 1]
        w = [(1 - dxmj / G.dx) * (1 - dymi / G.dy), (1 - dxmj / G.dx) * (dymi / G.dy),
             (dxmj / G.dx) * (1 - dymi / G.dy), (dxmj / G.dx) * (dymi / G.dy)]
        cells = [(i - 1, j - 1), (i, j - 1), (i - 1, j), (i, j)]
        d0 = tk[q] - sum(g["tk1"][c] * wc for c, wc in zip(cells, w))
        t = int(m["tm"][q]) - 1
        ph = m["phim"][q]
        if t < 2:
            rcp = rs[t] * (1 - ph) + rf[t] * ph
            a = ks[t] * (3 * ph - 2) + kf[t] * (1 - 3 * ph)
            k = (ks[t] * kf[t] / 2 + a ** 2 / 16) ** 0.5 - a / 4
        else:
            rcp, k = rs[t], ks[t]
        d1 = d0 * math.exp(-p.dsubgridt * k * dt / rcp * (2 / G.dx ** 2 + 2 / G.dy ** 2))
        dd = d1 - d0
        tk[q] += dd
        for c, wc in zip(cells, w):
            TKSUM[c] += dd * rcp * wc
            RCP[c] += rcp * wc
    nz = RCP > 0
    DT[nz] -= TKSUM[nz] / RCP[nz]
    np.testing.assert_allclose(m["tkm"][:n], tk, rtol=RTOL)
    np.testing.assert_allclose(g["DT"], DT, rtol=RTOL, atol=1e-12)
