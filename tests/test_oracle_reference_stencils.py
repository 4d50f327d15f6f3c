"""The oracle's Stokes-Darcy post-processing, plastic iteration, heating terms
and iteration control against re-expressions of the reference's own tests.

Each test restates one testset of test/runtests.jl (cited T:<line>), whose
verification is a loop-by-loop formulation from the MATLAB codes the model
comes from (HTM-planetary.m, HTM-hydration.m), and applies it to the C
restatement (oracle/erebus_oracle.c) on inputs drawn from the ranges the
testset states, with its tolerance (rtol 1e-9, == where it tests ==).  The
grid is that of src/test_constants.jl (15 x 15 basic nodes over 14 km).

compute_nodal_adjustment! is also checked with yielding nodes already marked
(YNY set), which the reference's testset leaves out: there the reference
counts a node that was yielding and still yields twice in the error sum
(its `ynn` flag is never set, E:4042-4073), and the oracle keeps that.
"""
import ctypes

import numpy as np
import pytest

from test_oracle_reference import G, L, P, _ref  # noqa: F401

RTOL = 1e-9


@pytest.fixture
def st(pkg, P):
    return pkg.HostState(P, capacity=1)


def test_process_hydromechanical_solution(L, P, G, st):
    """T:4451-4507 (HTM-planetary.m line 1058ff)."""
    rng = np.random.default_rng(4451)
    n = G.Nx1 * G.Ny1
    S = rng.random(6 * n) * 2e-10 - 1e-10
    assert L.oracle_process_hydromech(_ref(P), S.ctypes.data_as(ctypes.c_void_p),
                                      _ref(st.grid_struct())) == 0
    g = st.grid
    # unknown k = ((j-1) Ny1 + i - 1) * 6 + {1..6}: column-major node order
    R = S.reshape(G.Nx1, G.Ny1, 6)
    ver = {"vx": R[:, :, 0].T, "vy": R[:, :, 1].T, "pr": R[:, :, 2].T * P.Kcont,
           "qxD": R[:, :, 3].T, "qyD": R[:, :, 4].T, "pf": R[:, :, 5].T * P.Kcont}
    for k, v in ver.items():
        np.testing.assert_allclose(g[k], v, rtol=RTOL, err_msg=k)


def test_compute_aphi(L, P, G, st):
    """T:4509-4547 (HTM-planetary.m line 1078ff), dt = dt_longest."""
    rng = np.random.default_rng(4509)
    g, shp, Nx, Ny = st.grid, (G.Ny1, G.Nx1), G.Nx, G.Ny
    g["APHI"][...] = rng.random(shp)
    g["ETAPHI"][...] = rng.random(shp) * 1e15
    g["BETAPHI"][...] = rng.random(shp) * 1e-10
    g["PHI"][...] = rng.random(shp)
    for k in ("pr", "pf", "pr0", "pf0"):
        g[k][...] = rng.random(shp) * 1e4
    dt = P.dt_longest
    aphimax = L.oracle_compute_aphi(_ref(P), _ref(st.grid_struct()), dt)
    s = (slice(1, Ny), slice(1, Nx))
    ver = ((g["pr"][s] - g["pf"][s]) / g["ETAPHI"][s] +
           ((g["pr"][s] - g["pr0"][s]) - (g["pf"][s] - g["pf0"][s])) / dt *
           g["BETAPHI"][s]) / (1 - g["PHI"][s]) / g["PHI"][s]
    np.testing.assert_allclose(g["APHI"][s], ver, rtol=RTOL)
    np.testing.assert_allclose(aphimax, np.max(np.abs(ver)), rtol=RTOL)


def test_fluid_velocities(L, P, G, st):
    """T:4549-4604 (HTM-planetary.m line 1090ff)."""
    rng = np.random.default_rng(4549)
    g, shp, Nx, Ny = st.grid, (G.Ny1, G.Nx1), G.Nx, G.Ny
    for k in ("PHIX", "PHIY", "qxD", "qyD", "vx", "vy"):
        g[k][...] = rng.random(shp)
    g["vxf"][...] = 0.0
    g["vyf"][...] = 0.0
    assert L.oracle_fluid_velocities(_ref(P), _ref(st.grid_struct())) == 0
    vxf = np.zeros(shp)
    vxf[1:Ny, 0:Nx] = g["qxD"][1:Ny, 0:Nx] / g["PHIX"][1:Ny, 0:Nx]
    vxf[0, :] = -P.bcftop * vxf[1, :]
    vxf[Ny, :] = -P.bcfbottom * vxf[Ny - 1, :]
    vyf = np.zeros(shp)
    vyf[0:Ny, 1:Nx] = g["qyD"][0:Ny, 1:Nx] / g["PHIY"][0:Ny, 1:Nx]
    vyf[:, 0] = -P.bcfleft * vyf[:, 1]
    vyf[:, Nx] = -P.bcfright * vyf[:, Nx - 1]
    np.testing.assert_allclose(g["vxf"], vxf + g["vx"], rtol=RTOL)
    np.testing.assert_allclose(g["vyf"], vyf + g["vy"], rtol=RTOL)


@pytest.mark.parametrize("vscale", [1.0, 1e-20])
def test_displacement_timestep(L, P, G, st, vscale):
    """T:4606-4648 (HTM-planetary.m line 1117ff); with vscale 1e-20 the
    velocities no longer limit dt and the porosity limit decides."""
    rng = np.random.default_rng(4606)
    g, shp = st.grid, (G.Ny1, G.Nx1)
    aphimax = rng.random()
    for k in ("vx", "vy", "vxf", "vyf"):
        g[k][...] = rng.random(shp) * vscale
    dt = P.dt_longest
    dtm = L.oracle_displacement_timestep(_ref(P), _ref(st.grid_struct()), dt, aphimax)
    ver = dt
    for k, d in (("vx", G.dx), ("vy", G.dy), ("vxf", G.dx), ("vyf", G.dy)):
        mv = np.max(np.abs(g[k]))
        if ver * mv > P.dxymax * d:
            ver = P.dxymax * d / mv
    if aphimax * ver > P.dphimax:
        ver = P.dphimax / aphimax
    np.testing.assert_allclose(dtm, ver, rtol=RTOL)


def test_stress_strainrate(L, P, G, st):
    """T:4650-4735 (HTM-planetary.m line 1144ff), dtm = dt_longest."""
    rng = np.random.default_rng(4650)
    g, Nx, Ny = st.grid, G.Nx, G.Ny
    pshp, bshp = (G.Ny1, G.Nx1), (Ny, Nx)
    for k in ("vx", "vy", "ETAP", "GGGP", "SXX0", "EXX", "SXX", "DSXX"):
        g[k][...] = rng.random(pshp)
    for k in ("ETA", "GGG", "SXY0", "EXY", "SXY", "DSXY"):
        g[k][...] = rng.random(bshp)
    g["EII"][...] = 0.0
    g["SII"][...] = 0.0
    inp = {k: g[k].copy() for k in g}
    dtm = P.dt_longest
    assert L.oracle_stress_strainrate(_ref(P), _ref(st.grid_struct()), dtm) == 0
    vx, vy = inp["vx"], inp["vy"]
    E, GG, S0 = inp["ETA"], inp["GGG"], inp["SXY0"]
    EXY = 0.5 * ((vx[1:Ny + 1, 0:Nx] - vx[0:Ny, 0:Nx]) / G.dy +
                 (vy[0:Ny, 1:Nx + 1] - vy[0:Ny, 0:Nx]) / G.dx)
    SXY = 2 * E * EXY * GG * dtm / (GG * dtm + E) + S0 * E / (GG * dtm + E)
    np.testing.assert_allclose(g["EXY"], EXY, rtol=RTOL)
    np.testing.assert_allclose(g["SXY"], SXY, rtol=RTOL)
    np.testing.assert_allclose(g["DSXY"], SXY - S0, rtol=RTOL)
    s = (slice(1, Ny), slice(1, Nx))
    EXX = ((vx[1:Ny, 1:Nx] - vx[1:Ny, 0:Nx - 1]) / G.dx -
           (vy[1:Ny, 1:Nx] - vy[0:Ny - 1, 1:Nx]) / G.dy) / 2
    EP, GP, X0 = inp["ETAP"][s], inp["GGGP"][s], inp["SXX0"][s]
    SXX = 2 * EP * EXX * GP * dtm / (GP * dtm + EP) + X0 * EP / (GP * dtm + EP)
    avg = lambda A: (A[1:Ny, 1:Nx] + A[0:Ny - 1, 1:Nx] + A[1:Ny, 0:Nx - 1] +
                     A[0:Ny - 1, 0:Nx - 1]) / 4
    np.testing.assert_allclose(g["EXX"][s], EXX, rtol=RTOL)
    np.testing.assert_allclose(g["SXX"][s], SXX, rtol=RTOL)
    np.testing.assert_allclose(g["DSXX"][s], SXX - X0, rtol=RTOL)
    np.testing.assert_allclose(g["EII"][s], np.sqrt(EXX ** 2 + avg(EXY) ** 2), rtol=RTOL)
    np.testing.assert_allclose(g["SII"][s], np.sqrt(SXX ** 2 + avg(SXY) ** 2), rtol=RTOL)


def test_symmetrize_p_node_observables(L, P, G, st):
    """T:4737-4811 (HTM-planetary.m line 1196ff): the boundary copies are
    exact (==), ps to rtol 1e-9."""
    rng = np.random.default_rng(4737)
    g, Nx, Ny = st.grid, G.Nx, G.Ny
    names = ("SXX", "APHI", "PHI", "pr", "pf")
    for k in names:
        g[k][...] = rng.random((G.Ny1, G.Nx1))
    ver = {k: g[k].copy() for k in names}
    assert L.oracle_symmetrize(_ref(P), _ref(st.grid_struct())) == 0
    for v in ver.values():
        v[0, 1:Nx] = v[1, 1:Nx]
        v[Ny, 1:Nx] = v[Ny - 1, 1:Nx]
        v[:, 0] = v[:, 1]
        v[:, Nx] = v[:, Nx - 1]
    for k in names:
        np.testing.assert_array_equal(g[k][0, 1:Nx], ver[k][0, 1:Nx], err_msg=k)
        np.testing.assert_array_equal(g[k][Ny, 1:Nx], ver[k][Ny, 1:Nx], err_msg=k)
        np.testing.assert_array_equal(g[k][:, 0], ver[k][:, 0], err_msg=k)
        np.testing.assert_array_equal(g[k][:, Nx], ver[k][:, Nx], err_msg=k)
    ps = (ver["pr"] - ver["pf"] * ver["PHI"]) / (1 - ver["PHI"])
    np.testing.assert_allclose(g["ps"], ps, rtol=RTOL)


def _nodal_ver(P, G, inp, dt, iplast, count_old_twice):
    """HTM-planetary.m line 1232ff as T:4880-4927 states it.  With
    `count_old_twice` a node that was yielding (YNY) and yields again enters
    the error sum twice, as the reference's own function does."""
    Ny, Nx = G.Ny, G.Nx
    ETA5 = inp["ETA0"].copy()
    YNY5 = np.zeros((Ny, Nx), bool)
    DSY = np.zeros((Ny, Nx))
    ynpl, ddd = 0, 0.0
    SXX, pr, pf = inp["SXX"], inp["pr"], inp["pf"]
    for i in range(Ny):
        for j in range(Nx):
            sxxa = (SXX[i, j] + SXX[i + 1, j] + SXX[i, j + 1] + SXX[i + 1, j + 1]) / 4
            SIIB = (inp["SXY"][i, j] ** 2 + sxxa ** 2) ** 0.5
            e, gg = inp["ETA"][i, j], inp["GGG"][i, j]
            siiel = SIIB * (gg * dt + e) / e
            prB = (pr[i, j] + pr[i + 1, j] + pr[i, j + 1] + pr[i + 1, j + 1]) / 4
            pfB = (pf[i, j] + pf[i + 1, j] + pf[i, j + 1] + pf[i + 1, j + 1]) / 4
            syc = inp["COH"][i, j] + inp["FRI"][i, j] * (prB - pfB)
            syt = inp["TEN"][i, j] + (prB - pfB)
            sy = max(min(syt, syc), 0)
            ynn = 0
            if inp["YNY"][i, j] > 0:
                ynn = 0 if count_old_twice else 1
                DSY[i, j] = SIIB - sy
                ddd += DSY[i, j] ** 2
                ynpl += 1
            if sy < siiel:
                etapl = dt * gg * sy / (siiel - sy)
                if etapl < inp["ETA0"][i, j]:
                    ETA5[i, j] = etapl ** (1 - P.etawt) * e ** P.etawt
                    YNY5[i, j] = True
                    ETA5[i, j] = min(max(ETA5[i, j], P.etamin), P.etamax)
                    if ynn == 0:
                        DSY[i, j] = SIIB - sy
                        ddd += DSY[i, j] ** 2
                        ynpl += 1
    yerr = (ddd / ynpl) ** 0.5 if ynpl > 0 else None
    return ETA5, YNY5, DSY, ynpl, yerr


@pytest.mark.parametrize("marked", [False, True])
def test_nodal_adjustment(L, P, G, st, marked):
    """T:4826-4933 with the testset's inputs (YNY all false); with `marked`
    also half the nodes marked as yielding, where the reference's double
    count of re-yielding nodes applies."""
    rng = np.random.default_rng(4826 + marked)
    g, Nx, Ny = st.grid, G.Nx, G.Ny
    bshp, pshp = (Ny, Nx), (G.Ny1, G.Nx1)
    for k in ("ETA", "ETA0", "GGG", "SXY", "COH", "TEN", "FRI", "DSY"):
        g[k][...] = rng.random(bshp)
    for k in ("SXX", "pr", "pf"):
        g[k][...] = rng.random(pshp)
    g["ETA5"][...] = 0.0
    g["YNY"][...] = (rng.random(bshp) < 0.5) if marked else False
    g["YNY5"][...] = False
    inp = {k: g[k].copy() for k in g}
    dt, iplast = P.dt_longest, 1
    yerr = np.zeros(1)
    ynpl = ctypes.c_int(0)
    done = L.oracle_nodal_adjustment(_ref(P), _ref(st.grid_struct()), dt, iplast,
                                     yerr.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ynpl))
    ETA5, YNY5, DSY, n, ye = _nodal_ver(P, G, inp, dt, iplast, count_old_twice=True)
    np.testing.assert_allclose(g["ETA5"], ETA5, rtol=RTOL)
    np.testing.assert_array_equal(g["YNY5"].astype(bool), YNY5)
    assert ynpl.value == n
    if ye is not None:
        np.testing.assert_allclose(yerr[0], ye, rtol=RTOL)
    assert bool(done) == (n == 0 or iplast == P.nplast or yerr[0] < P.yerrmax)
    if not marked:
        # with no node marked beforehand the double count never arises and the
        # reference test's own verification (ynn set) agrees
        ETA5b, YNY5b, _, nb, yeb = _nodal_ver(P, G, inp, dt, iplast, count_old_twice=False)
        assert nb == n and yeb == ye


@pytest.mark.parametrize("iplast", [1, 200])
def test_finalize_plastic_iteration_pass(L, P, G, st, iplast):
    """T:4935-4980 (HTM-planetary.m line 1301ff): iplast 1 takes the new
    viscosities; iplast = dtstep (200) halves dt and rolls back."""
    rng = np.random.default_rng(4935 + iplast)
    g, bshp = st.grid, (G.Ny, G.Nx)
    g["ETA"][...] = 0.0
    g["ETA5"][...] = rng.random(bshp)
    g["ETA00"][...] = rng.random(bshp)
    g["YNY"][...] = False
    g["YNY5"][...] = rng.random(bshp) < 0.5
    g["YNY00"][...] = rng.random(bshp) < 0.5
    inp = {k: g[k].copy() for k in g}
    dt = L.oracle_finalize_plastic(_ref(P), _ref(st.grid_struct()), P.dt_longest, iplast)
    if (iplast // P.dtstep) * P.dtstep == iplast:
        dt_ver, E, Y = P.dt_longest * P.dtcoefdn, inp["ETA00"], inp["YNY00"]
    else:
        dt_ver, E, Y = P.dt_longest, inp["ETA5"], inp["YNY5"]
    assert dt == dt_ver
    np.testing.assert_array_equal(g["ETA"], E)
    np.testing.assert_array_equal(g["YNY"], Y)
    np.testing.assert_array_equal(g["YNY_inv_ETA"], Y / E)


def test_thermochemical_iteration_control(P, G, oracle):
    """finalize_thermochemical_iteration_pass (T:4982-5003, HTM-hydration.m
    line 1230ff) and compute_thermochemical_iteration_outcome (T:5005-5031,
    line 1385ff), the two rules the oracle's step driver applies."""
    rng = np.random.default_rng(4982)
    shp = (G.Ny1, G.Nx1)
    for DT in (rng.random(shp), rng.random(shp) * P.DTmax * 2.0):
        for titer in (1, 2, 3):
            mx = float(np.max(np.abs(DT)))
            dt = oracle.finalize_thermochemical_iteration_pass(P, mx, P.dt_longest, titer)
            ver = P.dt_longest
            if titer == 1 and mx > P.DTmax:
                ver = ver / mx * P.DTmax
            np.testing.assert_allclose(dt, ver, rtol=RTOL)
    pf0 = rng.random(shp)
    pf_small, pf_large = rng.random(shp), rng.random(shp) * P.pferrmax * 2.0
    DMP_small, DMP_zero = rng.random(shp) * 2 - 1, np.zeros(shp)
    for titer in (1, 2, 3):
        for pf in (pf_small, pf_large):
            for DMP in (DMP_small, DMP_zero):
                got = oracle.thermochemical_iteration_outcome(P, DMP, pf, pf0, titer)
                pferrcur = np.max(np.abs(pf - pf0))
                DMPmax = np.max(np.abs(DMP))
                ver = bool(pferrcur < P.pferrmax and (titer > 2 or DMPmax <= 0))
                assert got == ver, (titer, got)


def test_shear_heating(L, P, G, st):
    """T:5272-5314 (HTM-planetary.m line 1551ff)."""
    rng = np.random.default_rng(5272)
    g, Nx, Ny = st.grid, G.Nx, G.Ny
    g["HS"][...] = 0.0
    for k in ("ETA", "SXY"):
        g[k][...] = rng.random((Ny, Nx))
    for k in ("ETAP", "SXX", "RX", "RY", "qxD", "qyD", "PHI", "ETAPHI", "pr", "pf"):
        g[k][...] = rng.random((G.Ny1, G.Nx1))
    assert L.oracle_shear_heating(_ref(P), _ref(st.grid_struct())) == 0
    ver = np.zeros((G.Ny1, G.Nx1))
    S, E = g["SXY"], g["ETA"]
    for j in range(1, Nx):
        for i in range(1, Ny):
            sxyexy = (S[i, j] ** 2 / E[i, j] + S[i - 1, j] ** 2 / E[i - 1, j] +
                      S[i, j - 1] ** 2 / E[i, j - 1] + S[i - 1, j - 1] ** 2 / E[i - 1, j - 1]) / 4
            ver[i, j] = (g["SXX"][i, j] ** 2 / g["ETAP"][i, j] + sxyexy +
                         (g["pr"][i, j] - g["pf"][i, j]) ** 2 / (1 - g["PHI"][i, j]) /
                         g["ETAPHI"][i, j] +
                         (g["RX"][i, j - 1] * g["qxD"][i, j - 1] ** 2 +
                          g["RX"][i, j] * g["qxD"][i, j] ** 2) / 2 +
                         (g["RY"][i - 1, j] * g["qyD"][i - 1, j] ** 2 +
                          g["RY"][i, j] * g["qyD"][i, j] ** 2) / 2)
    np.testing.assert_allclose(g["HS"], ver, rtol=RTOL)


def test_adiabatic_heating(L, P, G, st):
    """T:5316-5375 (HTM-planetary.m line 1573ff), including the use of the
    solid-pressure gradients in the fluid term that the verification shares
    with the reference."""
    rng = np.random.default_rng(5316)
    g, Nx, Ny = st.grid, G.Nx, G.Ny
    g["HA"][...] = 0.0
    for k in ("tk1", "ALPHA", "ALPHAF", "PHI", "vx", "vy", "vxf", "vyf", "ps", "pf"):
        g[k][...] = rng.random((G.Ny1, G.Nx1)) - (0.5 if k in ("vx", "vy", "vxf", "vyf")
                                                  else 0.0)
    assert L.oracle_adiabatic_heating(_ref(P), _ref(st.grid_struct())) == 0
    ver = np.zeros((G.Ny1, G.Nx1))
    vx, vy, vxf, vyf, ps = g["vx"], g["vy"], g["vxf"], g["vyf"], g["ps"]
    for j in range(1, Nx):
        for i in range(1, Ny):
            VXP = (vx[i, j] + vx[i, j - 1]) / 2
            VYP = (vy[i, j] + vy[i - 1, j]) / 2
            VXFP = (vxf[i, j] + vxf[i, j - 1]) / 2
            VYFP = (vyf[i, j] + vyf[i - 1, j]) / 2
            dpsdx = (ps[i, j] - ps[i, j - 1]) / G.dx if VXP < 0 else (ps[i, j + 1] - ps[i, j]) / G.dx
            dpsdy = (ps[i, j] - ps[i - 1, j]) / G.dy if VYP < 0 else (ps[i + 1, j] - ps[i, j]) / G.dy
            dpsdt = VXP * dpsdx + VYP * dpsdy
            dpfdt = VXFP * dpsdx + VYFP * dpsdy
            ver[i, j] = ((1 - g["PHI"][i, j]) * g["tk1"][i, j] * g["ALPHA"][i, j] * dpsdt +
                         g["PHI"][i, j] * g["tk1"][i, j] * g["ALPHAF"][i, j] * dpfdt)
    np.testing.assert_allclose(g["HA"], ver, rtol=RTOL, atol=1e-300)
