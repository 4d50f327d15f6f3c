"""CPU restatement of the heat-path adjoint and its finite-difference check.

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the product.

The reference has no derivatives.  The objective is that of the adjoint
entry point of the device library:

    J = mean over the basic nodes inside the body (distance from the centre
        < rplanet) of grid_average(tk2) (src/Erebus.jl:1176) after the last of
        N timesteps,

differentiated with respect to the per-marker porosity phim and the 26Al/27Al
ratio, for states at mechanical rest (G = 0, reactions off, no strain rate,
no subgrid diffusion, zero marker stresses): velocities, porosity change and
marker motion then vanish, and J depends on the parameters only through the
heat path of each timestep:

    marker laws (E:700-750, E:1116-1357, E:2272-2358) -> P/Vx/Vy scatter
    (E:1605-1863) -> node normalisation (E:2033-2189) and insulating copies
    (E:2432-2449) -> heat solve (E:4526-4611) -> marker temperature update
    (E:4782-4801).

`forward` runs the oracle's timestep (oracle.Oracle.step) and keeps a tape;
`adjoint` applies the transposed operations in reverse with scipy (the
transposed heat matrix is the oracle's assembled matrix, transposed);
`objective` evaluates J.  Central finite differences of `objective` over
oracle runs check both.
"""
import ctypes

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import Oracle, _p, lib

GVX, GVY, GP = 1, 2, 3


def body_mask(st):
    """Basic nodes (Ny, Nx) inside the body."""
    g = st.g
    x = (np.arange(1, g.Nx + 1) - 1) * g.dx
    y = (np.arange(1, g.Ny + 1) - 1) * g.dy
    dxc = x[None, :] - g.xcenter
    dyc = y[:, None] - g.ycenter
    return np.sqrt(dxc * dxc + dyc * dyc) < st.p.rplanet


def grid_average(A):
    """(Ny1, Nx1) P-node array -> (Ny, Nx) basic-node averages (E:1176)."""
    return 0.25 * (A[:-1, :-1] + A[1:, :-1] + A[:-1, 1:] + A[1:, 1:])


def objective(st):
    """J of the HostState's current tk2."""
    mask = body_mask(st)
    return float(grid_average(st.grid["tk2"])[mask].sum() / mask.sum())


def weight_matrix(st, grid):
    """(Ny1*Nx1, marknum) sparse matrix of the markers' bilinear weights on
    `grid` (fix_weights, E:1388), column-major node numbering."""
    L = lib()
    g, n = st.g, st.marknum
    R = g.Ny1
    rows = np.empty(4 * n, np.int64)
    vals = np.empty(4 * n)
    i, j = ctypes.c_int(), ctypes.c_int()
    w = (ctypes.c_double * 4)()
    pp = _p(st.p)
    xm, ym = st.m["xm"], st.m["ym"]
    for m in range(n):
        L.oracle_weights_grid(pp, grid, float(xm[m]), float(ym[m]), ctypes.byref(i),
                              ctypes.byref(j), w)
        base = (j.value - 1) * R + (i.value - 1)
        rows[4 * m: 4 * m + 4] = (base, base + 1, base + R, base + R + 1)
        vals[4 * m: 4 * m + 4] = w[0], w[1], w[2], w[3]
    cols = np.repeat(np.arange(n), 4)
    return sp.csr_matrix((vals, (rows, cols)), shape=(g.Ny1 * g.Nx1, n))


def forward(st, n_steps, first_timestep=1):
    """Runs the oracle for n_steps timesteps; returns the tape."""
    o = Oracle(st)
    tape = []
    for q in range(n_steps):
        rec = {"T": st.m["tkm"][: st.marknum].copy(), "t": st.timesum}
        s = o.step(first_timestep + q)
        gr = st.grid
        rec.update(dt=s["dt"], titer=s["titer"], timestep=first_timestep + q,
                   **{k: gr[k].copy(order="F") for k in ("tk2", "DT", "RHOCP", "KX", "KY")})
        tape.append(rec)
        if q == 0:
            W = {k: st.sums[k].copy(order="F") for k in ("WTPSUM", "WTXSUM", "WTYSUM")}
    return o, tape, W


def _thermal_matrix(o, st, rec):
    gr = st.grid
    saved = {k: gr[k].copy(order="F") for k in ("RHOCP", "KX", "KY")}
    for k in saved:
        gr[k][:] = rec[k]
    A, _ = o.thermal_system(rec["dt"])
    for k, v in saved.items():
        gr[k][:] = v
    return A


def _laws(p, T, phi, t):
    """Marker laws of rock markers and their derivatives (vectorised)."""
    mode1 = p.marker_property_mode == 1
    rcs = np.array(p.rhocpsolidm)[t - 1]
    if mode1:
        tm = p.tmfluidphase
        rcf = np.select([T < tm - 5, T < tm, T < tm + 5, T < 410.0],
                        [p.rhoH2Ofi * (7.67 * T), p.rhoH2Ofi * (7.67 * T + 0.1 * p.Lf),
                         p.rhoH2Of * (4200.0 + 0.1 * p.Lf), p.rhoH2Of * 4200.0 + 0 * T],
                        p.rhoH2Of * (-4.67e4 + 333 * T - 0.731 * (T * T) + 5.4e-4 * (T * T * T)))
        drcf = np.select([T < tm, T < 410.0], [p.rhoH2Ofi * 7.67 + 0 * T, 0 * T],
                         p.rhoH2Of * (333 - 2 * 0.731 * T + 3 * 5.4e-4 * (T * T)))
        ks = 0.73 + 1293.0 / (T + 77.0)
        dks = -1293.0 / (T + 77.0) ** 2
        kf = np.select([T < tm, T < 410], [0.465 + 488.0 / T, -0.581 + 6.34e-3 * T - 7.93e-6 * T * T],
                       -0.142 + 4.12e-3 * T - 5.01e-6 * T * T)
        dkf = np.select([T < tm, T < 410], [-488.0 / T ** 2, 6.34e-3 - 2 * 7.93e-6 * T],
                        4.12e-3 - 2 * 5.01e-6 * T)
    else:
        rcf = np.full_like(T, p.rhocpfluidm[0])
        drcf = np.zeros_like(T)
        ks = np.full_like(T, p.ksolidm[0])
        kf = np.full_like(T, p.kfluidm[0])
        dks = np.zeros_like(T)
        dkf = np.zeros_like(T)
    rc = rcs * (1 - phi) + rcf * phi
    a = ks * (3 * phi - 2) + kf * (1 - 3 * phi)
    r = np.sqrt(ks * kf / 2 + a * a / 16)
    da = a / (16 * r) - 0.25
    dk_ks = kf / (4 * r) + da * (3 * phi - 2)
    dk_kf = ks / (4 * r) + da * (1 - 3 * phi)
    dk_phi = da * 3 * (ks - kf)
    return rcs, rcf, drcf, rc, dks, dkf, dk_ks, dk_kf, dk_phi


def adjoint(o, st, tape, W):
    """dJ/dphim (marknum,) and dJ/dratio_al by the reverse sweep."""
    p, g = st.p, st.g
    n = st.marknum
    R, C = g.Ny1, g.Nx1
    shape = (R, C)
    Pm, Xm, Ym = (weight_matrix(st, gr) for gr in (GP, GVX, GVY))
    mask = body_mask(st)
    seed = np.zeros(shape, order="F")
    inv = 0.25 / mask.sum()
    for di in (0, 1):
        for dj in (0, 1):
            seed[di:di + g.Ny, dj:dj + g.Nx] += inv * mask
    tm = st.m["tm"][:n]
    rock = tm < 3
    phi = st.m["phim"][:n]
    rcm = st.m["rhocptotalm"][:n]
    inner = np.zeros(shape, bool)
    inner[1:-1, 1:-1] = True
    idx2, idy2 = 1.0 / (g.dx * g.dx), 1.0 / (g.dy * g.dy)
    Wp, Wx, Wy = W["WTPSUM"], W["WTXSUM"], W["WTYSUM"]
    tau = p.t_half_al / np.log(2.0)
    Tbar = np.zeros(n)
    phibar = np.zeros(n)
    rbar = 0.0
    N = len(tape)
    for q in range(N - 1, -1, -1):
        rec = tape[q]
        last = q == N - 1
        carry = rec["timestep"] > 1
        S = np.zeros(shape, order="F") if last else (Pm @ Tbar).reshape(shape, order="F")
        gvec = S + (seed if last else 0.0)
        A = _thermal_matrix(o, st, rec)
        lam = spla.spsolve(A.T.tocsc(), gvec.ravel(order="F")).reshape(shape, order="F")
        tk2, DT, rc = rec["tk2"], rec["DT"], rec["RHOCP"]
        dt = rec["dt"]
        tk1 = tk2 - DT
        # tk1 adjoint: RHS, then -S through the insulating copies
        t1b = np.where(inner, lam * rc / dt, 0.0)
        if carry and not last:
            s = S.copy(order="F")
            # ghost nodes fold onto the inner node they were copied from
            src_i = np.clip(np.arange(R), 1, R - 2)
            src_j = np.clip(np.arange(C), 1, C - 2)
            fold = np.zeros(shape, order="F")
            np.add.at(fold, (src_i[:, None].repeat(C, 1), src_j[None, :].repeat(R, 0)), s)
            t1b = t1b - np.where(inner, fold, 0.0)
        rc_b = np.where(inner, -lam * DT / dt, 0.0)
        ok = inner & (Wp > 0)
        srcp = np.where(ok, rc * Wp, 1.0)
        srcp_b = np.where(ok, rc_b / np.where(ok, Wp, 1.0) - t1b * tk1 / srcp, 0.0)
        str_b = np.where(ok, t1b / srcp, 0.0)
        shr_b = np.where(ok, lam / np.where(ok, Wp, 1.0), 0.0)
        kxb = np.zeros(shape)
        kyb = np.zeros(shape)
        lamI = np.where(inner, lam, 0.0)
        # KX(i,j): rows (i,j) and (i,j+1); KY(i,j): rows (i,j) and (i+1,j)
        kxb[:, :-1] -= lamI[:, :-1] * (tk2[:, :-1] - tk2[:, 1:]) * idx2
        kxb[:, :-1] -= lamI[:, 1:] * (tk2[:, 1:] - tk2[:, :-1]) * idx2
        kyb[:-1, :] -= lamI[:-1, :] * (tk2[:-1, :] - tk2[1:, :]) * idy2
        kyb[:-1, :] -= lamI[1:, :] * (tk2[1:, :] - tk2[:-1, :]) * idy2
        skx = np.where(Wx > 0, kxb / np.where(Wx > 0, Wx, 1.0), 0.0)
        sky = np.where(Wy > 0, kyb / np.where(Wy > 0, Wy, 1.0), 0.0)
        f = lambda a: a.ravel(order="F")
        rcb = Pm.T @ f(srcp_b)
        trb = Pm.T @ f(str_b)
        hrb = Pm.T @ f(shr_b)
        kb = Xm.T @ f(skx) + Ym.T @ f(sky)
        T = rec["T"]
        tb = Tbar.copy() if carry else np.zeros(n)
        tt = tm[rock]
        rcs, rcf, drcf, rcr, dks, dkf, dk_ks, dk_kf, dk_phi = _laws(p, T[rock], phi[rock], tt)
        rcbt = rcb[rock] + trb[rock] * T[rock]
        tb[rock] += (trb[rock] * rcr + rcbt * phi[rock] * drcf +
                     kb[rock] * (dk_ks * dks + dk_kf * dkf))
        tb[~rock] += trb[~rock] * rcm[~rock]
        e = np.exp(-rec["t"] * (1.0 / tau)) * (1.0 / tau) if p.hr_al else 0.0
        Q = p.f_al * p.ratio_al * p.E_al * e
        hrs = Q * np.array(p.rhosolidm)[tt - 1]
        hrf = np.zeros_like(hrs)
        if p.hr_fe:
            taufe = p.t_half_fe / np.log(2.0)
            Qfe = p.f_fe * p.ratio_fe * p.E_fe * np.exp(-rec["t"] / taufe) / taufe
            hrf = np.where(tt == 1, Qfe * p.rhofluidm[0], 0.0)
        phibar[rock] += rcbt * (rcf - rcs) + kb[rock] * dk_phi + hrb[rock] * (hrf - hrs)
        rbar += float(np.sum(hrb[rock] * (1 - phi[rock]) * p.f_al * p.E_al * e *
                            np.array(p.rhosolidm)[tt - 1]))
        Tbar = tb
    return phibar, rbar


def at_rest(st):
    """Sets the parameters of a state at mechanical rest."""
    st.p.G = 0.0
    st.p.reaction_active = 0
    st.p.strainrate = 0.0
    st.p.dsubgrids = 0.0
    st.p.dsubgridt = 0.0
    st.m["sxxm"][:] = 0.0
    st.m["sxym"][:] = 0.0
    return st
