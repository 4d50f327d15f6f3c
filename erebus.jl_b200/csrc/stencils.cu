// stencils.cu -- node-parallel phases of the timestep.
//
// Each kernel restates one reference function over the staggered grid with
// the reference's arithmetic order: recompute_bulk_viscosity! (E:3634),
// process_hydromechanical_solution! (E:3593), compute_Aphi! (E:3675),
// compute_fluid_velocities! (E:3716), compute_displacement_timestep
// (E:3777), compute_stress_strainrate! (E:3839),
// symmetrize_p_node_observables! (E:3945), compute_nodal_adjustment!
// (E:4015), finalize_plastic_iteration_pass! (E:4142),
// compute_shear_heating! (E:4415), compute_adiabatic_heating! (E:4458),
// process_gravitational_solution! (E:2865), compute_velocities! (E:4878)
// and compute_rotation_rate! (E:4946).  Maxima are reduced with atomicMax
// on the bit patterns of non-negative doubles (NaN propagates as in
// Julia's `maximum`); sums are reduced in a fixed order.
#include "stencils.cuh"

namespace erebus {

__device__ __forceinline__ void amax(double *slot, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(slot),
              (unsigned long long)__double_as_longlong(fabs(v)));
}
// The same maximum of |v| (as bits, so NaN wins as before), reduced over the
// warp first: one atomic per warp.  Every lane of the warp calls it; lanes
// without a value pass active = false.
__device__ __forceinline__ void amax_warp(double *slot, double v, bool active) {
    unsigned long long b = active ? (unsigned long long)__double_as_longlong(fabs(v)) : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long c = __shfl_xor_sync(0xffffffffu, b, o);
        b = c > b ? c : b;
    }
    if ((threadIdx.x & 31) == 0 && b) atomicMax(reinterpret_cast<unsigned long long *>(slot), b);
}

#define NODE_P(g, t)                                  \
    int t = blockIdx.x * blockDim.x + threadIdx.x;    \
    if (t >= (g).Ny1 * (g).Nx1) return;               \
    int i = t % (g).Ny1 + 1, j = t / (g).Ny1 + 1;
#define NODE_B(g, t)                                  \
    int t = blockIdx.x * blockDim.x + threadIdx.x;    \
    if (t >= (g).Ny * (g).Nx) return;                 \
    int i = t % (g).Ny + 1, j = t / (g).Ny + 1;

// process_gravitational_solution! (E:2865-2878); FI holds the solution
__global__ void k_gravity_post(Geo g, GridPtrs G) {
    NODE_P(g, t);
    int Ny1 = g.Ny1;
    if (j <= g.Nx) AT(G.gx, Ny1, i, j) = -(AT(G.FI, Ny1, i, j + 1) - AT(G.FI, Ny1, i, j)) / g.dx;
    if (i <= g.Ny) AT(G.gy, Ny1, i, j) = -(AT(G.FI, Ny1, i + 1, j) - AT(G.FI, Ny1, i, j)) / g.dy;
}

// recompute_bulk_viscosity! (E:3634-3647)
__global__ void k_bulk_viscosity(ErebusParams p, Geo g, GridPtrs G) {
    NODE_P(g, t);
    int Ny = g.Ny, Ny1 = g.Ny1;
    double etap = G.ETAP[t];
    if (i >= 2 && i <= Ny && j >= 2 && j <= g.Nx) {
        etap = 4.0 / (1.0 / AT(G.ETA, Ny, i - 1, j - 1) + 1.0 / AT(G.ETA, Ny, i, j - 1) +
                      1.0 / AT(G.ETA, Ny, i - 1, j) + 1.0 / AT(G.ETA, Ny, i, j));
        AT(G.ETAP, Ny1, i, j) = etap;
    }
    G.ETAPHI[t] = p.etaphikoef * etap * (1.0 / G.PHI[t]);
}

// process_hydromechanical_solution! (E:3593-3617)
__global__ void k_hydro_post(ErebusParams p, Geo g, GridPtrs G, const double *S) {
    NODE_P(g, t);
    (void)i; (void)j;
    G.vx[t] = S[6 * (int64_t)t + 0];
    G.vy[t] = S[6 * (int64_t)t + 1];
    G.pr[t] = S[6 * (int64_t)t + 2] * p.Kcont;
    G.qxD[t] = S[6 * (int64_t)t + 3];
    G.qyD[t] = S[6 * (int64_t)t + 4];
    G.pf[t] = S[6 * (int64_t)t + 5] * p.Kcont;
}

// compute_Aphi! (E:3675-3689) on [2:Ny, 2:Nx]; max |APHI| -> maxabs[X_APHI]
__global__ void k_aphi(Geo g, GridPtrs G, DevScalars *sc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t % g.Ny1 + 1, j = t / g.Ny1 + 1;
    const bool in = t < g.Ny1 * g.Nx1 && i >= 2 && i <= g.Ny && j >= 2 && j <= g.Nx;
    double v = 0.0;
    if (in) {
        double dt = sc->dt;
        double pr = G.pr[t], pf = G.pf[t], ph = G.PHI[t];
        v = ((pr - pf) / G.ETAPHI[t] + ((pr - G.pr0[t]) - (pf - G.pf0[t])) / dt * G.BETAPHI[t]) /
            (1 - ph) / ph;
        G.APHI[t] = v;
    }
    amax_warp(&sc->maxabs[X_APHI], v, in);
}

// compute_fluid_velocities! (E:3716-3757), first half: the values before
// `+= v` into tx / ty (column Nx1 rows 2..Ny of vxf and row Ny1 columns
// 2..Nx of vyf keep their previous values, as in the reference).
__global__ void k_fluid_pre(ErebusParams p, Geo g, GridPtrs G, double *tx, double *ty) {
    NODE_P(g, t);
    int Ny = g.Ny, Ny1 = g.Ny1, Nx = g.Nx;
    auto vxf_pre = [&](int ii, int jj) -> double {
        if (jj <= Nx) return AT(G.qxD, Ny1, ii, jj) / AT(G.PHIX, Ny1, ii, jj);
        return AT(G.vxf, Ny1, ii, jj);
    };
    double vx;
    if (i == 1) vx = -p.bcftop * vxf_pre(2, j);
    else if (i == Ny1) vx = -p.bcfbottom * vxf_pre(Ny, j);
    else vx = vxf_pre(i, j);
    tx[t] = vx;
    auto vyf_pre = [&](int ii, int jj) -> double {
        if (ii <= Ny) return AT(G.qyD, Ny1, ii, jj) / AT(G.PHIY, Ny1, ii, jj);
        return AT(G.vyf, Ny1, ii, jj);
    };
    double vy;
    if (j == 1) vy = -p.bcfleft * vyf_pre(i, 2);
    else if (j == g.Nx1) vy = -p.bcfright * vyf_pre(i, Nx);
    else vy = vyf_pre(i, j);
    ty[t] = vy;
}

// second half (vxf += vx, vyf += vy) and the maxima of
// compute_displacement_timestep (E:3786-3789)
__global__ void k_fluid_fin(Geo g, GridPtrs G, const double *tx, const double *ty,
                            DevScalars *sc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < g.Ny1 * g.Nx1;
    double vx = 0.0, vy = 0.0, a = 0.0, b = 0.0;
    if (in) {
        vx = G.vx[t];
        vy = G.vy[t];
        a = tx[t] + vx;
        b = ty[t] + vy;
        G.vxf[t] = a;
        G.vyf[t] = b;
    }
    amax_warp(&sc->maxabs[X_VX], vx, in);
    amax_warp(&sc->maxabs[X_VY], vy, in);
    amax_warp(&sc->maxabs[X_VXF], a, in);
    amax_warp(&sc->maxabs[X_VYF], b, in);
}

// compute_displacement_timestep (E:3777-3803)
__global__ void k_displacement_dt(ErebusParams p, Geo g, DevScalars *sc) {
    double dt = sc->dt;
    double lx = p.dxymax * g.dx, ly = p.dxymax * g.dy;
    double mvx = sc->maxabs[X_VX], mvy = sc->maxabs[X_VY];
    double mvxf = sc->maxabs[X_VXF], mvyf = sc->maxabs[X_VYF], ap = sc->maxabs[X_APHI];
    dt = (dt * mvx > lx) ? lx * (1.0 / mvx) : dt;
    dt = (dt * mvy > ly) ? ly * (1.0 / mvy) : dt;
    dt = (dt * mvxf > lx) ? lx * (1.0 / mvxf) : dt;
    dt = (dt * mvyf > ly) ? ly * (1.0 / mvyf) : dt;
    dt = (dt * ap > p.dphimax) ? p.dphimax * (1.0 / ap) : dt;
    sc->dt = dt;
    sc->maxabs[X_APHI] = 0.0;   // reset for the second compute_Aphi!
}

// compute_stress_strainrate! (E:3839-3925), basic nodes
__global__ void k_stress_basic(Geo g, GridPtrs G, const DevScalars *sc) {
    NODE_B(g, t);
    int Ny1 = g.Ny1;
    double dt = sc->dt;
    double exy = 0.5 * ((AT(G.vx, Ny1, i + 1, j) - AT(G.vx, Ny1, i, j)) / g.dy +
                        (AT(G.vy, Ny1, i, j + 1) - AT(G.vy, Ny1, i, j)) / g.dx);
    G.EXY[t] = exy;
    double e = G.ETA[t], gg = G.GGG[t];
    double sxy = 2 * e * exy * gg * dt / (gg * dt + e) + G.SXY0[t] * e / (gg * dt + e);
    G.SXY[t] = sxy;
    G.DSXY[t] = sxy - G.SXY0[t];
}

// ... and P nodes [2:Ny, 2:Nx]
__global__ void k_stress_p(Geo g, GridPtrs G, const DevScalars *sc) {
    NODE_P(g, t);
    if (i < 2 || i > g.Ny || j < 2 || j > g.Nx) return;
    int Ny = g.Ny, Ny1 = g.Ny1;
    double dt = sc->dt;
    double exx = 0.5 * ((AT(G.vx, Ny1, i, j) - AT(G.vx, Ny1, i, j - 1)) / g.dx -
                        (AT(G.vy, Ny1, i, j) - AT(G.vy, Ny1, i - 1, j)) / g.dy);
    G.EXX[t] = exx;
    double e = G.ETAP[t], gg = G.GGGP[t];
    double sxx = 2 * e * exx * gg * dt / (gg * dt + e) + G.SXX0[t] * e / (gg * dt + e);
    G.SXX[t] = sxx;
    G.DSXX[t] = sxx - G.SXX0[t];
    double ae = grid_average(G.EXY, Ny, i - 1, j - 1);
    double as = grid_average(G.SXY, Ny, i - 1, j - 1);
    G.EII[t] = sqrt(exx * exx + ae * ae);
    G.SII[t] = sqrt(sxx * sxx + as * as);
}

// symmetrize_p_node_observables! (E:3945-3984): rows 1 and Ny1 ...
__global__ void k_sym_rows(Geo g, GridPtrs G) {
    int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
    if (j > g.Nx) return;
    int Ny1 = g.Ny1;
    double *F[5] = {G.SXX, G.APHI, G.PHI, G.pr, G.pf};
#pragma unroll
    for (int f = 0; f < 5; f++) {
        AT(F[f], Ny1, 1, j) = AT(F[f], Ny1, 2, j);
        AT(F[f], Ny1, Ny1, j) = AT(F[f], Ny1, g.Ny, j);
    }
}
// ... then columns 1 and Nx1, then ps everywhere
__global__ void k_sym_cols_ps(Geo g, GridPtrs G) {
    NODE_P(g, t);
    int Ny1 = g.Ny1;
    double *F[5] = {G.SXX, G.APHI, G.PHI, G.pr, G.pf};
    if (j == 1 || j == g.Nx1) {
        int js = j == 1 ? 2 : g.Nx;
#pragma unroll
        for (int f = 0; f < 5; f++) AT(F[f], Ny1, i, j) = AT(F[f], Ny1, i, js);
    }
    G.ps[t] = (G.pr[t] - G.pf[t] * G.PHI[t]) * (1.0 / (1 - G.PHI[t]));
}

// compute_nodal_adjustment! (E:4015-4094), per basic node; the squared
// yielding errors go to `dd` for a fixed-order sum.
__global__ void k_nodal(ErebusParams p, Geo g, GridPtrs G, const DevScalars *sc0,
                        DevScalars *sc, double *dd) {
    NODE_B(g, t);
    int Ny1 = g.Ny1;
    double dt = sc0->dt;
    G.ETA5[t] = G.ETA0[t];
    G.YNY5[t] = 0;
    G.DSY[t] = 0.0;
    double sxy = G.SXY[t], asxx = grid_average(G.SXX, Ny1, i, j);
    double SIIB = sqrt(sxy * sxy + asxx * asxx);
    double e = G.ETA[t], gg = G.GGG[t];
    double siiel = SIIB * (gg * dt + e) / e;
    double prB = grid_average(G.pr, Ny1, i, j), pfB = grid_average(G.pf, Ny1, i, j);
    double syc = G.COH[t] + G.FRI[t] * (prB - pfB);
    double syt = G.TEN[t] + (prB - pfB);
    double sy = jmax(jmin(syc, syt), 0.0);
    int cnt = 0;
    double acc = 0.0;
    if (G.YNY[t] > 0) {
        double d = SIIB - sy;
        G.DSY[t] = d;
        acc += d * d;
        cnt++;
    }
    if (sy < siiel) {
        double etapl = dt * gg * sy / (siiel - sy);
        if (etapl < G.ETA0[t]) {
            double e5 = pow(etapl, 1.0 - p.etawt) * pow(e, p.etawt);
            if (e5 > p.etamax) e5 = p.etamax;
            else if (e5 < p.etamin) e5 = p.etamin;
            G.ETA5[t] = e5;
            G.YNY5[t] = 1;
            double d = SIIB - sy;
            G.DSY[t] = d;
            acc += d * d;
            cnt++;
        }
    }
    dd[t] = acc;
    if (cnt) atomicAdd(&sc->ynpl, cnt);
}

__global__ void k_sum_fixed(const double *a, int n, double *out) {
    __shared__ double s[1024];
    int T = blockDim.x, t = threadIdx.x;
    int chunk = (n + T - 1) / T, lo = t * chunk, hi = min(n, lo + chunk);
    double x = 0.0;
    for (int k = lo; k < hi; k++) x += a[k];
    s[t] = x;
    __syncthreads();
    for (int off = T / 2; off > 0; off >>= 1) {
        if (t < off) s[t] += s[t + off];
        __syncthreads();
    }
    if (t == 0) *out = s[0];
}

// finalize_plastic_iteration_pass! (E:4142-4169); `rollback` when
// iplast % dtstep == 0
__global__ void k_finalize_plastic(Geo g, GridPtrs G, int rollback) {
    NODE_B(g, t);
    (void)i; (void)j;
    double e = rollback ? G.ETA00[t] : G.ETA5[t];
    uint8_t y = rollback ? G.YNY00[t] : G.YNY5[t];
    G.ETA[t] = e;
    G.YNY[t] = y;
    G.YNY_inv_ETA[t] = (double)y / e;
}

// compute_shear_heating! (E:4415-4433)
__global__ void k_shear_heating(Geo g, GridPtrs G) {
    NODE_P(g, t);
    if (i < 2 || i > g.Ny || j < 2 || j > g.Nx) return;
    int Ny = g.Ny, Ny1 = g.Ny1;
    double s1 = AT(G.SXY, Ny, i - 1, j - 1), s2 = AT(G.SXY, Ny, i, j - 1);
    double s3 = AT(G.SXY, Ny, i - 1, j), s4 = AT(G.SXY, Ny, i, j);
    double SXYEXY = 0.25 * (s1 * s1 / AT(G.ETA, Ny, i - 1, j - 1) + s2 * s2 / AT(G.ETA, Ny, i, j - 1) +
                            s3 * s3 / AT(G.ETA, Ny, i - 1, j) + s4 * s4 / AT(G.ETA, Ny, i, j));
    double sxx = G.SXX[t], dp = G.pr[t] - G.pf[t];
    double q1 = AT(G.qxD, Ny1, i, j - 1), q2 = G.qxD[t];
    double q3 = AT(G.qyD, Ny1, i - 1, j), q4 = G.qyD[t];
    G.HS[t] = sxx * sxx / G.ETAP[t] + SXYEXY + dp * dp / (1 - G.PHI[t]) / G.ETAPHI[t] +
              0.5 * (AT(G.RX, Ny1, i, j - 1) * (q1 * q1) + G.RX[t] * (q2 * q2)) +
              0.5 * (AT(G.RY, Ny1, i - 1, j) * (q3 * q3) + G.RY[t] * (q4 * q4));
}

// compute_adiabatic_heating! (E:4458-4501), with the reference's use of the
// solid-pressure gradients in the fluid term (E:4492)
__global__ void k_adiabatic_heating(Geo g, GridPtrs G) {
    NODE_P(g, t);
    if (i < 2 || i > g.Ny || j < 2 || j > g.Nx) return;
    int Ny1 = g.Ny1;
    double idx = 1.0 / g.dx, idy = 1.0 / g.dy;
    double VXP = 0.5 * (G.vx[t] + AT(G.vx, Ny1, i, j - 1));
    double VYP = 0.5 * (G.vy[t] + AT(G.vy, Ny1, i - 1, j));
    double VXFP = 0.5 * (G.vxf[t] + AT(G.vxf, Ny1, i, j - 1));
    double VYFP = 0.5 * (G.vyf[t] + AT(G.vyf, Ny1, i - 1, j));
    double dpsdx = VXP < 0.0 ? (G.ps[t] - AT(G.ps, Ny1, i, j - 1)) * idx
                             : (AT(G.ps, Ny1, i, j + 1) - G.ps[t]) * idx;
    double dpsdy = VYP < 0.0 ? (G.ps[t] - AT(G.ps, Ny1, i - 1, j)) * idy
                             : (AT(G.ps, Ny1, i + 1, j) - G.ps[t]) * idy;
    double dpsdt = VXP * dpsdx + VYP * dpsdy;
    double dpfdt = VXFP * dpsdx + VYFP * dpsdy;
    double ph = G.PHI[t], tk = G.tk1[t];
    G.HA[t] = (1 - ph) * tk * G.ALPHA[t] * dpsdt + ph * tk * G.ALPHAF[t] * dpfdt;
}

// tk2 from the solution, DT = tk2 - tk1 (E:6926-6927) and the maxima of
// E:6929, E:4218-4219
__global__ void k_thermal_post(Geo g, GridPtrs G, const double *S, DevScalars *sc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < g.Ny1 * g.Nx1;
    double d = 0.0, e = 0.0, m = 0.0;
    if (in) {
        double tk2 = S[t];
        G.tk2[t] = tk2;
        d = tk2 - G.tk1[t];
        G.DT[t] = d;
        e = G.pf[t] - G.pf0[t];
        m = G.DMP[t];
    }
    amax_warp(&sc->maxabs[X_DT], d, in);
    amax_warp(&sc->maxabs[X_PFERR], e, in);
    amax_warp(&sc->maxabs[X_DMP], m, in);
}

// compute_velocities! (E:4878-4928): interior, then rows, then columns
__global__ void k_vel_interior(Geo g, GridPtrs G) {
    NODE_P(g, t);
    if (i < 2 || i > g.Ny || j < 2 || j > g.Nx) return;
    int Ny1 = g.Ny1;
    G.vxp[t] = 0.5 * (G.vx[t] + AT(G.vx, Ny1, i, j - 1));
    G.vyp[t] = 0.5 * (G.vy[t] + AT(G.vy, Ny1, i - 1, j));
    G.vxpf[t] = 0.5 * (G.vxf[t] + AT(G.vxf, Ny1, i, j - 1));
    G.vypf[t] = 0.5 * (G.vyf[t] + AT(G.vyf, Ny1, i - 1, j));
}
__global__ void k_vel_edges1(ErebusParams p, Geo g, GridPtrs G) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int Ny1 = g.Ny1, Nx = g.Nx, Ny = g.Ny;
    // vxp/vxpf rows 1, Ny1 for j = 2..Nx-1; vyp/vypf columns 1, Nx1 for i = 2..Ny-1
    int j = k + 2;
    if (j <= Nx - 1) {
        AT(G.vxp, Ny1, 1, j) = -p.bctop * AT(G.vxp, Ny1, 2, j);
        AT(G.vxp, Ny1, Ny1, j) = -p.bcbottom * AT(G.vxp, Ny1, Ny, j);
        AT(G.vxpf, Ny1, 1, j) = -p.bcftop * AT(G.vxpf, Ny1, 2, j);
        AT(G.vxpf, Ny1, Ny1, j) = -p.bcfbottom * AT(G.vxpf, Ny1, Ny, j);
    }
    int i = k + 2;
    if (i <= Ny - 1) {
        AT(G.vyp, Ny1, i, 1) = -p.bcleft * AT(G.vyp, Ny1, i, 2);
        AT(G.vyp, Ny1, i, g.Nx1) = -p.bcright * AT(G.vyp, Ny1, i, Nx);
        AT(G.vypf, Ny1, i, 1) = -p.bcfleft * AT(G.vypf, Ny1, i, 2);
        AT(G.vypf, Ny1, i, g.Nx1) = -p.bcfright * AT(G.vypf, Ny1, i, Nx);
    }
}
__global__ void k_vel_edges2(Geo g, GridPtrs G) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int Ny1 = g.Ny1, Nx1 = g.Nx1;
    int i = k + 1;
    if (i <= Ny1) {   // vxp/vxpf columns 1, Nx1 (all rows)
        AT(G.vxp, Ny1, i, 1) = 2.0 * g.vxleft - AT(G.vxp, Ny1, i, 2);
        AT(G.vxp, Ny1, i, Nx1) = 2.0 * g.vxright - AT(G.vxp, Ny1, i, g.Nx);
        AT(G.vxpf, Ny1, i, 1) = 2.0 * g.vxleft - AT(G.vxpf, Ny1, i, 2);
        AT(G.vxpf, Ny1, i, Nx1) = 2.0 * g.vxright - AT(G.vxpf, Ny1, i, g.Nx);
    }
    int j = k + 1;
    if (j <= Nx1) {   // vyp/vypf rows 1, Ny1 (all columns)
        AT(G.vyp, Ny1, 1, j) = 2.0 * g.vytop - AT(G.vyp, Ny1, 2, j);
        AT(G.vyp, Ny1, Ny1, j) = 2.0 * g.vybottom - AT(G.vyp, Ny1, g.Ny, j);
        AT(G.vypf, Ny1, 1, j) = 2.0 * g.vytop - AT(G.vypf, Ny1, 2, j);
        AT(G.vypf, Ny1, Ny1, j) = 2.0 * g.vybottom - AT(G.vypf, Ny1, g.Ny, j);
    }
}

// compute_rotation_rate! (E:4946-4956)
__global__ void k_rotation(Geo g, GridPtrs G) {
    NODE_B(g, t);
    int Ny1 = g.Ny1;
    G.wyx[t] = 0.5 * ((AT(G.vy, Ny1, i, j + 1) - AT(G.vy, Ny1, i, j)) * (1.0 / g.dx) -
                      (AT(G.vx, Ny1, i + 1, j) - AT(G.vx, Ny1, i, j)) * (1.0 / g.dy));
}

// ---------------------------------------------------------------------------
// host wrappers
// ---------------------------------------------------------------------------
static int np_of(erebus_state *s) { return s->g.Nx1 * s->g.Ny1; }
static int nb_of(erebus_state *s) { return s->g.Nx * s->g.Ny; }

int gravity_post(erebus_state *s) {
    EREBUS_LAUNCH(s, k_gravity_post, nblocks(np_of(s)), kThreads, 0, s->g, grid_ptrs(s));
    return check_cuda(s, cudaGetLastError(), "gravity_post");
}

int bulk_viscosity(erebus_state *s) {
    EREBUS_LAUNCH(s, k_bulk_viscosity, nblocks(np_of(s)), kThreads, 0, s->p, s->g,
                  grid_ptrs(s));
    return check_cuda(s, cudaGetLastError(), "bulk_viscosity");
}

// E:6754-6846 after the solve: unpack, Aphi, fluid velocities, dt limit,
// stresses, Aphi again, symmetrize, nodal adjustment.  Leaves dt, ynpl and
// the yielding error sum in the device scalars.
static int hydro_post_launch(erebus_state *s, const double *S) {
    int np = np_of(s), nb = nb_of(s);
    GridPtrs G = grid_ptrs(s);
    cudaMemsetAsync(s->dsc->maxabs, 0, sizeof(s->dsc->maxabs), s->stream);
    cudaMemsetAsync(&s->dsc->ynpl, 0, sizeof(int), s->stream);
    EREBUS_LAUNCH(s, k_hydro_post, nblocks(np), kThreads, 0, s->p, s->g, G, S);
    EREBUS_LAUNCH(s, k_aphi, nblocks(np), kThreads, 0, s->g, G, s->dsc);
    double *tx = s->tmp_node, *ty = s->tmp_node + np;
    EREBUS_LAUNCH(s, k_fluid_pre, nblocks(np), kThreads, 0, s->p, s->g, G, tx, ty);
    EREBUS_LAUNCH(s, k_fluid_fin, nblocks(np), kThreads, 0, s->g, G, tx, ty, s->dsc);
    EREBUS_LAUNCH(s, k_displacement_dt, 1, 1, 0, s->p, s->g, s->dsc);
    EREBUS_LAUNCH(s, k_stress_basic, nblocks(nb), kThreads, 0, s->g, G, s->dsc);
    EREBUS_LAUNCH(s, k_stress_p, nblocks(np), kThreads, 0, s->g, G, s->dsc);
    EREBUS_LAUNCH(s, k_aphi, nblocks(np), kThreads, 0, s->g, G, s->dsc);
    EREBUS_LAUNCH(s, k_sym_rows, nblocks(s->g.Nx), kThreads, 0, s->g, G);
    EREBUS_LAUNCH(s, k_sym_cols_ps, nblocks(np), kThreads, 0, s->g, G);
    double *dd = s->tmp_node;
    EREBUS_LAUNCH(s, k_nodal, nblocks(nb), kThreads, 0, s->p, s->g, G, s->dsc, s->dsc, dd);
    EREBUS_LAUNCH(s, k_sum_fixed, 1, 1024, 0, dd, nb, &s->dsc->sum_ddd);
    return check_cuda(s, cudaGetLastError(), "hydro_post");
}

// The post-processing of a Stokes-Darcy pass is a fixed sequence of 13
// kernels and 2 memsets whose arguments (parameters, geometry, grid and
// scratch buffers, all fixed at erebus_create) change only with the solution
// vector S.  It runs right after the host has read the refinement's
// residual, so launched one by one the GPU waits on the host's launch rate.
// It is captured into a CUDA graph once per S and replayed with one launch.
// The graph freezes every by-value argument (s->p, s->g, the grid pointers,
// tmp_node, dsc).  That is correct only because none of them changes after
// erebus_create: any future entry point that changes the parameters or
// rebinds the grid must destroy s->post_graph so that it is captured again.
int hydro_post(erebus_state *s, const double *S) {
    if (!s->post_graph || s->post_graph_S != S) {
        if (s->post_graph) {
            cudaGraphExecDestroy(s->post_graph);
            s->post_graph = nullptr;
        }
        const int64_t l0 = s->launches;
        int rc = check_cuda(s, cudaStreamBeginCapture(s->stream,
                                                      cudaStreamCaptureModeThreadLocal),
                            "hydro_post capture");
        if (rc) return rc;
        rc = hydro_post_launch(s, S);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s->stream, &g);
        if (!rc) rc = check_cuda(s, e, "hydro_post capture");
        if (!rc) rc = check_cuda(s, cudaGraphInstantiate(&s->post_graph, g, 0),
                                 "hydro_post graph");
        if (g) cudaGraphDestroy(g);
        s->post_graph_launches = s->launches - l0;
        s->launches = l0;
        if (rc) {
            s->post_graph = nullptr;
            return rc;
        }
        s->post_graph_S = S;
    }
    s->launches += s->post_graph_launches;
    return check_cuda(s, cudaGraphLaunch(s->post_graph, s->stream), "hydro_post");
}

int finalize_plastic(erebus_state *s, int rollback) {
    EREBUS_LAUNCH(s, k_finalize_plastic, nblocks(nb_of(s)), kThreads, 0, s->g, grid_ptrs(s),
                  rollback);
    return check_cuda(s, cudaGetLastError(), "finalize_plastic");
}

int heating(erebus_state *s) {
    GridPtrs G = grid_ptrs(s);
    EREBUS_LAUNCH(s, k_shear_heating, nblocks(np_of(s)), kThreads, 0, s->g, G);
    return check_cuda(s, cudaGetLastError(), "shear_heating");
}
int adiabatic(erebus_state *s) {
    EREBUS_LAUNCH(s, k_adiabatic_heating, nblocks(np_of(s)), kThreads, 0, s->g, grid_ptrs(s));
    return check_cuda(s, cudaGetLastError(), "adiabatic_heating");
}

int thermal_post(erebus_state *s, const double *S) {
    cudaMemsetAsync(&s->dsc->maxabs[X_DT], 0, 3 * sizeof(double), s->stream);
    EREBUS_LAUNCH(s, k_thermal_post, nblocks(np_of(s)), kThreads, 0, s->g, grid_ptrs(s), S,
                  s->dsc);
    return check_cuda(s, cudaGetLastError(), "thermal_post");
}

int velocities_rotation(erebus_state *s) {
    GridPtrs G = grid_ptrs(s);
    int np = np_of(s);
    int edge = (s->g.Nx1 > s->g.Ny1 ? s->g.Nx1 : s->g.Ny1);
    EREBUS_LAUNCH(s, k_vel_interior, nblocks(np), kThreads, 0, s->g, G);
    EREBUS_LAUNCH(s, k_vel_edges1, nblocks(edge), kThreads, 0, s->p, s->g, G);
    EREBUS_LAUNCH(s, k_vel_edges2, nblocks(edge), kThreads, 0, s->g, G);
    EREBUS_LAUNCH(s, k_rotation, nblocks(nb_of(s)), kThreads, 0, s->g, G);
    return check_cuda(s, cudaGetLastError(), "velocities");
}

}  // namespace erebus
