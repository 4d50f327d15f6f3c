// assemble.cu -- the three linear systems of a timestep, assembled on the
// device.
//
// One device function per equation row emits that row's entries in the
// order of the reference's updateindex! calls: the Stokes-Darcy system of
// assemble_hydromechanical_lse! (E:3089-3572), the heat equation of
// assemble_thermal_lse! (E:4526-4611) and the self-gravity Poisson equation
// of assemble_gravitational_lse! (E:2798-2848).  The rows are written either
// as COO triplets (parity export) or, scaled by the inverse of their
// absolute row sum, into the block-banded storage of the LU solver (the row
// scaling UMFPACK applies by default; without it the pressures at
// sticky-air nodes, whose rows are ~1e-24 smaller than the Darcy rows, are
// undetermined to ~1e7 Pa).
#include "solver.cuh"

namespace erebus {

// ---------------------------------------------------------------------------
// row functions
// ---------------------------------------------------------------------------
struct Row {
    int n;
    int64_t col[12];
    double val[12];
    double rhs;
    __device__ void put(int64_t c, double v) {
        col[n] = c;
        val[n] = v;
        n++;
    }
};

// Row `eq` (0 vx, 1 vy, 2 Ptotal, 3 qx, 4 qy, 5 Pfluid) of node (i,j).
__device__ void hydro_row(const ErebusParams &p, const Geo &g, const GridPtrs &G,
                          double dt, int i, int j, int eq, Row &r) {
    const int Ny = g.Ny, Ny1 = g.Ny1, Nx = g.Nx, Nx1 = g.Nx1;
    const double dx = g.dx, dy = g.dy, Kc = p.Kcont;
    const int64_t S6 = 6 * (int64_t)Ny1;
    const int64_t kvx = ((int64_t)(j - 1) * Ny1 + i - 1) * 6;
    const int64_t kvy = kvx + 1, kpm = kvx + 2, kqx = kvx + 3, kqy = kvx + 4, kpf = kvx + 5;
    r.n = 0;
    r.rhs = 0.0;
    const double *ETA = G.ETA, *GGG = G.GGG, *SXY0 = G.SXY0;
    const double *ETAP = G.ETAP, *GGGP = G.GGGP, *SXX0 = G.SXX0;
    int ring = (i == 2 && 2 <= j && j <= Nx) || (j == 2 && 2 < i && i < Ny) ||
               (i == Ny && 2 <= j && j <= Nx) || (j == Nx && 2 < i && i < Ny);
    switch (eq) {
    case 0:  // x-Stokes (E:3128-3262)
        if (i == 1 || i == Ny1 || j == 1 || j == Nx || j == Nx1) {
            r.put(kvx, 1.0);
            if (j == 1) r.rhs = g.vxleft;
            if (j == Nx) r.rhs = g.vxright;
            if (i == 1 && 1 < j && j < Nx) r.put(kvx + 6, p.bctop);
            if (i == Ny1 && 1 < j && j < Nx) r.put(kvx - 6, p.bcbottom);
        } else {
            double e1 = AT(ETA, Ny, i - 1, j), g1 = AT(GGG, Ny, i - 1, j);
            double e2 = AT(ETA, Ny, i, j), g2 = AT(GGG, Ny, i, j);
            double ep1 = AT(ETAP, Ny1, i, j), gp1 = AT(GGGP, Ny1, i, j);
            double ep2 = AT(ETAP, Ny1, i, j + 1), gp2 = AT(GGGP, Ny1, i, j + 1);
            double ETA1 = e1 * g1 * dt / (g1 * dt + e1);
            double ETA2 = e2 * g2 * dt / (g2 * dt + e2);
            double ETAP1 = ep1 * gp1 * dt / (gp1 * dt + ep1);
            double ETAP2 = ep2 * gp2 * dt / (gp2 * dt + ep2);
            double SXY1 = AT(SXY0, Ny, i - 1, j) * e1 / (g1 * dt + e1);
            double SXY2 = AT(SXY0, Ny, i, j) * e2 / (g2 * dt + e2);
            double SXX1 = AT(SXX0, Ny1, i, j) * ep1 / (gp1 * dt + ep1);
            double SXX2 = AT(SXX0, Ny1, i, j + 1) * ep2 / (gp2 * dt + ep2);
            double dRdx = 0.5 * (AT(G.RHOX, Ny1, i, j + 1) - AT(G.RHOX, Ny1, i, j - 1)) * (1.0 / dx);
            double dRdy = 0.5 * (AT(G.RHOX, Ny1, i + 1, j) - AT(G.RHOX, Ny1, i - 1, j)) * (1.0 / dy);
            double gxij = AT(G.gx, Ny1, i, j);
            double idx = 1.0 / dx, idy = 1.0 / dy;
            r.put(kvx - S6, ETAP1 / (dx * dx));
            r.put(kvx - 6, ETA1 / (dy * dy));
            r.put(kvx, -(ETAP1 + ETAP2) * (1.0 / (dx * dx)) - (ETA1 + ETA2) * (1.0 / (dy * dy)) -
                           dRdx * gxij * dt);
            r.put(kvx + 6, ETA2 / (dy * dy));
            r.put(kvx + S6, ETAP2 / (dx * dx));
            r.put(kvy, ETAP1 * idx * idy - ETA2 * idx * idy - dRdy * gxij * dt * 0.25);
            r.put(kvy + S6, -ETAP2 * idx * idy + ETA2 * idx * idy - dRdy * gxij * dt * 0.25);
            r.put(kvy - 6, -ETAP1 * idx * idy + ETA1 * idx * idy - dRdy * gxij * dt * 0.25);
            r.put(kvy + S6 - 6, ETAP2 * idx * idy - ETA1 * idx * idy - dRdy * gxij * dt * 0.25);
            r.put(kpm, Kc * idx);
            r.put(kpm + S6, -Kc * idx);
            r.rhs = -AT(G.RHOX, Ny1, i, j) * gxij - (SXY2 - SXY1) * idy - (SXX2 - SXX1) * idx;
        }
        break;
    case 1:  // y-Stokes (E:3264-3396)
        if (i == 1 || i == Ny || i == Ny1 || j == 1 || j == Nx1) {
            r.put(kvy, 1.0);
            if (i == 1) r.rhs = g.vytop;
            if (i == Ny) r.rhs = g.vybottom;
            if (j == 1 && 1 < i && i < Ny) r.put(kvy + S6, p.bcleft);
            if (j == Nx1 && 1 < i && i < Ny) r.put(kvy - S6, p.bcright);
        } else {
            double e1 = AT(ETA, Ny, i, j - 1), g1 = AT(GGG, Ny, i, j - 1);
            double e2 = AT(ETA, Ny, i, j), g2 = AT(GGG, Ny, i, j);
            double ep1 = AT(ETAP, Ny1, i, j), gp1 = AT(GGGP, Ny1, i, j);
            double ep2 = AT(ETAP, Ny1, i + 1, j), gp2 = AT(GGGP, Ny1, i + 1, j);
            double ETA1 = e1 * g1 * dt / (g1 * dt + e1);
            double ETA2 = e2 * g2 * dt / (g2 * dt + e2);
            double ETAP1 = ep1 * gp1 * dt / (gp1 * dt + ep1);
            double ETAP2 = ep2 * gp2 * dt / (gp2 * dt + ep2);
            double SXY1 = AT(SXY0, Ny, i, j - 1) * e1 / (g1 * dt + e1);
            double SXY2 = AT(SXY0, Ny, i, j) * e2 / (g2 * dt + e2);
            double SYY1 = -AT(SXX0, Ny1, i, j) * ep1 / (gp1 * dt + ep1);
            double SYY2 = -AT(SXX0, Ny1, i + 1, j) * ep2 / (gp2 * dt + ep2);
            double dRdx = 0.5 * (AT(G.RHOY, Ny1, i, j + 1) - AT(G.RHOY, Ny1, i, j - 1)) / dx;
            double dRdy = 0.5 * (AT(G.RHOY, Ny1, i + 1, j) - AT(G.RHOY, Ny1, i - 1, j)) / dy;
            double gyij = AT(G.gy, Ny1, i, j);
            double idx = 1.0 / dx, idy = 1.0 / dy;
            r.put(kvy - S6, ETA1 / (dx * dx));
            r.put(kvy - 6, ETAP1 / (dy * dy));
            r.put(kvy, -(ETAP1 + ETAP2) * (1.0 / (dy * dy)) - (ETA1 + ETA2) * (1.0 / (dx * dx)) -
                           dRdy * gyij * dt);
            r.put(kvy + 6, ETAP2 * (1.0 / (dy * dy)));
            r.put(kvy + S6, ETA2 * (1.0 / (dx * dx)));
            r.put(kvx, ETAP1 * idx * idy - ETA2 * idx * idy - dRdx * gyij * dt * 0.25);
            r.put(kvx + 6, -ETAP2 * idx * idy + ETA2 * idx * idy - dRdx * gyij * dt * 0.25);
            r.put(kvx - S6, -ETAP1 * idx * idy + ETA1 * idx * idy - dRdx * gyij * dt * 0.25);
            r.put(kvx + 6 - S6, ETAP2 * idx * idy - ETA1 * idx * idy - dRdx * gyij * dt * 0.25);
            r.put(kpm, Kc * idy);
            r.put(kpm + 6, -Kc * idy);
            r.rhs = -AT(G.RHOY, Ny1, i, j) * gyij - (SXY2 - SXY1) * idx - (SYY2 - SYY1) * idy;
        }
        break;
    case 2:  // P total continuity (E:3398-3452)
        if (i == 1 || i == Ny1 || j == 1 || j == Nx1) {
            r.put(kpm, 1.0);
        } else if (ring) {
            r.put(kpm, Kc);
            r.rhs = p.psurface;
        } else {
            double ph = AT(G.PHI, Ny1, i, j), etph = AT(G.ETAPHI, Ny1, i, j);
            double bph = AT(G.BETAPHI, Ny1, i, j);
            r.put(kvx - S6, -1.0 / dx);
            r.put(kvx, 1.0 / dx);
            r.put(kvy - 6, -1.0 / dy);
            r.put(kvy, 1.0 / dy);
            r.put(kpm, Kc / (1 - ph) * (1.0 / etph + bph / dt));
            r.put(kpf, -Kc / (1 - ph) * (1.0 / etph + bph / dt));
            r.rhs = (AT(G.pr0, Ny1, i, j) - AT(G.pf0, Ny1, i, j)) / (1 - ph) * bph / dt +
                    AT(G.DMP, Ny1, i, j);
        }
        break;
    case 3:  // qx Darcy (E:3454-3480)
        if (i == 1 || i == Ny1 || j == 1 || j == Nx || j == Nx1) {
            r.put(kqx, 1.0);
            if (i == 1 && 1 < j && j < Nx) r.put(kqx + 6, p.bcftop);
            if (i == Ny1 && 1 < j && j < Nx) r.put(kqx - 6, p.bcfbottom);
        } else {
            r.put(kqx, AT(G.RX, Ny1, i, j));
            r.put(kpf, -Kc * (1.0 / dx));
            r.put(kpf + S6, Kc * (1.0 / dx));
            r.rhs = AT(G.RHOFX, Ny1, i, j) * AT(G.gx, Ny1, i, j);
        }
        break;
    case 4:  // qy Darcy (E:3482-3514)
        if (i == 1 || i == Ny || i == Ny1 || j == 1 || j == Nx1) {
            r.put(kqy, 1.0);
            if (j == 1 && 1 < i && i < Ny) r.put(kqy + S6, p.bcfleft);
            if (j == Nx1 && 1 < i && i < Ny) r.put(kqy - S6, p.bcfright);
        } else {
            r.put(kqy, AT(G.RY, Ny1, i, j));
            r.put(kpf, -Kc * (1.0 / dy));
            r.put(kpf + 6, Kc * (1.0 / dy));
            r.rhs = AT(G.RHOFY, Ny1, i, j) * AT(G.gy, Ny1, i, j);
        }
        break;
    default:  // P fluid continuity (E:3516-3565)
        if (i == 1 || i == Ny1 || j == 1 || j == Nx1) {
            r.put(kpf, 1.0);
        } else if (ring) {
            r.put(kpf, Kc);
            r.rhs = p.psurface;
        } else {
            double ph = AT(G.PHI, Ny1, i, j), etph = AT(G.ETAPHI, Ny1, i, j);
            double bph = AT(G.BETAPHI, Ny1, i, j);
            r.put(kqx - S6, -(1.0 / dx));
            r.put(kqx, 1.0 / dx);
            r.put(kqy - 6, -(1.0 / dy));
            r.put(kqy, 1.0 / dy);
            r.put(kpm, -Kc / (1.0 - ph) * (1.0 / etph + bph / dt));
            r.put(kpf, Kc / (1.0 - ph) * (1.0 / etph + bph / dt));
            r.rhs = -(AT(G.pr0, Ny1, i, j) - AT(G.pf0, Ny1, i, j)) / (1 - ph) * bph / dt;
        }
        break;
    }
}

// assemble_thermal_lse! row of node (i,j) (E:4534-4605)
__device__ void thermal_row(const Geo &g, const GridPtrs &G, double dt, int i, int j, Row &r) {
    const int Ny1 = g.Ny1, Nx1 = g.Nx1;
    const int64_t gk = (int64_t)(j - 1) * Ny1 + i - 1;
    r.n = 0;
    r.rhs = 0.0;
    if (i == 1 || i == Ny1 || j == 1 || j == Nx1) {
        r.put(gk, 1.0);
        if (j == 1) r.put(gk + Ny1, -1.0);
        if (j == Nx1) r.put(gk - Ny1, -1.0);
        if (i == 1 && 1 < j && j < Nx1) r.put(gk + 1, -1.0);
        if (i == Ny1 && 1 < j && j < Nx1) r.put(gk - 1, -1.0);
    } else {
        double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
        double Kx1 = AT(G.KX, Ny1, i, j - 1), Kx2 = AT(G.KX, Ny1, i, j);
        double Ky1 = AT(G.KY, Ny1, i - 1, j), Ky2 = AT(G.KY, Ny1, i, j);
        double rc = AT(G.RHOCP, Ny1, i, j);
        r.put(gk - Ny1, -Kx1 * idx2);
        r.put(gk - 1, -Ky1 * idy2);
        r.put(gk, rc / dt + (Kx1 + Kx2) * idx2 + (Ky1 + Ky2) * idy2);
        r.put(gk + 1, -Ky2 * idy2);
        r.put(gk + Ny1, -Kx2 * idx2);
        r.rhs = rc / dt * AT(G.tk1, Ny1, i, j) + AT(G.HR, Ny1, i, j) + AT(G.HA, Ny1, i, j) +
                AT(G.HS, Ny1, i, j) + AT(G.DHP, Ny1, i, j);
    }
}

// assemble_gravitational_lse! row of node (i,j) (E:2806-2844)
__device__ void gravity_row(const ErebusParams &p, const Geo &g, const GridPtrs &G, int i,
                            int j, Row &r) {
    const int Ny1 = g.Ny1, Nx1 = g.Nx1;
    const int64_t gk = (int64_t)(j - 1) * Ny1 + i - 1;
    r.n = 0;
    r.rhs = 0.0;
    double xpj = ax(-g.dx / 2, g.dx, j), ypi = ax(-g.dy / 2, g.dy, i);
    double dxc = xpj - g.xcenter, dyc = ypi - g.ycenter;
    double dist = sqrt(dxc * dxc + dyc * dyc);
    if (i == 1 || i == Ny1 || j == 1 || j == Nx1 || dist > g.xcenter) {
        r.put(gk, 1.0);
    } else {
        double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
        r.put(gk - Ny1, idx2);
        r.put(gk - 1, idy2);
        r.put(gk, -2.0 * (idx2 + idy2));
        r.put(gk + 1, idy2);
        r.put(gk + Ny1, idx2);
        r.rhs = 4.0 * 2.0 * (1.0 / 3.0) * 3.141592653589793 * p.G * AT(G.RHO, Ny1, i, j);
    }
}

__device__ __forceinline__ void system_row(int kind, const ErebusParams &p, const Geo &g,
                                           const GridPtrs &G, double dt, int64_t row,
                                           Row &r) {
    if (kind == SYS_HYDRO) {
        int64_t node = row / 6;
        int eq = (int)(row % 6);
        hydro_row(p, g, G, dt, (int)(node % g.Ny1) + 1, (int)(node / g.Ny1) + 1, eq, r);
    } else {
        int i = (int)(row % g.Ny1) + 1, j = (int)(row / g.Ny1) + 1;
        if (kind == SYS_THERMAL) thermal_row(g, G, dt, i, j, r);
        else gravity_row(p, g, G, i, j, r);
    }
}

// ---------------------------------------------------------------------------
// COO export (parity): 12 slots per row, unused slots col = -1
// ---------------------------------------------------------------------------
__global__ void k_assemble_coo(int kind, ErebusParams p, Geo g, GridPtrs G,
                               const double *dtp, int64_t n, int64_t *rows, int64_t *cols,
                               double *vals, double *rhs) {
    int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    Row r;
    system_row(kind, p, g, G, *dtp, row, r);
    for (int k = 0; k < 12; k++) {
        rows[row * 12 + k] = row;
        cols[row * 12 + k] = k < r.n ? r.col[k] : -1;
        vals[row * 12 + k] = k < r.n ? r.val[k] : 0.0;
    }
    rhs[row] = r.rhs;
}

// ---------------------------------------------------------------------------
// scaled block-banded assembly
// ---------------------------------------------------------------------------
// Rows -> scaled ELL entries, scaled right-hand side and row scales; any
// entry that differs from the last factorised matrix sets *changed.
__global__ void k_assemble_ell(int kind, ErebusParams p, Geo g, GridPtrs G,
                               const double *dtp, BandView B, const double *prev,
                               int *changed) {
    int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= B.NB * (int64_t)B.nb) return;
    int diff = 0;
    if (row >= B.n) {   // padding: identity rows
        B.rhs[row] = 0.0;
        B.rscale[row] = 1.0;
        for (int k = 0; k < B.ell; k++) {
            double v = k == 0 ? 1.0 : 0.0;
            B.ell_cols[row * B.ell + k] = k == 0 ? (int)row : -1;
            B.ell_vals[row * B.ell + k] = v;
            diff |= __double_as_longlong(prev[row * B.ell + k]) != __double_as_longlong(v);
        }
    } else {
        Row r;
        system_row(kind, p, g, G, *dtp, row, r);
        double sum = 0.0;
        for (int k = 0; k < r.n; k++) sum += fabs(r.val[k]);
        double sc = sum > 0.0 ? 1.0 / sum : 1.0;
        B.rhs[row] = r.rhs * sc;
        B.rscale[row] = sc;
        for (int k = 0; k < B.ell; k++) {
            double v = k < r.n ? r.val[k] * sc : 0.0;
            B.ell_cols[row * B.ell + k] = k < r.n ? (int)r.col[k] : -1;
            B.ell_vals[row * B.ell + k] = v;
            diff |= __double_as_longlong(prev[row * B.ell + k]) != __double_as_longlong(v);
        }
    }
    // one atomic per warp (every changed row of a refactored matrix sets it)
    const unsigned am = __activemask(), any = __ballot_sync(am, diff);
    if (any && (threadIdx.x & 31) == __ffs(am) - 1) atomicOr(changed, 1);
}

// Scaled ELL rows -> block-banded tiles (zeroed beforehand); also keeps the
// entries as the reference copy of the factorised matrix.
__global__ void k_ell_to_band(BandView B, double *prev) {
    int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= B.NB * (int64_t)B.nb) return;
    for (int k = 0; k < B.ell; k++) {
        int c = B.ell_cols[row * B.ell + k];
        double v = B.ell_vals[row * B.ell + k];
        if (c >= 0) *band_at(B, row, c) += v;
        prev[row * B.ell + k] = v;
    }
}

// Assembles system `kind` from the current device state.  The LU factors
// are kept when the scaled matrix is bitwise equal to the one they were
// computed from (then only the right-hand side changes).
int assemble_system(erebus_state *s, int kind) {
    BandSystem &sys = band_of(s, kind);
    BandView B = band_view(sys);
    int64_t rows = (int64_t)sys.NB * sys.nb;
    cudaMemsetAsync(sys.changed, 0, sizeof(int), s->stream);
    EREBUS_LAUNCH(s, k_assemble_ell, nblocks(rows, 128), 128, 0, kind, s->p, s->g,
                  grid_ptrs(s), &s->dsc->dt, B, sys.ell_prev, sys.changed);
    int changed = 1;
    int rc = check_cuda(s, cudaMemcpyAsync(&changed, sys.changed, sizeof(int),
                                           cudaMemcpyDeviceToHost, s->stream), "assemble");
    if (rc) return rc;
    rc = stream_sync(s, "assemble");
    if (rc) return rc;
    if (changed || !sys.factored || !s->opt.reuse_factors) {
        rc = commit_assembly(s, sys);
        if (rc) return rc;
    }
    return check_cuda(s, cudaGetLastError(), "assemble");
}

int commit_assembly(erebus_state *s, BandSystem &sys) {
    int64_t rows = (int64_t)sys.NB * sys.nb;
    if (use_multifrontal(s)) {
        // the multifrontal factorisation reads the ELL entries itself
        int rc = check_cuda(s, cudaMemcpyAsync(sys.ell_prev, sys.ell_vals,
                                               rows * sys.ell * sizeof(double),
                                               cudaMemcpyDeviceToDevice, s->stream),
                            "assemble");
        if (rc) return rc;
    } else {
        int rc = band_zero(s, sys);   // allocates the band storage on first use
        if (rc) return rc;
        EREBUS_LAUNCH(s, k_ell_to_band, nblocks(rows, 128), 128, 0, band_view(sys),
                      sys.ell_prev);
    }
    sys.factored = false;
    return check_cuda(s, cudaGetLastError(), "assemble");
}

int export_system(erebus_state *s, int kind, int64_t *nnz_out, int64_t *rows_h,
                  int64_t *cols_h, double *vals_h, double *rhs_h) {
    BandSystem &sys = band_of(s, kind);
    int64_t n = sys.n;
    int64_t *dr = nullptr, *dc = nullptr;
    double *dv = nullptr, *db = nullptr;
    cudaError_t e = cudaMallocAsync(&dr, n * 12 * 8, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync(&dc, n * 12 * 8, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync(&dv, n * 12 * 8, s->stream);
    if (e == cudaSuccess) e = cudaMallocAsync(&db, n * 8, s->stream);
    int rc = check_cuda(s, e, "export alloc");
    if (rc) return rc;
    EREBUS_LAUNCH(s, k_assemble_coo, nblocks(n, 128), 128, 0, kind, s->p, s->g, grid_ptrs(s),
                  &s->dsc->dt, n, dr, dc, dv, db);
    std::vector<int64_t> r(n * 12), c(n * 12);
    std::vector<double> v(n * 12);
    cudaMemcpyAsync(r.data(), dr, n * 12 * 8, cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(c.data(), dc, n * 12 * 8, cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(v.data(), dv, n * 12 * 8, cudaMemcpyDeviceToHost, s->stream);
    if (rhs_h) cudaMemcpyAsync(rhs_h, db, n * 8, cudaMemcpyDeviceToHost, s->stream);
    rc = stream_sync(s, "export");
    cudaFreeAsync(dr, s->stream);
    cudaFreeAsync(dc, s->stream);
    cudaFreeAsync(dv, s->stream);
    cudaFreeAsync(db, s->stream);
    if (rc) return rc;
    int64_t k = 0;
    for (int64_t t = 0; t < n * 12; t++) {
        if (c[t] < 0) continue;
        if (rows_h) {
            rows_h[k] = r[t];
            cols_h[k] = c[t];
            vals_h[k] = v[t];
        }
        k++;
    }
    *nnz_out = k;
    return EREBUS_OK;
}

}  // namespace erebus
