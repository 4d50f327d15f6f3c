// adjoint.cu -- reverse-mode gradient of the heat path over several timesteps
// (erebus_adjoint_heat).  No reference counterpart: the reference has no
// derivatives; the gradient is that of its timestep (simulation_loop,
// E:6370-7235) for states at mechanical rest.
//
// Forward, per timestep n (at rest: markers fixed, porosity constant):
//   marker laws      rc_m = total(rcs, rcf(T_m), phi_m), k_m = ktotal(ks(T),
//                    kf(T), phi_m), hr_m = total(hrs(t_n), hrf(t_n), phi_m),
//                    tr_m = T_m rc_m                          (E:700-750)
//   scatter          Srcp, Str, Shr (P nodes), Skx, Sky (Vx, Vy nodes) and
//                    the weight sums W                       (E:1605-1863)
//   normalise        RHOCP = Srcp/W, tk1 = Str/Srcp, HR = Shr/W, KX, KY,
//                    then the insulating copies on tk1       (E:2033-2189, E:2432)
//   heat solve       A(RHOCP, KX, KY, dt) tk2 = RHOCP/dt tk1 + HR  (E:4526-4611)
//   markers          T_m += gather(tk2 - tk1), or gather(tk2) at timestep 1
//                                                            (E:4782-4801)
// J = mean over the basic nodes inside the body of the 4-P-node average of
// the last tk2 (grid_average, E:1176).
//
// Reverse, per timestep from the last: scatter the marker adjoint (marker
// order merge, as the forward scatter) into tk2_bar and -tk1_bar, solve
// A^T lambda = tk2_bar (the transposed heat system is assembled from the
// taped RHOCP, KX, KY, dt and factored by the same direct solver), form the
// adjoints of RHOCP, tk1, HR, KX, KY, undo the insulating copies and the
// normalisations, gather them to the markers and apply the derivatives of
// the marker laws.  Marker temperatures are checkpointed every k steps and
// recomputed in between from the taped node temperatures.
#include <algorithm>
#include <cmath>
#include <vector>
#include "laws.cuh"
#include "solver.cuh"

namespace erebus {

constexpr int ADJ_BLOCKS = 296;   // partial sums of the deterministic reductions

// Basic node (i,j) lies inside the body: distance from the centre < rplanet.
EREBUS_HD bool in_body(const Geo &g, double rplanet, int i, int j) {
    double dxc = ax(0.0, g.dx, j) - g.xcenter, dyc = ax(0.0, g.dy, i) - g.ycenter;
    return sqrt(dxc * dxc + dyc * dyc) < rplanet;
}

__device__ __forceinline__ bool inner_p(const Geo &g, int i, int j) {
    return i >= 2 && i <= g.Ny1 - 1 && j >= 2 && j <= g.Nx1 - 1;
}

// Sum over a 256-thread block (fixed order, so the result is deterministic).
__device__ double block_sum256(double v) {
    __shared__ double sh[8];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < 8; k++) r += sh[k];
    __syncthreads();
    return r;
}

__global__ void k_adj_sum(const double *part, int n, double *out) {
    double v = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) v += part[k];
    v = block_sum256(v);
    if (threadIdx.x == 0) *out = v;
}

// dJ/dtk2 of every P node: 0.25 for each adjacent basic node inside the body,
// over the number of such nodes.
__global__ void k_adj_seed(Geo g, double rplanet, double inv_nb, double *seed) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.Ny1 * g.Nx1) return;
    int I = t % g.Ny1 + 1, J = t / g.Ny1 + 1, c = 0;
    for (int bj = J - 1; bj <= J; bj++)
        for (int bi = I - 1; bi <= I; bi++)
            if (bi >= 1 && bi <= g.Ny && bj >= 1 && bj <= g.Nx && in_body(g, rplanet, bi, bj))
                c++;
    seed[t] = 0.25 * c * inv_nb;
}

// Partial sums of grid_average(tk2) over the basic nodes inside the body.
__global__ void k_adj_objective(Geo g, double rplanet, const double *tk2, double *part) {
    double v = 0.0;
    int nb = g.Ny * g.Nx;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += gridDim.x * blockDim.x) {
        int i = t % g.Ny + 1, j = t / g.Ny + 1;
        if (in_body(g, rplanet, i, j)) v += grid_average(tk2, g.Ny1, i, j);
    }
    v = block_sum256(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// Preconditions and postconditions on the markers: any non-zero stress, any
// position that differs bitwise from the start.
__global__ void k_adj_nonzero(const double *a, const double *b, int n, int *flag) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n && (a[m] != 0.0 || b[m] != 0.0)) atomicOr(flag, 1);
}
__global__ void k_adj_moved(const double *x0, const double *y0, const double *x,
                            const double *y, int n, int *flag) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n && (__double_as_longlong(x0[m]) != __double_as_longlong(x[m]) ||
                  __double_as_longlong(y0[m]) != __double_as_longlong(y[m])))
        atomicOr(flag, 1);
}

// Marker temperatures of the next step from the taped node fields, as
// update_marker_temperature! (E:4782-4801).
__global__ void k_adj_replay(Geo g, const double *xm, const double *ym, int n,
                             const double *Tin, double *Tout, const double *tk2,
                             const double *DT, int step_one) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    int i, j;
    double w[4];
    grid_weights(g, GP, xm[m], ym[m], i, j, w);
    Tout[m] = step_one ? gather4(tk2, g.Ny1, i, j, w) : Tin[m] + gather4(DT, g.Ny1, i, j, w);
}

// Row r of the transposed heat matrix (column r of assemble_thermal_lse!'s
// matrix, E:4526-4611), row-scaled, with right-hand side
// seed_scale * seed + S.  Entries in column order.  Any scaled entry that
// differs from the last factorised matrix (prev) sets *changed.
__global__ void k_adj_assemble(Geo g, const double *rhocp, const double *KX,
                               const double *KY, double dt, const double *seed,
                               double seed_scale, const double *S, BandView B,
                               const double *prev, int *changed) {
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B.NB * (int64_t)B.nb) return;
    int col[5];
    double val[5];
    int ne = 0;
    double rhs = 0.0;
    if (r >= B.n) {   // padding: identity rows
        col[ne] = (int)r;
        val[ne++] = 1.0;
    } else {
        const int R = g.Ny1, C = g.Nx1;
        const int i = (int)(r % R) + 1, j = (int)(r / R) + 1;
        const double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
        double v;
        // q = (i, j-1): its row reaches r as the right neighbour
        // (an interior q always has the entry, a boundary q only where its
        // row reads r, so the pattern does not depend on the values)
        if (j > 1 && (inner_p(g, i, j - 1) || j - 1 == 1)) {
            v = inner_p(g, i, j - 1) ? -AT(KX, R, i, j - 1) * idx2 : -1.0;
            col[ne] = (int)(r - R);
            val[ne++] = v;
        }
        // q = (i-1, j): reaches r as the lower neighbour
        if (i > 1 && (inner_p(g, i - 1, j) || (i - 1 == 1 && j > 1 && j < C))) {
            v = inner_p(g, i - 1, j) ? -AT(KY, R, i - 1, j) * idy2 : -1.0;
            col[ne] = (int)(r - 1);
            val[ne++] = v;
        }
        if (inner_p(g, i, j))
            v = AT(rhocp, R, i, j) / dt + (AT(KX, R, i, j - 1) + AT(KX, R, i, j)) * idx2 +
                (AT(KY, R, i - 1, j) + AT(KY, R, i, j)) * idy2;
        else
            v = 1.0;
        col[ne] = (int)r;
        val[ne++] = v;
        // q = (i+1, j): reaches r as the upper neighbour
        if (i < R && (inner_p(g, i + 1, j) || (i + 1 == R && j > 1 && j < C))) {
            v = inner_p(g, i + 1, j) ? -AT(KY, R, i, j) * idy2 : -1.0;
            col[ne] = (int)(r + 1);
            val[ne++] = v;
        }
        // q = (i, j+1): reaches r as the left neighbour
        if (j < C && (inner_p(g, i, j + 1) || j + 1 == C)) {
            v = inner_p(g, i, j + 1) ? -AT(KX, R, i, j) * idx2 : -1.0;
            col[ne] = (int)(r + R);
            val[ne++] = v;
        }
        rhs = seed_scale * seed[r] + (S ? S[r] : 0.0);
    }
    double sum = 0.0;
    for (int k = 0; k < ne; k++) sum += fabs(val[k]);
    double sc = sum > 0.0 ? 1.0 / sum : 1.0;
    B.rhs[r] = rhs * sc;
    B.rscale[r] = sc;
    int diff = 0;
    for (int k = 0; k < B.ell; k++) {
        double v = k < ne ? val[k] * sc : 0.0;
        B.ell_cols[r * B.ell + k] = k < ne ? col[k] : -1;
        B.ell_vals[r * B.ell + k] = v;
        diff |= __double_as_longlong(prev[r * B.ell + k]) != __double_as_longlong(v);
    }
    // one atomic per warp (every changed row of a refactored matrix sets it)
    const unsigned am = __activemask(), any = __ballot_sync(am, diff);
    if (any && (threadIdx.x & 31) == __ffs(am) - 1) atomicOr(changed, 1);
}

struct AdjNodeIn {
    const double *tk2, *DT, *rhocp, *lam, *S, *Wp, *Wx, *Wy;
    double dt;
    int minus;   // the marker update was T += gather(DT): -S enters tk1_bar
};
struct AdjNodeOut {
    double *srcp, *str, *shr, *skx, *sky;
};

// Adjoints of the scatter sums at every node of the (Ny1, Nx1) arrays.
__global__ void k_adj_nodes(Geo g, AdjNodeIn a, AdjNodeOut o) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int R = g.Ny1, C = g.Nx1;
    if (t >= R * C) return;
    const int i = t % R + 1, j = t / R + 1;
    const double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
    const double lam = a.lam[t];
    double srcp_b = 0.0, str_b = 0.0, shr_b = 0.0;
    if (inner_p(g, i, j) && a.Wp[t] > 0.0) {
        double wt = a.Wp[t], rc = a.rhocp[t];
        double tk1 = a.tk2[t] - a.DT[t];
        double rc_b = -lam * a.DT[t] / a.dt;   // from the diagonal and the RHS
        double t1b = lam * rc / a.dt;          // from the RHS
        if (a.minus) {
            // -S of this node and of the ghost nodes copied from it
            // (apply_insulating_boundary_conditions!, E:2432-2449)
            double s = a.S[t];
            bool top = i == 2, bot = i == R - 1, lft = j == 2, rgt = j == C - 1;
            if (top) s += AT(a.S, R, 1, j);
            if (bot) s += AT(a.S, R, R, j);
            if (lft) s += AT(a.S, R, i, 1);
            if (rgt) s += AT(a.S, R, i, C);
            if (top && lft) s += AT(a.S, R, 1, 1);
            if (top && rgt) s += AT(a.S, R, 1, C);
            if (bot && lft) s += AT(a.S, R, R, 1);
            if (bot && rgt) s += AT(a.S, R, R, C);
            t1b -= s;
        }
        double srcp = rc * wt;
        srcp_b = rc_b / wt - t1b * tk1 / srcp;
        str_b = t1b / srcp;
        shr_b = lam / wt;
    }
    // KX(i,j) enters rows (i,j) and (i,j+1); KY(i,j) rows (i,j) and (i+1,j)
    double kxb = 0.0, kyb = 0.0;
    if (inner_p(g, i, j)) {
        if (j < C) kxb -= lam * (a.tk2[t] - AT(a.tk2, R, i, j + 1)) * idx2;
        if (i < R) kyb -= lam * (a.tk2[t] - AT(a.tk2, R, i + 1, j)) * idy2;
    }
    if (j < C && inner_p(g, i, j + 1))
        kxb -= AT(a.lam, R, i, j + 1) * (AT(a.tk2, R, i, j + 1) - a.tk2[t]) * idx2;
    if (i < R && inner_p(g, i + 1, j))
        kyb -= AT(a.lam, R, i + 1, j) * (AT(a.tk2, R, i + 1, j) - a.tk2[t]) * idy2;
    o.srcp[t] = srcp_b;
    o.str[t] = str_b;
    o.shr[t] = shr_b;
    o.skx[t] = a.Wx[t] > 0.0 ? kxb / a.Wx[t] : 0.0;
    o.sky[t] = a.Wy[t] > 0.0 ? kyb / a.Wy[t] : 0.0;
}

struct AdjMarkerIn {
    const double *xm, *ym, *phim, *rcm, *T;
    const int8_t *tm;
    const double *srcp, *str, *shr, *skx, *sky;
    double hrs[3], hrf[3];
    double dQ;   // d hrs[t] / d ratio_al = dQ * rhosolidm[t]
    int keep;    // T_next = T + gather(DT): the marker adjoint carries over
};

// Marker adjoints: gathers of the node adjoints (transposed scatter) and the
// derivatives of the marker laws (E:700-750, E:1116-1234, E:2272-2358).
__global__ void k_adj_markers(ErebusParams p, Geo g, AdjMarkerIn a, int n, double *Tbar,
                              double *phibar, double *ratio_acc) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    double dr = 0.0;
    if (m < n) {
        int i, j;
        double w[4];
        double x = a.xm[m], y = a.ym[m];
        grid_weights(g, GP, x, y, i, j, w);
        double rcb = gather4(a.srcp, g.Ny1, i, j, w);
        double trb = gather4(a.str, g.Ny1, i, j, w);
        double hrb = gather4(a.shr, g.Ny1, i, j, w);
        grid_weights(g, GVX, x, y, i, j, w);
        double kb = gather4(a.skx, g.Ny1, i, j, w);
        grid_weights(g, GVY, x, y, i, j, w);
        kb += gather4(a.sky, g.Ny1, i, j, w);
        int t = a.tm[m];
        double T = a.T[m];
        double tb = a.keep ? Tbar[m] : 0.0;
        if (t < 3) {
            double phi = a.phim[m];
            double rcs = p.rhocpsolidm[t - 1], rcf = rhocpfluid(p, T);
            double rc = total(rcs, rcf, phi);
            double rcbt = rcb + trb * T;
            double ks = ksolid(p, T), kf = kfluid(p, T);
            KtotalGrad kg = ktotal_grad(ks, kf, phi);
            tb += trb * rc + rcbt * phi * rhocpfluid_dT(p, T) +
                  kb * (kg.ks * ksolid_dT(p, T) + kg.kf * kfluid_dT(p, T));
            phibar[m] += rcbt * (rcf - rcs) + kb * kg.phi +
                         hrb * (a.hrf[t - 1] - a.hrs[t - 1]);
            dr = hrb * (1.0 - phi) * a.dQ * p.rhosolidm[t - 1];
        } else {
            tb += trb * a.rcm[m];   // sticky air: constant properties
        }
        Tbar[m] = tb;
    }
    dr = block_sum256(dr);
    if (threadIdx.x == 0) ratio_acc[blockIdx.x] += dr;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

struct AdjLayout {
    double *tk2, *DT, *rhocp, *KX, *KY;   // N * np each
    double *ckpt, *Tseg;                  // nck * n, k * n
    double *Wp, *Wx, *Wy, *seed, *S, *Swt;
    double *srcp, *str, *shr, *skx, *sky;
    double *Tbar, *phibar, *x0, *y0;
    double *ratio_acc, *part, *out;
    int *flag;
};

size_t adj_words(int N, int nck, int k, int64_t n, int64_t np, int mblocks) {
    return (size_t)(5 * (int64_t)N + 11) * np + (size_t)(nck + k + 4) * n + mblocks +
           ADJ_BLOCKS + 8;
}

AdjLayout adj_layout(double *base, int N, int nck, int k, int64_t n, int64_t np,
                     int mblocks) {
    AdjLayout L;
    double *p = base;
    auto take = [&](int64_t words) {
        double *r = p;
        p += words;
        return r;
    };
    L.tk2 = take(N * np);
    L.DT = take(N * np);
    L.rhocp = take(N * np);
    L.KX = take(N * np);
    L.KY = take(N * np);
    L.Wp = take(np);
    L.Wx = take(np);
    L.Wy = take(np);
    L.seed = take(np);
    L.S = take(np);
    L.Swt = take(np);
    L.srcp = take(np);
    L.str = take(np);
    L.shr = take(np);
    L.skx = take(np);
    L.sky = take(np);
    L.ckpt = take(nck * n);
    L.Tseg = take(k * n);
    L.Tbar = take(n);
    L.phibar = take(n);
    L.x0 = take(n);
    L.y0 = take(n);
    L.ratio_acc = take(mblocks);
    L.part = take(ADJ_BLOCKS);
    L.out = take(4);
    L.flag = reinterpret_cast<int *>(take(4));
    return L;
}

int fail_adj(erebus_state *s, const char *msg) {
    s->last_error = std::string("adjoint: ") + msg;
    return EREBUS_EINVAL;
}

#define ATRY(x)                  \
    do {                         \
        int rc_ = (x);           \
        if (rc_) return rc_;     \
    } while (0)

int read_flag(erebus_state *s, int *flag, int *out) {
    ATRY(check_cuda(s, cudaMemcpyAsync(out, flag, sizeof(int), cudaMemcpyDeviceToHost,
                                       s->stream), "adjoint flag"));
    return stream_sync(s, "adjoint flag");
}

}  // namespace

}  // namespace erebus

using namespace erebus;

extern "C" int erebus_adjoint_heat(erebus_state *s, int32_t first_timestep, int32_t n_steps,
                                   int32_t checkpoint_every, double *J, double *dJ_dphim,
                                   double *dJ_dratio_al, ErebusAdjointStats *st) {
    if (!s || first_timestep < 1 || n_steps < 1 || checkpoint_every < 1)
        return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    const ErebusParams &p = s->p;
    const Geo &g = s->g;
    if (p.G != 0.0 || p.reaction_active || p.dsubgrids != 0.0 || p.dsubgridt != 0.0 ||
        p.strainrate != 0.0)
        return fail_adj(s, "the state is not at mechanical rest (needs G = 0, no strain "
                           "rate, reactions off, no subgrid diffusion)");
    const int64_t n = s->marknum;
    if (n < 1) return fail_adj(s, "no markers");
    const int N = n_steps, k = checkpoint_every > n_steps ? n_steps : checkpoint_every;
    const int nck = (N + k - 1) / k;
    const int64_t np = (int64_t)g.Nx1 * g.Ny1;
    const int mblocks = nblocks(n);
    // basic nodes inside the body
    int64_t nbody = 0;
    for (int j = 1; j <= g.Nx; j++)
        for (int i = 1; i <= g.Ny; i++) nbody += in_body(g, p.rplanet, i, j);
    if (nbody == 0) return fail_adj(s, "no basic node inside the body");

    size_t words = adj_words(N, nck, k, n, np, mblocks);
    if (s->adj_cap < words) {
        if (s->adj_mem) cudaFree(s->adj_mem);
        s->adj_mem = nullptr;
        s->adj_cap = 0;
        if (cudaMalloc(&s->adj_mem, words * sizeof(double)) != cudaSuccess) {
            s->last_error = "adjoint: tape allocation failed";
            return EREBUS_ENOMEM;
        }
        s->adj_cap = words;
    }
    AdjLayout L = adj_layout(s->adj_mem, N, nck, k, n, np, mblocks);
    if (!s->heat_adjoint.x) {
        if (band_alloc(s, s->heat_adjoint, np, g.Ny1, 64, 5)) return EREBUS_ENOMEM;
        s->heat_adjoint.name = "heat adjoint";
    }
    BandSystem &A = s->heat_adjoint;
    int f0 = A.factorizations;

    // preconditions on the markers
    int flag = 0;
    ATRY(check_cuda(s, cudaMemsetAsync(L.flag, 0, sizeof(int), s->stream), "adjoint"));
    EREBUS_LAUNCH(s, k_adj_nonzero, nblocks(n), kThreads, 0, s->m[M_sxxm], s->m[M_sxym],
                  (int)n, L.flag);
    ATRY(read_flag(s, L.flag, &flag));
    if (flag) return fail_adj(s, "non-zero marker stresses");
    cudaMemcpyAsync(L.x0, s->m[M_xm], n * 8, cudaMemcpyDeviceToDevice, s->stream);
    cudaMemcpyAsync(L.y0, s->m[M_ym], n * 8, cudaMemcpyDeviceToDevice, s->stream);

    // ---- forward: timesteps, tape, checkpoints ----
    std::vector<double> dts(N), times(N);
    for (int q = 0; q < N; q++) {
        if (q % k == 0)
            cudaMemcpyAsync(L.ckpt + (size_t)(q / k) * n, s->m[M_tkm], n * 8,
                            cudaMemcpyDeviceToDevice, s->stream);
        double expect = std::fmin(s->dt * p.dtcoefup, p.dt_longest);
        times[q] = s->timesum;
        ErebusStepStats ss = {};
        ATRY(erebus_step(s, first_timestep + q, &ss));
        if (ss.titer != 1 || ss.dt != expect)
            return fail_adj(s, "a time-step limiter acted or a second thermochemical "
                               "iteration was taken");
        if (ss.marknum != n) return fail_adj(s, "the marker count changed");
        dts[q] = ss.dt;
        const size_t o = (size_t)q * np, b = np * 8;
        cudaMemcpyAsync(L.tk2 + o, s->grid[G_tk2], b, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(L.DT + o, s->grid[G_DT], b, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(L.rhocp + o, s->grid[G_RHOCP], b, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(L.KX + o, s->grid[G_KX], b, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(L.KY + o, s->grid[G_KY], b, cudaMemcpyDeviceToDevice, s->stream);
        if (q == 0) {
            cudaMemcpyAsync(L.Wp, s->sums[S_WTPSUM], b, cudaMemcpyDeviceToDevice, s->stream);
            cudaMemcpyAsync(L.Wx, s->sums[S_WTXSUM], b, cudaMemcpyDeviceToDevice, s->stream);
            cudaMemcpyAsync(L.Wy, s->sums[S_WTYSUM], b, cudaMemcpyDeviceToDevice, s->stream);
        }
    }
    ATRY(check_cuda(s, cudaMemsetAsync(L.flag, 0, sizeof(int), s->stream), "adjoint"));
    EREBUS_LAUNCH(s, k_adj_moved, nblocks(n), kThreads, 0, L.x0, L.y0, s->m[M_xm],
                  s->m[M_ym], (int)n, L.flag);
    ATRY(read_flag(s, L.flag, &flag));
    if (flag) return fail_adj(s, "markers moved");

    // ---- objective ----
    const double *tk2N = L.tk2 + (size_t)(N - 1) * np;
    EREBUS_LAUNCH(s, k_adj_objective, ADJ_BLOCKS, 256, 0, g, p.rplanet, tk2N, L.part);
    EREBUS_LAUNCH(s, k_adj_sum, 1, 256, 0, L.part, ADJ_BLOCKS, L.out);
    EREBUS_LAUNCH(s, k_adj_seed, nblocks(np), kThreads, 0, g, p.rplanet, 1.0 / (double)nbody,
                  L.seed);

    // ---- reverse ----
    ATRY(build_cell_sort(s));   // markers are where the forward scattered them
    cudaMemsetAsync(L.Tbar, 0, n * 8, s->stream);
    cudaMemsetAsync(L.phibar, 0, n * 8, s->stream);
    cudaMemsetAsync(L.ratio_acc, 0, mblocks * 8, s->stream);
    int solves = 0;
    const int64_t rows = (int64_t)A.NB * A.nb;
    for (int seg = nck - 1; seg >= 0; seg--) {
        const int s0 = seg * k, s1 = std::min(s0 + k, N) - 1;
        // marker temperatures T^q for q = s0..s1 from the checkpoint
        cudaMemcpyAsync(L.Tseg, L.ckpt + (size_t)seg * n, n * 8, cudaMemcpyDeviceToDevice,
                        s->stream);
        for (int q = s0; q < s1; q++)
            EREBUS_LAUNCH(s, k_adj_replay, nblocks(n), kThreads, 0, g, s->m[M_xm],
                          s->m[M_ym], (int)n, L.Tseg + (size_t)(q - s0) * n,
                          L.Tseg + (size_t)(q - s0 + 1) * n, L.tk2 + (size_t)q * np,
                          L.DT + (size_t)q * np, first_timestep + q == 1);
        for (int q = s1; q >= s0; q--) {
            const bool last = q == N - 1;
            const size_t o = (size_t)q * np;
            if (!last) ATRY(scatter_p_values(s, L.Tbar, L.S, L.Swt));
            // the factors of the previous (later) step are kept when the
            // transposed matrix is bitwise the same
            ATRY(check_cuda(s, cudaMemsetAsync(A.changed, 0, sizeof(int), s->stream),
                            "adjoint"));
            EREBUS_LAUNCH(s, k_adj_assemble, nblocks(rows, 128), 128, 0, g, L.rhocp + o,
                          L.KX + o, L.KY + o, dts[q], L.seed, last ? 1.0 : 0.0,
                          last ? (const double *)nullptr : L.S, band_view(A), A.ell_prev,
                          A.changed);
            int changed = 1;
            ATRY(read_flag(s, A.changed, &changed));
            if (changed || !A.factored || !s->opt.reuse_factors) ATRY(commit_assembly(s, A));
            ErebusSolveStats ss = {};
            ATRY(band_solve_refined(s, A, s->opt.thermal_rtol, s->opt.max_refinements, &ss));
            solves += ss.iterations;
            const bool carry = first_timestep + q > 1;
            AdjNodeIn ni = {L.tk2 + o, L.DT + o, L.rhocp + o, A.x, L.S,
                            L.Wp, L.Wx, L.Wy, dts[q], carry && !last};
            AdjNodeOut no = {L.srcp, L.str, L.shr, L.skx, L.sky};
            EREBUS_LAUNCH(s, k_adj_nodes, nblocks(np), kThreads, 0, g, ni, no);
            AdjMarkerIn mi = {};
            mi.xm = s->m[M_xm];
            mi.ym = s->m[M_ym];
            mi.phim = s->m[M_phim];
            mi.rcm = s->m[M_rhocptotalm];
            mi.T = L.Tseg + (size_t)(q - s0) * n;
            mi.tm = s->tm8;
            mi.srcp = L.srcp;
            mi.str = L.str;
            mi.shr = L.shr;
            mi.skx = L.skx;
            mi.sky = L.sky;
            // calculate_radioactive_heating (E:1336-1357) at this step's time
            if (p.hr_al) {
                double e = std::exp(-times[q] * (1.0 / g.tau_al)) * (1.0 / g.tau_al);
                double Q = p.f_al * p.ratio_al * p.E_al * e;
                mi.hrs[0] = Q * p.rhosolidm[0];
                mi.hrs[1] = Q * p.rhosolidm[1];
                mi.dQ = p.f_al * p.E_al * e;
            }
            if (p.hr_fe) {
                double Q = p.f_fe * p.ratio_fe * p.E_fe *
                           std::exp(-times[q] * (1.0 / g.tau_fe)) * (1.0 / g.tau_fe);
                mi.hrf[0] = Q * p.rhofluidm[0];
            }
            mi.keep = carry;
            EREBUS_LAUNCH(s, k_adj_markers, mblocks, kThreads, 0, p, g, mi, (int)n, L.Tbar,
                          L.phibar, L.ratio_acc);
        }
    }
    EREBUS_LAUNCH(s, k_adj_sum, 1, 256, 0, L.ratio_acc, mblocks, L.out + 1);
    double host_out[2] = {0.0, 0.0};
    ATRY(check_cuda(s, cudaMemcpyAsync(host_out, L.out, 16, cudaMemcpyDeviceToHost, s->stream),
                    "adjoint"));
    if (dJ_dphim)
        ATRY(check_cuda(s, cudaMemcpyAsync(dJ_dphim, L.phibar, n * 8, cudaMemcpyDeviceToHost,
                                           s->stream), "adjoint"));
    ATRY(stream_sync(s, "adjoint"));
    double Jv = host_out[0] / (double)nbody;
    if (J) *J = Jv;
    if (dJ_dratio_al) *dJ_dratio_al = host_out[1];
    if (st) {
        st->steps = N;
        st->checkpoints = nck;
        st->adjoint_solves = solves;
        st->factorizations = A.factorizations - f0;
        st->markers = n;
        st->J = Jv;
        st->body_nodes = (double)nbody;
    }
    return EREBUS_OK;
}
