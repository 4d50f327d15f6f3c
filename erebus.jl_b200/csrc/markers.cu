// markers.cu -- marker kernels of the timestep.
//
// * cell sort: for each of the four node sets the markers are bucketed by
//   their clamped cell (fix, E:1456) with a counting sort, and each bucket is
//   ordered by marker number;
// * scatter (marker_to_*_nodes!, E:1605-1863, and the reaction / melt
//   scatters E:2681-2683, E:1883-1939): every node merges the sorted buckets
//   of its (up to) four adjacent cells by marker number and accumulates
//   property*weight in that order.  This is the reference's serial
//   summation order (markers m = 1..marknum), so the node sums are
//   bit-identical to the reference's and need no atomics;
// * per-marker gathers: compute_marker_properties! (E:700), the reaction
//   (E:2558), update_marker_{viscosity,stress,temperature,porosity}!
//   (E:774, E:4354, E:4782, E:4822), move_markers_rk4! (E:4990) and
//   backtrace_pressures_rk4! (E:5284);
// * replenish_markers! (E:5586) as per-anchor reductions plus a prefix sum.
#include <climits>
#include "laws.cuh"
#include "state.cuh"

namespace erebus {

struct MP {
    double *f[M_COUNT];
    int8_t *tm;
};
struct GPtr {
    double *f[G_COUNT];
};

static MP mptr(erebus_state *s) {
    MP r;
    for (int k = 0; k < M_COUNT; k++) r.f[k] = s->m[k];
    r.tm = s->tm8;
    return r;
}
static GPtr gptr(erebus_state *s) {
    GPtr r;
    for (int k = 0; k < G_COUNT; k++) r.f[k] = s->grid[k];
    return r;
}

// ---------------------------------------------------------------------------
// compute_marker_properties! (E:700-750)
// ---------------------------------------------------------------------------
struct Heat {
    double hrs[3], hrf[3];
};

__global__ void k_marker_props(ErebusParams p, Geo g, MP M, int n, Heat h) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    int t = M.tm[m];
    double tk = M.f[M_tkm][m], phi = M.f[M_phim][m];
    double etafluidcur;
    if (t < 3) {
        double XW = M.f[M_XWsolidm0][m];
        double XD = 1.0 - XW;
        double rhos = (p.MD + p.MH2O * XW) / (g.VDs * XD + g.VWs * XW);
        double rhof = tk > p.tmfluidphase ? p.rhoH2Of : p.rhoH2Ofi;
        M.f[M_rhototalm][m] = total(rhos, rhof, phi);
        M.f[M_rhocptotalm][m] = total(p.rhocpsolidm[t - 1], rhocpfluid(p, tk), phi);
        double es = tk > p.tmsolidphase
                        ? p.etasolidmm[t - 1]
                        : (p.per_marker_eta ? M.f[M_etasolidm_m][m] : p.etasolidm[t - 1]);
        etafluidcur = tk > p.tmfluidphase ? p.etafluidmm[t - 1] : p.etafluidm[t - 1];
        M.f[M_etatotalm][m] = jmax(jmax(p.etamin, es), etafluidcur);
        M.f[M_hrtotalm][m] = total(h.hrs[t - 1], h.hrf[t - 1], phi);
        M.f[M_ktotalm][m] = ktotal(ksolid(p, tk), kfluid(p, tk), phi);
    } else {
        etafluidcur = p.etafluidm[t - 1];
    }
    M.f[M_tkm_rhocptotalm][m] = tk * M.f[M_rhocptotalm][m];
    M.f[M_etafluidcur_inv_kphim][m] = etaf_inv_kphi(p, p.kphim0[t - 1], phi, etafluidcur);
}

// ---------------------------------------------------------------------------
// cell sort
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cell_of(const Geo &g, int grid, double x, double y) {
    GridSpec s = grid_spec(g, grid);
    int i, j;
    fix(x, y, s.x0, s.y0, g.dx, g.dy, s.jmin, s.jmax, s.imin, s.imax, i, j);
    return (j - 1) * s.rows + (i - 1);
}

struct SortPtrs {
    int *count[4], *start[4], *cursor[4], *idx[4], *tmp[4];
    int ncells[4];
};

__global__ void k_sort_count(Geo g, const double *xm, const double *ym, int n,
                             SortPtrs S) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double x = xm[m], y = ym[m];
#pragma unroll
    for (int gr = 0; gr < 4; gr++) atomicAdd(&S.count[gr][cell_of(g, gr, x, y)], 1);
}

// Bilinear weights of every marker on the four node sets (fix_weights,
// E:1388), wc[(grid * cap + m) * 4 + k].  They hold while the markers do not
// move (as the cell sort does), and the merges read them instead of
// recomputing them at every node visit.
__global__ void k_marker_weights(Geo g, const double *xm, const double *ym, int n, int64_t cap,
                                 double *wc) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double x = xm[m], y = ym[m];
#pragma unroll
    for (int gr = 0; gr < 4; gr++) {
        int i, j;
        double w[4];
        grid_weights(g, gr, x, y, i, j, w);
        double2 *d = reinterpret_cast<double2 *>(wc + ((size_t)gr * cap + m) * 4);
        d[0] = make_double2(w[0], w[1]);
        d[1] = make_double2(w[2], w[3]);
    }
}

// Exclusive scan of count -> start (start[ncells] = total), one block per grid.
__global__ void k_sort_scan(SortPtrs S) {
    int gr = blockIdx.x;
    int n = S.ncells[gr];
    const int *cnt = S.count[gr];
    int *st = S.start[gr];
    __shared__ int part[1024];
    int T = blockDim.x, t = threadIdx.x;
    int chunk = (n + T - 1) / T;
    int lo = t * chunk, hi = min(n, lo + chunk);
    int sum = 0;
    for (int k = lo; k < hi; k++) sum += cnt[k];
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < T; off <<= 1) {
        int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - sum;
    for (int k = lo; k < hi; k++) {
        st[k] = run;
        run += cnt[k];
    }
    if (t == T - 1) st[n] = part[T - 1];
}

__global__ void k_sort_place(Geo g, const double *xm, const double *ym, int n,
                             SortPtrs S) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double x = xm[m], y = ym[m];
#pragma unroll
    for (int gr = 0; gr < 4; gr++) {
        int c = cell_of(g, gr, x, y);
        int pos = S.start[gr][c] + atomicAdd(&S.cursor[gr][c], 1);
        S.tmp[gr][pos] = m;
    }
}

// One warp per cell: rank sort of the bucket by marker number.
__global__ void k_sort_segments(SortPtrs S, int gr) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= S.ncells[gr]) return;
    int b = S.start[gr][warp], e = S.start[gr][warp + 1];
    const int *src = S.tmp[gr];
    int *dst = S.idx[gr];
    for (int a = b + lane; a < e; a += 32) {
        int v = src[a], rank = 0;
        for (int c = b; c < e; c++) rank += src[c] < v;
        dst[b + rank] = v;
    }
}

// ---------------------------------------------------------------------------
// merge scatter
// ---------------------------------------------------------------------------
enum MergeMode { MM_SCATTER = 0, MM_REACTION = 1, MM_MELT = 2, MM_SUBGRID_S = 3,
                 MM_SUBGRID_T = 4, MM_VALUES = 5 };

template <int GRID, int MODE>
struct MergeFields;
// marker_to_basic_nodes! (E:1638-1645)
template <>
struct MergeFields<GB, MM_SCATTER> {
    static constexpr int N = 8;
    __device__ static void load(const MP &M, const double *, const double *, int m,
                                double v[N]) {
        v[0] = M.f[M_etatotalm][m]; v[1] = M.f[M_etavpm][m];
        v[2] = M.f[M_inv_gggtotalm][m]; v[3] = M.f[M_sxym][m];
        v[4] = M.f[M_cohestotalm][m]; v[5] = M.f[M_tenstotalm][m];
        v[6] = M.f[M_fricttotalm][m]; v[7] = 1.0;
    }
};
// marker_to_vx_nodes! / marker_to_vy_nodes! (E:1705-1710, E:1770-1775)
template <>
struct MergeFields<GVX, MM_SCATTER> {
    static constexpr int N = 6;
    __device__ static void load(const MP &M, const double *, const double *, int m,
                                double v[N]) {
        v[0] = M.f[M_rhototalm][m]; v[1] = M.f[M_rhofluidcur][m];
        v[2] = M.f[M_ktotalm][m]; v[3] = M.f[M_phim][m];
        v[4] = M.f[M_etafluidcur_inv_kphim][m]; v[5] = 1.0;
    }
};
template <>
struct MergeFields<GVY, MM_SCATTER> : MergeFields<GVX, MM_SCATTER> {};
// marker_to_p_nodes! (E:1851-1860)
template <>
struct MergeFields<GP, MM_SCATTER> {
    static constexpr int N = 10;
    __device__ static void load(const MP &M, const double *, const double *, int m,
                                double v[N]) {
        v[0] = M.f[M_inv_gggtotalm][m]; v[1] = M.f[M_sxxm][m];
        v[2] = M.f[M_rhototalm][m]; v[3] = M.f[M_rhocptotalm][m];
        v[4] = M.f[M_alphasolidcur][m]; v[5] = M.f[M_alphafluidcur][m];
        v[6] = M.f[M_hrtotalm][m]; v[7] = M.f[M_phim][m];
        v[8] = M.f[M_tkm_rhocptotalm][m]; v[9] = 1.0;
    }
};
// reaction scatter (E:2681-2683): DMPSUM, DHPSUM, WTPSUM
template <>
struct MergeFields<GP, MM_REACTION> {
    static constexpr int N = 3;
    __device__ static void load(const MP &, const double *dM, const double *dH, int m,
                                double v[N]) {
        v[0] = dM[m]; v[1] = dH[m]; v[2] = 1.0;
    }
};
// molarfraction_marker_to_p_nodes! (E:1904-1905): XWSSUM, WTPSUM
template <>
struct MergeFields<GP, MM_MELT> {
    static constexpr int N = 2;
    __device__ static void load(const MP &M, const double *, const double *, int m,
                                double v[N]) {
        v[0] = M.f[M_XWsolidm0][m]; v[1] = 1.0;
    }
};

// subgrid stress diffusion (E:4309-4320): SXXSUM/WTPSUM on P nodes and
// SXYSUM/WTSUM on basic nodes of the marker corrections (dM: xx, dH: xy)
template <>
struct MergeFields<GP, MM_SUBGRID_S> {
    static constexpr int N = 2;
    __device__ static void load(const MP &, const double *dM, const double *, int m,
                                double v[N]) {
        v[0] = dM[m]; v[1] = 1.0;
    }
};
template <>
struct MergeFields<GB, MM_SUBGRID_S> {
    static constexpr int N = 2;
    __device__ static void load(const MP &, const double *, const double *dH, int m,
                                double v[N]) {
        v[0] = dH[m]; v[1] = 1.0;
    }
};
// subgrid temperature diffusion (E:4750-4751): TKSUM, RHOCPSUM
template <>
struct MergeFields<GP, MM_SUBGRID_T> {
    static constexpr int N = 2;
    __device__ static void load(const MP &, const double *dM, const double *dH, int m,
                                double v[N]) {
        v[0] = dM[m]; v[1] = dH[m];
    }
};

// per-marker values (dM) and the weight sum, for scatter_p_values
template <>
struct MergeFields<GP, MM_VALUES> {
    static constexpr int N = 2;
    __device__ static void load(const MP &, const double *dM, const double *, int m,
                                double v[N]) {
        v[0] = dM[m]; v[1] = 1.0;
    }
};

struct MergeArgs {
    const int *start, *idx;
    const int8_t *flag;        // reaction: only flagged markers contribute
    const double *dM, *dH;
    double *sums[10];          // destination SUM arrays
    const double *wc;          // the markers' weights on this grid (k_marker_weights), or
                               // NULL: computed at each visit
};

// Bucket bounds of node (I,J): the cells (I,J), (I-1,J), (I,J-1), (I-1,J-1),
// with weights w0..w3 (E:1517).
__device__ __forceinline__ void node_buckets(const GridSpec &s, const MergeArgs &a, int I,
                                             int J, int beg[4], int end[4]) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int ci = I - (k & 1), cj = J - (k >> 1);
        if (ci >= s.imin && ci <= s.imax && cj >= s.jmin && cj <= s.jmax) {
            int c = (cj - 1) * s.rows + (ci - 1);
            beg[k] = a.start[c];
            end[k] = a.start[c + 1];
        } else {
            beg[k] = end[k] = 0;
        }
    }
}

// Weight of marker m on corner k of its cell.
template <int GRID>
__device__ __forceinline__ double merge_weight(const Geo &g, const MP &M, const MergeArgs &a,
                                               int m, int k) {
    if (a.wc) return a.wc[(size_t)m * 4 + k];
    int i, j;
    double w[4];
    grid_weights(g, GRID, M.f[M_xm][m], M.f[M_ym][m], i, j, w);
    return k == 0 ? w[0] : k == 1 ? w[1] : k == 2 ? w[2] : w[3];
}

// One thread walks the four buckets in marker order and sums every field.
template <int GRID, int MODE>
__device__ __forceinline__ void merge_serial(const Geo &g, const MP &M, const MergeArgs &a,
                                             int beg[4], const int end[4],
                                             double (&acc)[MergeFields<GRID, MODE>::N]) {
    using F = MergeFields<GRID, MODE>;
#pragma unroll
    for (int f = 0; f < F::N; f++) acc[f] = 0.0;
    while (true) {
        int best = -1, bm = INT_MAX;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (beg[k] < end[k]) {
                int mk = a.idx[beg[k]];
                if (mk < bm) { bm = mk; best = k; }
            }
        if (best < 0) break;
        beg[best]++;
        if (MODE == MM_REACTION && !a.flag[bm]) continue;
        double wk = merge_weight<GRID>(g, M, a, bm, best);
        double v[F::N];
        F::load(M, a.dM, a.dH, bm, v);
#pragma unroll
        for (int f = 0; f < F::N; f++) acc[f] = acc[f] + v[f] * wk;
    }
}

// The SUM arrays of a node and the node properties computed from them.
template <int GRID, int MODE>
__device__ __forceinline__ void merge_finish(const Geo &g, const MergeArgs &a, const GPtr &G,
                                             int node, int I, int J,
                                             const double (&acc)[MergeFields<GRID, MODE>::N],
                                             int write_props) {
    using F = MergeFields<GRID, MODE>;
#pragma unroll
    for (int f = 0; f < F::N; f++) a.sums[f][node] = acc[f];
    if (!write_props) return;
    double wt = acc[F::N - 1];
    if (MODE == MM_SCATTER && GRID == GB) {
        // compute_basic_node_properties! (E:1970-2007)
        if (wt > 0.0) {
            double eta0 = acc[0] * (1.0 / wt), eta = acc[1] * (1.0 / wt);
            G.f[G_ETA0][node] = eta0;
            G.f[G_ETA][node] = eta;
            if (eta < eta0) reinterpret_cast<uint8_t *>(G.f[G_YNY])[node] = 1;
            G.f[G_GGG][node] = (1.0 / acc[2]) * wt;
            G.f[G_SXY0][node] = acc[3] * (1.0 / wt);
            G.f[G_COH][node] = acc[4] * (1.0 / wt);
            G.f[G_TEN][node] = acc[5] * (1.0 / wt);
            G.f[G_FRI][node] = acc[6] * (1.0 / wt);
        }
    } else if (MODE == MM_SCATTER && (GRID == GVX || GRID == GVY)) {
        // compute_vx_node_properties! / compute_vy_node_properties!
        // (E:2033-2113)
        if (wt > 0.0) {
            bool X = GRID == GVX;
            G.f[X ? G_RHOX : G_RHOY][node] = acc[0] * (1.0 / wt);
            G.f[X ? G_RHOFX : G_RHOFY][node] = acc[1] * (1.0 / wt);
            G.f[X ? G_KX : G_KY][node] = acc[2] * (1.0 / wt);
            G.f[X ? G_PHIX : G_PHIY][node] = acc[3] * (1.0 / wt);
            G.f[X ? G_RX : G_RY][node] = acc[4] * (1.0 / wt);
        }
    } else if (MODE == MM_SCATTER && GRID == GP) {
        // compute_p_node_properties! (E:2148-2189)
        if (wt > 0.0) {
            G.f[G_RHO][node] = acc[2] * (1.0 / wt);
            G.f[G_RHOCP][node] = acc[3] * (1.0 / wt);
            G.f[G_ALPHA][node] = acc[4] * (1.0 / wt);
            G.f[G_ALPHAF][node] = acc[5] * (1.0 / wt);
            G.f[G_HR][node] = acc[6] * (1.0 / wt);
            double gggp = (1.0 / acc[0]) * wt;
            G.f[G_GGGP][node] = gggp;
            G.f[G_SXX0][node] = acc[1] * (1.0 / wt);
            G.f[G_tk1][node] = acc[8] * (1.0 / acc[3]);
            double phi = acc[7] * (1.0 / wt);
            G.f[G_PHI][node] = phi;
            G.f[G_BETAPHI][node] = (1.0 / gggp) * phi;
        }
    } else if (MODE == MM_SUBGRID_S && GRID == GP) {
        // DSXX at inner P nodes (E:4323-4326)
        if (I >= 2 && I <= g.Ny && J >= 2 && J <= g.Nx && wt > 0.0)
            G.f[G_DSXX][node] -= acc[0] / wt;
    } else if (MODE == MM_SUBGRID_S) {
        // DSXY at all basic nodes (E:4328-4329)
        if (wt > 0.0) G.f[G_DSXY][node] -= acc[0] / wt;
    } else if (MODE == MM_SUBGRID_T) {
        // DT -= TKSUM / RHOCPSUM (E:4754-4758)
        if (wt > 0.0) G.f[G_DT][node] -= acc[0] / wt;
    } else if (MODE == MM_REACTION) {
        // compute_thermodynamic_xfer! (E:2208-2222)
        if (wt > 0.0) {
            G.f[G_DMP][node] = acc[0] * (1.0 / wt);
            G.f[G_DHP][node] = acc[1] * (1.0 / wt);
        } else {
            G.f[G_DMP][node] = 0.0;
            G.f[G_DHP][node] = 0.0;
        }
    } else {
        // compute_molarfraction! (E:2239-2252)
        G.f[G_XWS][node] = wt > 0.0 ? acc[0] * (1.0 / wt) : 0.0;
    }
}


// One thread per node.
template <int GRID, int MODE>
__global__ void k_merge(Geo g, MP M, MergeArgs a, GPtr G, int write_props) {
    using F = MergeFields<GRID, MODE>;
    GridSpec s = grid_spec(g, GRID);
    int node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= s.rows * s.cols) return;
    int I = node % s.rows + 1, J = node / s.rows + 1;
    int beg[4], end[4];
    node_buckets(s, a, I, J, beg, end);
    double acc[F::N];
    merge_serial<GRID, MODE>(g, M, a, beg, end, acc);
    merge_finish<GRID, MODE>(g, a, G, node, I, J, acc, write_props);
}

// One warp per node.  The lanes copy the node's four sorted buckets into
// shared memory and place every marker at its rank in the merged marker
// order (its position in its bucket plus, by binary search, the number of
// smaller marker numbers in the other three).  Then, a window of positions
// at a time, the lanes load the markers' values and weights in parallel and
// store the products, and lane f adds field f's products in merged order.
// The products and the order of the additions are those of the one-thread
// walk, so the sums are the same bits.  Nodes with more than kMergeCap
// markers take the one-thread walk on lane 0.
constexpr int kMergeWarps = 4;      // nodes per block
constexpr int kMergeCap = 256;      // markers of a node held in shared memory
constexpr int kMergeWin = 64;       // merged positions per product window (two per lane)

// Rank of v in the merged order: the number of smaller keys in the four
// sorted buckets key[b[k], b[k] + n[k]) (in its own bucket, its position).
// The four searches advance together; their trip counts depend only on the
// bucket lengths, which all lanes of the warp share.
__device__ __forceinline__ int merged_rank(const int *key, const int b[4], const int n[4],
                                           int v) {
    int lo[4], len[4];
#pragma unroll
    for (int k = 0; k < 4; k++) { lo[k] = b[k]; len[k] = n[k]; }
    while (max(max(len[0], len[1]), max(len[2], len[3])) > 1) {
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (len[k] > 1) {
                int h = len[k] >> 1;
                lo[k] += key[lo[k] + h - 1] < v ? h : 0;
                len[k] -= h;
            }
    }
    int r = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) r += lo[k] - b[k] + (len[k] == 1 && key[lo[k]] < v ? 1 : 0);
    return r;
}

template <int GRID, int MODE>
__global__ void __launch_bounds__(kMergeWarps * 32)
k_merge_warp(Geo g, MP M, MergeArgs a, GPtr G, int write_props) {
    using F = MergeFields<GRID, MODE>;
    constexpr int N = F::N;
    __shared__ int s_key[kMergeWarps][kMergeCap];
    __shared__ unsigned short s_ord[kMergeWarps][kMergeCap];
    __shared__ double s_prod[kMergeWarps][N][kMergeWin + 1];
    GridSpec s = grid_spec(g, GRID);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int node = blockIdx.x * kMergeWarps + w;
    if (node >= s.rows * s.cols) return;        // uniform over the warp
    const int I = node % s.rows + 1, J = node / s.rows + 1;
    int beg[4], end[4];
    node_buckets(s, a, I, J, beg, end);
    const int o1 = end[0] - beg[0], o2 = o1 + end[1] - beg[1], o3 = o2 + end[2] - beg[2];
    int L = o3 + end[3] - beg[3];
    double acc[N];
    if (L > kMergeCap) {
        if (lane == 0) {
            merge_serial<GRID, MODE>(g, M, a, beg, end, acc);
            merge_finish<GRID, MODE>(g, a, G, node, I, J, acc, write_props);
        }
        return;
    }
    int *key = s_key[w];
    unsigned short *ord = s_ord[w];
    for (int e = lane; e < L; e += 32) {
        int k = e < o1 ? 0 : e < o2 ? 1 : e < o3 ? 2 : 3;
        int o = k == 0 ? 0 : k == 1 ? o1 : k == 2 ? o2 : o3;
        key[e] = a.idx[beg[k] + e - o];
    }
    __syncwarp();
    {
        const int bb[4] = {0, o1, o2, o3}, nn[4] = {o1, o2 - o1, o3 - o2, L - o3};
        for (int e = lane; e < L; e += 32) ord[merged_rank(key, bb, nn, key[e])] = e;
    }
    __syncwarp();
    if (MODE == MM_REACTION) {
        // keep the flagged markers, in merged order
        int kept = 0;
        for (int r0 = 0; r0 < L; r0 += 32) {
            int r = r0 + lane;
            unsigned short e = 0;
            bool keep = false;
            if (r < L) {
                e = ord[r];
                keep = a.flag[key[e]] != 0;
            }
            unsigned b = __ballot_sync(0xffffffffu, keep);
            __syncwarp();
            if (keep) ord[kept + __popc(b & ((1u << lane) - 1u))] = e;
            kept += __popc(b);
            __syncwarp();
        }
        L = kept;
    }
    double sum = 0.0;
    double (*prod)[kMergeWin + 1] = s_prod[w];
    for (int r0 = 0; r0 < L; r0 += kMergeWin) {
        const int cnt = min(kMergeWin, L - r0);
        // positions lane and lane + 32 of the window, loads issued together
        double wk[2], v[2][N];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int t = lane + 32 * u;
            if (t < cnt) {
                int e = ord[r0 + t];
                int k = e < o1 ? 0 : e < o2 ? 1 : e < o3 ? 2 : 3;
                int m = key[e];
                wk[u] = merge_weight<GRID>(g, M, a, m, k);
                F::load(M, a.dM, a.dH, m, v[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < 2; u++)
            if (lane + 32 * u < cnt) {
#pragma unroll
                for (int f = 0; f < N; f++) prod[f][lane + 32 * u] = v[u][f] * wk[u];
            }
        __syncwarp();
        if (lane < N) {
            const double *q = prod[lane];
            int t = 0;
            for (; t + 8 <= cnt; t += 8) {
                double x[8];
#pragma unroll
                for (int u = 0; u < 8; u++) x[u] = q[t + u];
#pragma unroll
                for (int u = 0; u < 8; u++) sum = sum + x[u];
            }
            for (; t < cnt; t++) sum = sum + q[t];
        }
        __syncwarp();
    }
#pragma unroll
    for (int f = 0; f < N; f++) acc[f] = __shfl_sync(0xffffffffu, sum, f);
    if (lane == 0) merge_finish<GRID, MODE>(g, a, G, node, I, J, acc, write_props);
}

// apply_insulating_boundary_conditions! (E:2432-2449) on tk1, two passes
__global__ void k_insulate_rows(Geo g, double *t) {
    int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
    int R = g.Ny1, C = g.Nx1;
    if (j > C - 1) return;
    AT(t, R, 1, j) = AT(t, R, 2, j);
    AT(t, R, R, j) = AT(t, R, R - 1, j);
}
__global__ void k_insulate_cols(Geo g, double *t) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int R = g.Ny1, C = g.Nx1;
    if (i > R) return;
    AT(t, R, i, 1) = AT(t, R, i, 2);
    AT(t, R, i, C) = AT(t, R, i, C - 1);
}

static SortPtrs sort_ptrs(erebus_state *s) {
    SortPtrs S;
    for (int gr = 0; gr < 4; gr++) {
        S.count[gr] = s->sort[gr].count;
        S.start[gr] = s->sort[gr].start;
        S.cursor[gr] = s->sort[gr].cursor;
        S.idx[gr] = s->sort[gr].idx;
        S.tmp[gr] = s->sort[gr].tmp;
        S.ncells[gr] = s->sort[gr].ncells;
    }
    return S;
}

int build_cell_sort(erebus_state *s) {
    int n = (int)s->marknum;
    SortPtrs S = sort_ptrs(s);
    for (int gr = 0; gr < 4; gr++) {
        cudaMemsetAsync(S.count[gr], 0, sizeof(int) * S.ncells[gr], s->stream);
        cudaMemsetAsync(S.cursor[gr], 0, sizeof(int) * S.ncells[gr], s->stream);
    }
    if (n > 0) {
        EREBUS_LAUNCH(s, k_sort_count, nblocks(n), kThreads, 0, s->g, s->m[M_xm],
                      s->m[M_ym], n, S);
        EREBUS_LAUNCH(s, k_marker_weights, nblocks(n), kThreads, 0, s->g, s->m[M_xm],
                      s->m[M_ym], n, s->capacity, s->wcache);
    }
    EREBUS_LAUNCH(s, k_sort_scan, 4, 1024, 0, S);
    if (n > 0) {
        EREBUS_LAUNCH(s, k_sort_place, nblocks(n), kThreads, 0, s->g, s->m[M_xm],
                      s->m[M_ym], n, S);
    }
    for (int gr = 0; gr < 4; gr++)
        EREBUS_LAUNCH(s, k_sort_segments, nblocks((int64_t)S.ncells[gr] * 32), kThreads,
                      0, S, gr);
    s->sorted_valid = true;
    return check_cuda(s, cudaGetLastError(), "cell sort");
}

template <int GRID, int MODE>
static void launch_merge(erebus_state *s, MergeArgs a, int write_props) {
    GridSpec sp = grid_spec(s->g, GRID);
    EREBUS_LAUNCH(s, (k_merge_warp<GRID, MODE>),
                  nblocks((int64_t)sp.rows * sp.cols, kMergeWarps), kMergeWarps * 32, 0, s->g,
                  mptr(s), a, gptr(s), write_props);
}

static MergeArgs merge_args(erebus_state *s, int gr, std::initializer_list<int> sums) {
    MergeArgs a = {};
    a.start = s->sort[gr].start;
    a.idx = s->sort[gr].idx;
    a.wc = s->wcache + (size_t)gr * s->capacity * 4;
    a.flag = s->r_flag;
    a.dM = s->r_dM;
    a.dH = s->r_dH;
    int k = 0;
    for (int f : sums) a.sums[k++] = s->sums[f];
    return a;
}

int scatter_p_values(erebus_state *s, const double *vals, double *sum, double *wt) {
    if (!s->sorted_valid) {
        int rc = build_cell_sort(s);
        if (rc) return rc;
    }
    MergeArgs a = {};
    a.start = s->sort[GP].start;
    a.idx = s->sort[GP].idx;
    a.wc = s->wcache + (size_t)GP * s->capacity * 4;
    a.dM = vals;
    a.sums[0] = sum;
    a.sums[1] = wt;
    launch_merge<GP, MM_VALUES>(s, a, 0);
    return check_cuda(s, cudaGetLastError(), "scatter_p_values");
}

// E:6376-6604
int markers_to_nodes(erebus_state *s, double timesum) {
    const ErebusParams &p = s->p;
    Heat h = {};
    // calculate_radioactive_heating (E:1336-1357), evaluated on the host
    if (p.hr_al) {
        double Q = p.f_al * p.ratio_al * p.E_al * exp(-timesum * (1.0 / s->g.tau_al)) *
                   (1.0 / s->g.tau_al);
        h.hrs[0] = Q * p.rhosolidm[0];
        h.hrs[1] = Q * p.rhosolidm[1];
    }
    if (p.hr_fe) {
        double Q = p.f_fe * p.ratio_fe * p.E_fe * exp(-timesum * (1.0 / s->g.tau_fe)) *
                   (1.0 / s->g.tau_fe);
        h.hrf[0] = Q * p.rhofluidm[0];
    }
    int n = (int)s->marknum;
    if (n > 0)
        EREBUS_LAUNCH(s, k_marker_props, nblocks(n), kThreads, 0, p, s->g, mptr(s), n, h);
    int rc = build_cell_sort(s);
    if (rc) return rc;
    timer_begin(s, PH_SCATTER_MERGE);
    launch_merge<GB, MM_SCATTER>(
        s, merge_args(s, GB, {S_ETA0SUM, S_ETASUM, S_GGGSUM, S_SXYSUM, S_COHSUM,
                              S_TENSUM, S_FRISUM, S_WTSUM}), 1);
    launch_merge<GVX, MM_SCATTER>(
        s, merge_args(s, GVX, {S_RHOXSUM, S_RHOFXSUM, S_KXSUM, S_PHIXSUM, S_RXSUM,
                               S_WTXSUM}), 1);
    launch_merge<GVY, MM_SCATTER>(
        s, merge_args(s, GVY, {S_RHOYSUM, S_RHOFYSUM, S_KYSUM, S_PHIYSUM, S_RYSUM,
                               S_WTYSUM}), 1);
    launch_merge<GP, MM_SCATTER>(
        s, merge_args(s, GP, {S_GGGPSUM, S_SXXSUM, S_RHOSUM, S_RHOCPSUM, S_ALPHASUM,
                              S_ALPHAFSUM, S_HRSUM, S_PHISUM, S_TKSUM, S_WTPSUM}), 1);
    timer_end(s, PH_SCATTER_MERGE);
    EREBUS_LAUNCH(s, k_insulate_rows, nblocks(s->g.Nx1), kThreads, 0, s->g,
                  s->grid[G_tk1]);
    EREBUS_LAUNCH(s, k_insulate_cols, nblocks(s->g.Ny1), kThreads, 0, s->g,
                  s->grid[G_tk1]);
    return check_cuda(s, cudaGetLastError(), "markers_to_nodes");
}

// ---------------------------------------------------------------------------
// perform_thermochemical_reaction! (E:2558-2694)
// ---------------------------------------------------------------------------
__global__ void k_reaction(ErebusParams p, Geo g, MP M, GPtr G, int n, double dt,
                           int timestep, int titer, double *dMo, double *dHo,
                           int8_t *flag) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    flag[m] = 0;
    if (M.tm[m] >= 3) return;
    int Ny1 = g.Ny1, i, j;
    double w[4];
    grid_weights(g, GP, M.f[M_xm][m], M.f[M_ym][m], i, j, w);
    double tknm = gather4(G.f[G_tk2], Ny1, i, j, w);
    double pfnm = jmax(0.0, gather4(G.f[G_pf], Ny1, i, j, w));
    if (titer > 2) pfnm = pfnm * (1.0 - p.pfcoeff) + M.f[M_pfm0][m] * p.pfcoeff;
    M.f[M_pfm0][m] = pfnm;
    double XW0 = M.f[M_XWsolidm0][m], phi = M.f[M_phim][m];
    double XD0 = 1.0 - XW0;
    double VH2O = tknm > p.tmfluidphase ? g.VH2Of : g.VH2Ofi;
    double Xf0 = phi * (XW0 * g.VWs + XD0 * g.VDs) /
                 ((1.0 - phi) * VH2O + phi * (XW0 * g.VWs + XD0 * g.VDs));
    double Xs0 = 1.0 - Xf0;
    double XH2Ot = (XW0 * Xs0 + Xf0) / (1.0 + XW0 * Xs0);
    double XDt = 1.0 - XH2Ot;
    double rhos0 = (p.MD + p.MH2O * XW0) / (g.VDs * XD0 + g.VWs * XW0);
    double rhof0 = tknm > p.tmfluidphase ? p.rhoH2Of : p.rhoH2Ofi;
    double dtr = dtreaction_of(p, tknm, phi);
    double Ht0 = -Xs0 * XW0 * p.dHWD / (p.MD + p.MH2O);
    double dGWD0;
    if (dt < dtr)
        dGWD0 = (p.dHWD - tknm * p.dSWD + pfnm * g.dVWD + p.RG * tknm * log(XD0 / XW0)) *
                (1.0 - dt / dtr);
    else
        dGWD0 = 0.0;
    double KWD = exp(-(p.dHWD - tknm * p.dSWD + g.dVWD * pfnm - dGWD0) / (p.RG * tknm));
    double XW1 = 1.0 / (KWD + 1.0);
    double XD1 = 1.0 - XW1;
    double Xs1 = XDt / (1.0 - XDt * XW1);
    double Xf1 = 1.0 - Xs1;
    if (0.0 < Xf1 && Xf1 < 1.0) {
        double phi1 = Xf1 * VH2O / (Xf1 * VH2O + Xs1 * (XW1 * g.VWs + XD1 * g.VDs));
        double rhos1 = (p.MD + p.MH2O * XW1) / (g.VDs * XD1 + g.VWs * XW1);
        double rhof1 = tknm > p.tmfluidphase ? p.rhoH2Of : p.rhoH2Ofi;
        double Ht1 = -Xs1 * XW1 * p.dHWD / (p.MD + p.MH2O);
        double dHt = Ht1 - Ht0;
        double RV = (rhos1 * (1.0 - phi1) + rhof1 * phi1) / (rhos0 * (1.0 - phi) + rhof0 * phi);
        double Gmass = (rhos0 * RV * (1.0 - phi) - rhos1 * (1.0 - phi1)) / dt;
        M.f[M_XWsolidm][m] = XW1;
        M.f[M_phinewm][m] = phi1;
        if (timestep == 1) {
            M.f[M_XWsolidm0][m] = XW1;
            M.f[M_phim][m] = phi1;
        }
        dMo[m] = (1.0 - RV) / dt;
        dHo[m] = Gmass * dHt;
        flag[m] = 1;
    }
}

int thermochemical_reaction(erebus_state *s, double dt, int timestep, int titer) {
    int n = (int)s->marknum;
    if (!s->sorted_valid) {
        int rc = build_cell_sort(s);
        if (rc) return rc;
    }
    if (n > 0)
        EREBUS_LAUNCH(s, k_reaction, nblocks(n), kThreads, 0, s->p, s->g, mptr(s), gptr(s),
                      n, dt, timestep, titer, s->r_dM, s->r_dH, s->r_flag);
    launch_merge<GP, MM_REACTION>(s, merge_args(s, GP, {S_DMPSUM, S_DHPSUM, S_WTPSUM}), 1);
    return check_cuda(s, cudaGetLastError(), "thermochemical_reaction");
}

// ---------------------------------------------------------------------------
// node -> marker (E:6945-7019)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double etatotal_rocks(const ErebusParams &p, double tk, int t,
                                                 double eta_marker) {
    double es = tk > p.tmsolidphase ? p.etasolidmm[t - 1]
                                    : (p.per_marker_eta ? eta_marker : p.etasolidm[t - 1]);
    double ef = tk > p.tmfluidphase ? p.etafluidmm[t - 1] : p.etafluidm[t - 1];
    return jmax(jmax(p.etamin, es), ef);
}

// apply_subgrid_stress_diffusion! (E:4253-4333), marker part: the
// marker-node differences of sxx (P grid) and sxy (basic grid) relaxed over
// dt with the reference's viscosity factor 1 (E:4276); markers corrected,
// corrections to dM (xx) and dH (xy) for the marker-order node sums.
__global__ void k_subgrid_stress(ErebusParams p, Geo g, MP M, GPtr G, int n, double dt,
                                 double *dM, double *dH) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const double etam = 1.0;
    double x = M.f[M_xm][m], y = M.f[M_ym][m], w[4];
    int i, j;
    double relax = exp(-p.dsubgrids * dt / (etam * M.f[M_inv_gggtotalm][m])) - 1.0;
    grid_weights(g, GP, x, y, i, j, w);
    double d = M.f[M_sxxm][m] - gather4(G.f[G_SXX0], g.Ny1, i, j, w);
    d *= relax;
    M.f[M_sxxm][m] += d;
    dM[m] = d;
    grid_weights(g, GB, x, y, i, j, w);
    d = M.f[M_sxym][m] - gather4(G.f[G_SXY0], g.Ny, i, j, w);
    d *= relax;
    M.f[M_sxym][m] += d;
    dH[m] = d;
}

// apply_subgrid_temperature_diffusion! (E:4710-4761), marker part: the
// marker-node temperature difference relaxed over dt with the marker's
// conductivity and heat capacity (the algorithm the reference test verifies,
// T:5480-5545; the reference body itself fails for rock markers), marker
// corrected; dM = correction * rhocp, dH = rhocp for the node sums.
__global__ void k_subgrid_temp(ErebusParams p, Geo g, MP M, GPtr G, int n, double dt,
                               double *dM, double *dH) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double x = M.f[M_xm][m], y = M.f[M_ym][m], w[4];
    int i, j;
    grid_weights(g, GP, x, y, i, j, w);
    double tk = M.f[M_tkm][m];
    double d = tk - gather4(G.f[G_tk1], g.Ny1, i, j, w);
    int t = M.tm[m];
    double rcp, k;
    if (t < 3) {
        double ph = M.f[M_phim][m];
        rcp = total(p.rhocpsolidm[t - 1], rhocpfluid(p, tk), ph);
        k = ktotal(ksolid(p, tk), kfluid(p, tk), ph);
    } else {
        rcp = p.rhocpsolidm[t - 1];
        k = p.ksolidm[t - 1];
    }
    const double geom = 2.0 * (1.0 / (g.dx * g.dx) + 1.0 / (g.dy * g.dy));
    d *= exp(-p.dsubgridt * k * dt / rcp * geom) - 1.0;
    M.f[M_tkm][m] = tk + d;
    dM[m] = d * rcp;
    dH[m] = rcp;
}

// update_marker_viscosity! (E:774-804) and update_marker_stress! (E:4354-4388)
__global__ void k_marker_visc_stress(ErebusParams p, Geo g, MP M, GPtr G, int n) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    int Ny = g.Ny, Ny1 = g.Ny1, i, j;
    double w[4], x = M.f[M_xm][m], y = M.f[M_ym][m];
    grid_weights(g, GB, x, y, i, j, w);
    int t = M.tm[m];
    double etot = M.f[M_etatotalm][m];
    if (t < 3) {
        etot = etatotal_rocks(p, M.f[M_tkm][m], t,
                              p.per_marker_eta ? M.f[M_etasolidm_m][m] : 0.0);
        M.f[M_etatotalm][m] = etot;
    }
    const uint8_t *YNY = reinterpret_cast<const uint8_t *>(G.f[G_YNY]);
    if (AT(YNY, Ny, i, j) || AT(YNY, Ny, i + 1, j) || AT(YNY, Ny, i, j + 1) ||
        AT(YNY, Ny, i + 1, j + 1)) {
        double v = 1.0 / gather4(G.f[G_YNY_inv_ETA], Ny, i, j, w);
        M.f[M_etavpm][m] = v > etot ? etot : v;
    } else {
        M.f[M_etavpm][m] = etot;
    }
    int ip, jp, ib, jb;
    double wp[4], wb[4];
    fix_weights(x, y, -g.dx / 2, -g.dy / 2, g.dx, g.dy, 2, g.Nx - 1, 2, g.Ny - 1, ip, jp, wp);
    fix_weights(x, y, 0.0, 0.0, g.dx, g.dy, 1, g.Nx - 1, 1, g.Ny - 1, ib, jb, wb);
    M.f[M_sxxm][m] += gather4(G.f[G_DSXX], Ny1, ip, jp, wp);
    M.f[M_sxym][m] += gather4(G.f[G_DSXY], Ny, ib, jb, wb);
}

// update_marker_temperature! (E:4782-4801), the copies E:7011-7012,
// update_marker_porosity! (E:4822-4856) and the copy E:7014
__global__ void k_marker_temp_poro(ErebusParams p, Geo g, MP M, GPtr G, int n,
                                   double dt, int timestep) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    int Ny1 = g.Ny1, i, j;
    double w[4];
    grid_weights(g, GP, M.f[M_xm][m], M.f[M_ym][m], i, j, w);
    if (timestep == 1) M.f[M_tkm][m] = gather4(G.f[G_tk2], Ny1, i, j, w);
    else M.f[M_tkm][m] += gather4(G.f[G_DT], Ny1, i, j, w);
    M.f[M_XWsolidm0][m] = M.f[M_XWsolidm][m];
    double ph = M.f[M_phinewm][m];
    if (M.tm[m] < 3) {
        double aphim = gather4(G.f[G_APHI], Ny1, i, j, w);
        ph = jmax(p.phimin, jmin(p.phimax, ph / ((1.0 - ph) * exp(aphim * dt) + ph)));
    }
    M.f[M_phim][m] = ph;
    M.f[M_phinewm][m] = ph;
}

int nodes_to_markers(erebus_state *s, double dt, int timestep) {
    int n = (int)s->marknum;
    size_t np = (size_t)s->g.Nx1 * s->g.Ny1;
    cudaMemcpyAsync(s->grid[G_DT0], s->grid[G_DT], np * 8, cudaMemcpyDeviceToDevice,
                    s->stream);
    if (!s->sorted_valid) {
        int rc = build_cell_sort(s);
        if (rc) return rc;
    }
    // The subgrid stress diffusion touches neither the viscosities nor what
    // they read, so it runs before the combined viscosity + stress kernel,
    // i.e. between update_marker_viscosity! and update_marker_stress! as in
    // E:6950-6981; likewise the subgrid temperature diffusion before
    // update_marker_temperature! (E:6986-7004).
    if (s->p.dsubgrids != 0.0) {
        EREBUS_LAUNCH(s, k_subgrid_stress, nblocks(n), kThreads, 0, s->p, s->g, mptr(s),
                      gptr(s), n, dt, s->r_dM, s->r_dH);
        launch_merge<GP, MM_SUBGRID_S>(s, merge_args(s, GP, {S_SXXSUM, S_WTPSUM}), 1);
        launch_merge<GB, MM_SUBGRID_S>(s, merge_args(s, GB, {S_SXYSUM, S_WTSUM}), 1);
    }
    EREBUS_LAUNCH(s, k_marker_visc_stress, nblocks(n), kThreads, 0, s->p, s->g, mptr(s),
                  gptr(s), n);
    if (s->p.dsubgridt != 0.0) {
        EREBUS_LAUNCH(s, k_subgrid_temp, nblocks(n), kThreads, 0, s->p, s->g, mptr(s),
                      gptr(s), n, dt, s->r_dM, s->r_dH);
        launch_merge<GP, MM_SUBGRID_T>(s, merge_args(s, GP, {S_TKSUM, S_RHOCPSUM}), 1);
    }
    EREBUS_LAUNCH(s, k_marker_temp_poro, nblocks(n), kThreads, 0, s->p, s->g, mptr(s),
                  gptr(s), n, dt, timestep);
    // update_p_nodes_melt_composition! (E:1929-1939)
    launch_merge<GP, MM_MELT>(s, merge_args(s, GP, {S_XWSSUM, S_WTPSUM}), 1);
    return check_cuda(s, cudaGetLastError(), "nodes_to_markers");
}

// ---------------------------------------------------------------------------
// move_markers_rk4! (E:4990-5257) and backtrace_pressures_rk4! (E:5284-5496)
// ---------------------------------------------------------------------------
// vx at (x,y) with the second-order correction (E:5057-5091); with `quirk`
// the left-half correction reads vq[i,j] in place of v[i,j] (E:5173).
// form 0: E:5091 weighting; form 1: E:5332 weighting.
__device__ __forceinline__ double vx_at(const Geo &g, const double *v, const double *vq,
                                        bool quirk, double x, double y, int form) {
    int i, j, Ny1 = g.Ny1;
    double dxmj, dymi, dx = g.dx, dy = g.dy;
    fix_distances(x, y, 0.0, -g.dy / 2, g.dx, g.dy, 1, g.Nx - 1, 1, g.Ny, i, j, dxmj, dymi);
    double v13 = AT(v, Ny1, i, j) * (1.0 - dxmj / dx) + AT(v, Ny1, i, j + 1) * dxmj / dx;
    double v24 = AT(v, Ny1, i + 1, j) * (1.0 - dxmj / dx) + AT(v, Ny1, i + 1, j + 1) * dxmj / dx;
    if (dxmj / dx >= 0.5) {
        if (j < g.Nx - 1) {
            double q = dxmj / dx - 0.5;
            v13 += 0.5 * (q * q) * (AT(v, Ny1, i, j) - 2.0 * AT(v, Ny1, i, j + 1) + AT(v, Ny1, i, j + 2));
            v24 += 0.5 * (q * q) * (AT(v, Ny1, i + 1, j) - 2.0 * AT(v, Ny1, i + 1, j + 1) + AT(v, Ny1, i + 1, j + 2));
        }
    } else {
        if (j > 1) {
            double q = dxmj / dx - 0.5;
            const double *c = quirk ? vq : v;
            v13 += 0.5 * (q * q) * (AT(v, Ny1, i, j - 1) - 2.0 * AT(c, Ny1, i, j) + AT(v, Ny1, i, j + 1));
            v24 += 0.5 * (q * q) * (AT(v, Ny1, i + 1, j - 1) - 2.0 * AT(v, Ny1, i + 1, j) + AT(v, Ny1, i + 1, j + 1));
        }
    }
    if (form == 0) return v13 * (1.0 - dymi / dy) + v24 * dymi / dy;
    return (1.0 - dymi / dy) * v13 + (dymi / dy) * v24;
}

// vy at (x,y) with the correction of E:5093-5127.
__device__ __forceinline__ double vy_at(const Geo &g, const double *v, double x, double y,
                                        int form) {
    int i, j, Ny1 = g.Ny1;
    double dxmj, dymi, dx = g.dx, dy = g.dy;
    fix_distances(x, y, -g.dx / 2, 0.0, g.dx, g.dy, 1, g.Nx, 1, g.Ny - 1, i, j, dxmj, dymi);
    double v12 = AT(v, Ny1, i, j) * (1.0 - dymi / dy) + AT(v, Ny1, i + 1, j) * dymi / dy;
    double v34 = AT(v, Ny1, i, j + 1) * (1.0 - dymi / dy) + AT(v, Ny1, i + 1, j + 1) * dymi / dy;
    if (dymi / dy >= 0.5) {
        if (i < g.Ny - 1) {
            double q = dymi / dy - 0.5;
            v12 += 0.5 * (q * q) * (AT(v, Ny1, i, j) - 2.0 * AT(v, Ny1, i + 1, j) + AT(v, Ny1, i + 2, j));
            v34 += 0.5 * (q * q) * (AT(v, Ny1, i, j + 1) - 2.0 * AT(v, Ny1, i + 1, j + 1) + AT(v, Ny1, i + 2, j + 1));
        }
    } else {
        if (i > 1) {
            double q = dymi / dy - 0.5;
            v12 += 0.5 * (q * q) * (AT(v, Ny1, i - 1, j) - 2.0 * AT(v, Ny1, i, j) + AT(v, Ny1, i + 1, j));
            v34 += 0.5 * (q * q) * (AT(v, Ny1, i - 1, j + 1) - 2.0 * AT(v, Ny1, i, j + 1) + AT(v, Ny1, i + 1, j + 1));
        }
    }
    if (form == 0) return v12 * (1.0 - dxmj / dx) + v34 * dxmj / dx;
    return (1.0 - dxmj / dx) * v12 + (dxmj / dx) * v34;
}

// The velocity interpolations of the RK4 advection with the cell fractions
// taken as products with 1/dx and 1/dy and the blends as fused multiply-adds
// (the k_backtrace versions above keep the reference's divisions and
// roundings).  The results differ from those by rounding only (~1e-16
// relative); the advection is bound by its FP64 instructions, not by HBM.
struct RkGeo {
    double dx, dy, idx, idy;
    int Nx, Ny, Ny1;
};
__device__ __forceinline__ void rk_cell(double x, double y, double x0, double y0,
                                        const RkGeo &r, int jmax_, int imax_, int &i, int &j,
                                        double &fx, double &fy) {
    int64_t jj = jtrunc((x - x0) * r.idx) + 1, ii = jtrunc((y - y0) * r.idy) + 1;
    jj = jj < 1 ? 1 : jj > jmax_ ? jmax_ : jj;
    ii = ii < 1 ? 1 : ii > imax_ ? imax_ : ii;
    j = (int)jj;
    i = (int)ii;
    fx = (x - ax(x0, r.dx, j)) * r.idx;
    fy = (y - ax(y0, r.dy, i)) * r.idy;
}
__device__ __forceinline__ double rk_vx(const RkGeo &r, const double *__restrict__ v,
                                        const double *__restrict__ vq, bool quirk, double x,
                                        double y) {
    int i, j;
    double fx, fy;
    rk_cell(x, y, 0.0, -r.dy / 2, r, r.Nx - 1, r.Ny, i, j, fx, fy);
    const int Ny1 = r.Ny1;
    const double a0 = AT(v, Ny1, i, j), a1 = AT(v, Ny1, i, j + 1);
    const double b0 = AT(v, Ny1, i + 1, j), b1 = AT(v, Ny1, i + 1, j + 1);
    double v13 = fma(fx, a1 - a0, a0), v24 = fma(fx, b1 - b0, b0);
    const double q = fx - 0.5, h = 0.5 * (q * q);
    if (fx >= 0.5) {
        if (j < r.Nx - 1) {
            v13 = fma(h, a0 - 2.0 * a1 + AT(v, Ny1, i, j + 2), v13);
            v24 = fma(h, b0 - 2.0 * b1 + AT(v, Ny1, i + 1, j + 2), v24);
        }
    } else if (j > 1) {
        const double c0 = quirk ? AT(vq, Ny1, i, j) : a0;
        v13 = fma(h, AT(v, Ny1, i, j - 1) - 2.0 * c0 + a1, v13);
        v24 = fma(h, AT(v, Ny1, i + 1, j - 1) - 2.0 * b0 + b1, v24);
    }
    return fma(fy, v24 - v13, v13);
}
__device__ __forceinline__ double rk_vy(const RkGeo &r, const double *__restrict__ v, double x,
                                        double y) {
    int i, j;
    double fx, fy;
    rk_cell(x, y, -r.dx / 2, 0.0, r, r.Nx, r.Ny - 1, i, j, fx, fy);
    const int Ny1 = r.Ny1;
    const double a0 = AT(v, Ny1, i, j), a1 = AT(v, Ny1, i + 1, j);
    const double b0 = AT(v, Ny1, i, j + 1), b1 = AT(v, Ny1, i + 1, j + 1);
    double v12 = fma(fy, a1 - a0, a0), v34 = fma(fy, b1 - b0, b0);
    const double q = fy - 0.5, h = 0.5 * (q * q);
    if (fy >= 0.5) {
        if (i < r.Ny - 1) {
            v12 = fma(h, a0 - 2.0 * a1 + AT(v, Ny1, i + 2, j), v12);
            v34 = fma(h, b0 - 2.0 * b1 + AT(v, Ny1, i + 2, j + 1), v34);
        }
    } else if (i > 1) {
        v12 = fma(h, AT(v, Ny1, i - 1, j) - 2.0 * a0 + a1, v12);
        v34 = fma(h, AT(v, Ny1, i - 1, j + 1) - 2.0 * b0 + b1, v34);
    }
    return fma(fx, v34 - v12, v12);
}

// 7 blocks of 128 threads per SM (72 registers a thread, against 84 and 6
// blocks unbounded): the kernel is bound by the latency of its FP64
// divisions and gathers, so it wants warps in flight more than registers.
__global__ void __launch_bounds__(128, 7)
k_rk4(ErebusParams p, Geo g, MP M, GPtr G, int n, double dt) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const double B[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    const double Cc[3] = {0.5, 0.5, 1.0};
    int Ny = g.Ny, Ny1 = g.Ny1, i, j;
    double w[4];
    double xmm = M.f[M_xm][m], ymm = M.f[M_ym][m];
    grid_weights(g, GP, xmm, ymm, i, j, w);
    double tksm0 = gather4(G.f[G_tk2], Ny1, i, j, w);
    grid_weights(g, GB, xmm, ymm, i, j, w);
    double om = gather4(G.f[G_wyx], Ny, i, j, w);
    double th = dt * om;
    double c, sn, s2, c2;
    sincos(th, &sn, &c);
    sincos(2.0 * th, &s2, &c2);
    double sxx = M.f[M_sxxm][m], sxy = M.f[M_sxym][m];
    M.f[M_sxxm][m] = sxx * (c * c) - sxx * (sn * sn) - sxy * s2;
    M.f[M_sxym][m] = sxx * s2 + sxy * c2;
    const double *vx = G.f[G_vx], *vy = G.f[G_vy], *vxf = G.f[G_vxf], *vyf = G.f[G_vyf];
    const RkGeo r = {g.dx, g.dy, 1.0 / g.dx, 1.0 / g.dy, g.Nx, g.Ny, g.Ny1};
    double vxr[4], vyr[4], xr = xmm, yr = ymm;
#pragma unroll
    for (int rk = 0; rk < 4; rk++) {
        vxr[rk] = rk_vx(r, vx, vx, false, xr, yr);
        vyr[rk] = rk_vy(r, vy, xr, yr);
        if (rk < 3) {
            xr = xmm + dt * Cc[rk] * vxr[rk];
            yr = ymm + dt * Cc[rk] * vyr[rk];
        }
    }
    double xn = xmm + dt * (B[0] * vxr[0] + B[1] * vxr[1] + B[2] * vxr[2] + B[3] * vxr[3]);
    double yn = ymm + dt * (B[0] * vyr[0] + B[1] * vyr[1] + B[2] * vyr[2] + B[3] * vyr[3]);
    M.f[M_xm][m] = xn;
    M.f[M_ym][m] = yn;
    xmm = xr = xn;
    ymm = yr = yn;
#pragma unroll
    for (int rk = 0; rk < 4; rk++) {
        vxr[rk] = rk_vx(r, vxf, vx, true, xr, yr);
        vyr[rk] = rk_vy(r, vyf, xr, yr);
        if (rk < 3) {
            xr = xmm - dt * Cc[rk] * vxr[rk];
            yr = ymm - dt * Cc[rk] * vyr[rk];
        }
    }
    xr = xmm - dt * (B[0] * vxr[0] + B[1] * vxr[1] + B[2] * vxr[2] + B[3] * vxr[3]);
    yr = ymm - dt * (B[0] * vyr[0] + B[1] * vyr[1] + B[2] * vyr[2] + B[3] * vyr[3]);
    grid_weights(g, GP, xr, yr, i, j, w);
    double tkfm0 = gather4(G.f[G_tk2], Ny1, i, j, w);
    double d = tkfm0 - tksm0;
    int t = M.tm[m];
    double ph = M.f[M_phim][m], tk = M.f[M_tkm][m];
    double rcs = p.rhocpsolidm[t - 1], rcf = rhocpfluid(p, tk);
    M.f[M_tkm][m] = ((1.0 - ph) * tk * rcs + ph * (tk + d) * rcf) / ((1.0 - ph) * rcs + ph * rcf);
}

// backtrace_pressures_rk4! interior nodes (2..Ny, 2..Nx), both passes
__global__ void k_backtrace(Geo g, GPtr G, double dt) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int ni = g.Ny - 1, nj = g.Nx - 1;
    if (t >= ni * nj) return;
    int ii = t % ni + 2, jj = t / ni + 2, Ny1 = g.Ny1;
    double xA = ax(-g.dx / 2, g.dx, jj), yA = ax(-g.dy / 2, g.dy, ii);
    for (int pass = 0; pass < 2; pass++) {
        const double *vx = pass == 0 ? G.f[G_vx] : G.f[G_vxf];
        const double *vy = pass == 0 ? G.f[G_vy] : G.f[G_vyf];
        double xc = xA, yc = yA, vxm[4], vym[4];
#pragma unroll
        for (int rk = 0; rk < 4; rk++) {
            vxm[rk] = vx_at(g, vx, vx, false, xc, yc, 1);
            vym[rk] = vy_at(g, vy, xc, yc, 1);
            if (rk == 0 || rk == 1) {
                xc = xA - 0.5 * dt * vxm[rk];
                yc = yA - 0.5 * dt * vym[rk];
            } else if (rk == 2) {
                xc = xA - dt * vxm[rk];
                yc = yA - dt * vym[rk];
            }
        }
        xc = xA - dt * (1.0 / 6.0) * (vxm[0] + 2 * vxm[1] + 2 * vxm[2] + vxm[3]);
        yc = yA - dt * (1.0 / 6.0) * (vym[0] + 2 * vym[1] + 2 * vym[2] + vym[3]);
        int i, j;
        double w[4];
        grid_weights(g, GP, xc, yc, i, j, w);
        if (pass == 0) {
            AT(G.f[G_pr0], Ny1, ii, jj) = gather4(G.f[G_pr], Ny1, i, j, w);
            AT(G.f[G_ps0], Ny1, ii, jj) = gather4(G.f[G_ps], Ny1, i, j, w);
        } else {
            AT(G.f[G_pf0], Ny1, ii, jj) = gather4(G.f[G_pf], Ny1, i, j, w);
        }
    }
}

int advect(erebus_state *s, double dt) {
    int n = (int)s->marknum;
    timer_begin(s, PH_RK4);
    if (n > 0)
        EREBUS_LAUNCH(s, k_rk4, nblocks(n, 128), 128, 0, s->p, s->g, mptr(s), gptr(s), n, dt);
    timer_end(s, PH_RK4);
    timer_begin(s, PH_BACKTRACE);
    size_t np = (size_t)s->g.Nx1 * s->g.Ny1;
    cudaMemcpyAsync(s->grid[G_pr0], s->grid[G_pr], np * 8, cudaMemcpyDeviceToDevice, s->stream);
    cudaMemcpyAsync(s->grid[G_ps0], s->grid[G_ps], np * 8, cudaMemcpyDeviceToDevice, s->stream);
    cudaMemcpyAsync(s->grid[G_pf0], s->grid[G_pf], np * 8, cudaMemcpyDeviceToDevice, s->stream);
    EREBUS_LAUNCH(s, k_backtrace, nblocks((int64_t)(s->g.Ny - 1) * (s->g.Nx - 1), 128), 128,
                  0, s->g, gptr(s), dt);
    timer_end(s, PH_BACKTRACE);
    s->sorted_valid = false;   // markers moved
    return check_cuda(s, cudaGetLastError(), "advect");
}

// ---------------------------------------------------------------------------
// replenish_markers! (E:5586-5698)
// ---------------------------------------------------------------------------
__global__ void k_repl_init(int na, unsigned long long *mdis, int *mnum, int *src,
                            int *flag) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    mdis[a] = (unsigned long long)__double_as_longlong(1.0e30);   // mdis_init (C:122)
    mnum[a] = INT_MAX;
    src[a] = -1;
    flag[a] = 0;
}

__device__ __forceinline__ void repl_cell(const Geo &g, double x, double y, int &i, int &j) {
    fix(x, y, g.dxm / 2, g.dym / 2, g.dxm, g.dym, 1, g.Nxm - 1, 1, g.Nym - 1, i, j);
}

// update_marker_population_geometry! (E:5518-5544) as a min-reduction of
// the distance per anchor ...
__global__ void k_repl_mindist(Geo g, const double *xm, const double *ym, int n,
                               unsigned long long *mdis) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    int i, j;
    double x = xm[m], y = ym[m];
    repl_cell(g, x, y, i, j);
#pragma unroll
    for (int c = 0; c < 4; c++) {
        int ii = i + (c & 1), jj = j + (c >> 1);
        double ddx = x - ax(g.dxm / 2, g.dxm, jj), ddy = y - ax(g.dym / 2, g.dym, ii);
        double d = sqrt(ddx * ddx + ddy * ddy);
        // non-negative doubles order like their bit patterns; strict `<`
        // against the initial 1e30 is kept by the reduction below
        atomicMin(&AT(mdis, g.Nym, ii, jj), (unsigned long long)__double_as_longlong(d));
    }
}
// ... then the smallest marker number among those at the minimum distance
// (the first one in marker order wins the strict `<`).
__global__ void k_repl_minidx(Geo g, const double *xm, const double *ym, int n,
                              const unsigned long long *mdis, int *mnum) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    int i, j;
    double x = xm[m], y = ym[m];
    repl_cell(g, x, y, i, j);
#pragma unroll
    for (int c = 0; c < 4; c++) {
        int ii = i + (c & 1), jj = j + (c >> 1);
        double ddx = x - ax(g.dxm / 2, g.dxm, jj), ddy = y - ax(g.dym / 2, g.dym, ii);
        double d = sqrt(ddx * ddx + ddy * ddy);
        unsigned long long b = (unsigned long long)__double_as_longlong(d);
        if (d < 1.0e30 && b == AT(mdis, g.Nym, ii, jj)) atomicMin(&AT(mnum, g.Nym, ii, jj), m);
    }
}
// Empty anchors search the +-5-cell window (E:5638-5653) in the reference's
// scan order among anchors that own a marker.
__global__ void k_repl_search(Geo g, int dii, int djj, const double *xm, const double *ym,
                              const int *mnum, int *src, int *flag) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    int Nym = g.Nym, Nxm = g.Nxm;
    if (a >= Nym * Nxm) return;
    if (mnum[a] != INT_MAX) return;
    int i = a % Nym + 1, j = a / Nym + 1;
    double xa = ax(g.dxm / 2, g.dxm, j), ya = ax(g.dym / 2, g.dym, i);
    double best = 1.0e30;
    int bm = -1;
    int jlo = max(j - djj, 1), jhi = min(j + djj, Nxm);
    int ilo = max(i - dii, 1), ihi = min(i + dii, Nym);
    for (int jj = jlo; jj <= jhi; jj++)
        for (int ii = ilo; ii <= ihi; ii++) {
            int mm = AT(mnum, Nym, ii, jj);
            if (mm != INT_MAX) {
                double ddx = xm[mm] - xa, ddy = ym[mm] - ya;
                double d = sqrt(ddx * ddx + ddy * ddy);
                if (d < best) { best = d; bm = mm; }
            }
        }
    src[a] = bm;
    flag[a] = bm >= 0;
}

// Exclusive scan of the anchor flags in anchor order, in three passes over
// tiles of SCAN_B anchors: tile sums, a scan of the tile sums (one block;
// also the number of new markers), and the scan inside each tile.
constexpr int SCAN_B = 1024;

// exclusive prefix of v over the SCAN_B threads of the block; *total = sum
__device__ int block_exclusive_scan(int v, int *wsum, int *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[lane] = s;   // inclusive warp-total prefix
    }
    __syncthreads();
    int excl = x - v + (w > 0 ? wsum[w - 1] : 0);
    *total = wsum[31];
    __syncthreads();
    return excl;
}

__global__ void k_repl_tile_sums(const int *flag, int na, int *part) {
    __shared__ int wsum[32];
    int k = blockIdx.x * SCAN_B + threadIdx.x, tot;
    block_exclusive_scan(k < na ? flag[k] : 0, wsum, &tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void k_repl_scan_tiles(int *part, int ntiles, DevScalars *sc) {
    __shared__ int wsum[32];
    int carry = 0;
    for (int b = 0; b < ntiles; b += SCAN_B) {
        int k = b + threadIdx.x, tot;
        int v = k < ntiles ? part[k] : 0;
        int e = block_exclusive_scan(v, wsum, &tot);
        if (k < ntiles) part[k] = carry + e;
        carry += tot;
    }
    if (threadIdx.x == 0) sc->repl_count = carry;
}

__global__ void k_repl_scan(const int *flag, int na, const int *part, int *rank) {
    __shared__ int wsum[32];
    int k = blockIdx.x * SCAN_B + threadIdx.x, tot;
    int e = block_exclusive_scan(k < na ? flag[k] : 0, wsum, &tot);
    if (k < na) rank[k] = part[blockIdx.x] + e;
}

__global__ void k_repl_append(ErebusParams p, Geo g, MP M, const int *src, const int *flag,
                              const int *rank, int marknum, int64_t capacity,
                              const DevScalars *sc, int timestep) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= g.Nym * g.Nxm || !flag[a]) return;
    if ((int64_t)marknum + sc->repl_count > capacity) return;
    int n = marknum + rank[a], sm = src[a];
    int i = a % g.Nym + 1, j = a / g.Nym + 1;
    double xa = ax(g.dxm / 2, g.dxm, j), ya = ax(g.dym / 2, g.dym, i);
    if (p.random_markers) {
        M.f[M_xm][n] = xa + (u01(p.seed, 2 * (uint64_t)timestep, a) - 0.5) * g.dxm;
        M.f[M_ym][n] = ya + (u01(p.seed, 2 * (uint64_t)timestep + 1, a) - 0.5) * g.dym;
    } else {
        M.f[M_xm][n] = xa;
        M.f[M_ym][n] = ya;
    }
    M.tm[n] = M.tm[sm];
    for (int f = M_tkm; f < M_COUNT; f++)
        if (M.f[f]) M.f[f][n] = M.f[f][sm];
}

int replenish(erebus_state *s, int timestep, int64_t *marknum) {
    const Geo &g = s->g;
    int na = g.Nxm * g.Nym, n = (int)s->marknum;
    int *flag = s->a_flag;
    EREBUS_LAUNCH(s, k_repl_init, nblocks(na), kThreads, 0, na, s->a_mdis, s->a_mnum,
                  s->a_src, flag);
    if (n > 0) {
        EREBUS_LAUNCH(s, k_repl_mindist, nblocks(n), kThreads, 0, g, s->m[M_xm], s->m[M_ym],
                      n, s->a_mdis);
        EREBUS_LAUNCH(s, k_repl_minidx, nblocks(n), kThreads, 0, g, s->m[M_xm], s->m[M_ym],
                      n, s->a_mdis, s->a_mnum);
    }
    EREBUS_LAUNCH(s, k_repl_search, nblocks(na), kThreads, 0, g, 5 * s->p.Nymc,
                  5 * s->p.Nxmc, s->m[M_xm], s->m[M_ym], s->a_mnum, s->a_src, flag);
    int ntiles = (int)((na + SCAN_B - 1) / SCAN_B);
    EREBUS_LAUNCH(s, k_repl_tile_sums, ntiles, SCAN_B, 0, flag, (int)na, s->a_part);
    EREBUS_LAUNCH(s, k_repl_scan_tiles, 1, SCAN_B, 0, s->a_part, ntiles, s->dsc);
    EREBUS_LAUNCH(s, k_repl_scan, ntiles, SCAN_B, 0, flag, (int)na, s->a_part, s->a_rank);
    EREBUS_LAUNCH(s, k_repl_append, nblocks(na), kThreads, 0, s->p, g, mptr(s), s->a_src,
                  flag, s->a_rank, n, s->capacity, s->dsc, timestep);
    int rc = check_cuda(s, cudaMemcpyAsync(&s->hsc->repl_count, &s->dsc->repl_count,
                                           sizeof(int), cudaMemcpyDeviceToHost, s->stream),
                        "replenish count");
    if (rc) return rc;
    rc = stream_sync(s, "replenish");
    if (rc) return rc;
    int add = s->hsc->repl_count;
    if ((int64_t)n + add > s->capacity) {
        s->last_error = "replenish_markers!: marker capacity exceeded";
        return EREBUS_ECAPACITY;
    }
    s->marknum = n + add;
    s->sorted_valid = false;
    if (marknum) *marknum = s->marknum;
    return EREBUS_OK;
}

}  // namespace erebus

// ---------------------------------------------------------------------------
// Allocation-free marker -> node pass (erebus_markers_to_nodes_noalloc)
//
// For callers that own all device memory themselves (a host framework with
// its own pool allocator, an application held to a fixed device-memory
// budget): the pass takes the caller's device buffers for inputs and
// outputs and keeps its scratch -- the four cell sorts and the weighted
// sums of one node set -- in the file-scope array below, so no call
// allocates.  The array occupies about 6.4 MB on every GPU that loads the
// library, until the process exits.  All calls share it and it keeps the
// last call's contents (counters are cleared at the start of each call);
// calls that overlap on the GPU race.
// ---------------------------------------------------------------------------
namespace erebus {

constexpr size_t NA_MARKERS = EREBUS_NOALLOC_MAX_MARKERS;
constexpr size_t NA_NODES = EREBUS_NOALLOC_MAX_NODES;
constexpr size_t NA_SUM_BYTES = 10 * NA_NODES * sizeof(double);
constexpr size_t NA_SORT_INTS = 4 * (3 * (NA_NODES + 1) + 2 * NA_MARKERS);
constexpr size_t NA_BYTES =
    ((NA_SUM_BYTES + NA_SORT_INTS * sizeof(int) + NA_MARKERS + 256 + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// tm (int64, the caller's layout) -> int8; types outside 1..3 become 3 (so
// every table index stays in range) and raise *err.
__global__ void k_noalloc_tm(const int64_t *tm, int8_t *tm8, int n, int *err) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    int64_t t = tm[m];
    if (t < 1 || t > 3) {
        atomicExch(err, 1);
        t = 3;
    }
    tm8[m] = (int8_t)t;
}

}  // namespace erebus

extern "C" int erebus_markers_to_nodes_noalloc(const ErebusParams *p,
                                               const ErebusMarkersDevice *md,
                                               int64_t marknum,
                                               const ErebusGridDevice *gd,
                                               double timesum, void *stream_) {
    using namespace erebus;
    if (!p || !md || !gd || marknum < 0) return EREBUS_EINVAL;
    if (erebus_check_params(p) != EREBUS_OK) return EREBUS_EINVAL;
    Geo g = make_geo(*p);
    if (marknum > (int64_t)NA_MARKERS || (size_t)g.Nx1 * g.Ny1 > NA_NODES)
        return EREBUS_ECAPACITY;
    const void *const *mp = reinterpret_cast<const void *const *>(md);
    for (int f = 0; f < M_COUNT; f++)
        if (!mp[f] && !(f == M_etasolidm_m && !p->per_marker_eta)) return EREBUS_EINVAL;
    const void *need[] = {gd->ETA0, gd->ETA, gd->GGG, gd->SXY0, gd->COH, gd->TEN, gd->FRI,
                          gd->YNY, gd->RHOX, gd->RHOFX, gd->KX, gd->PHIX, gd->RX, gd->RHOY,
                          gd->RHOFY, gd->KY, gd->PHIY, gd->RY, gd->RHO, gd->RHOCP, gd->ALPHA,
                          gd->ALPHAF, gd->HR, gd->GGGP, gd->SXX0, gd->tk1, gd->PHI,
                          gd->BETAPHI};
    for (const void *q : need)
        if (!q) return EREBUS_EINVAL;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream_);

    // Set-up, with the calling device current: the device address of the
    // scratch array (its host-side name is only a stand-in).  It is looked
    // up on every call rather than cached, because the address can change
    // when the device's primary context is torn down and created again
    // (cudaDeviceReset); after the first call on a device the lookup is a
    // host-side table read.
    unsigned char *base = nullptr;
    {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr)
            return EREBUS_ECUDA;
        base = static_cast<unsigned char *>(ptr);
    }
    // A launch error left behind by an unrelated earlier call is cleared
    // here, so that the check after this call's launches reports only its own.
    (void)cudaGetLastError();

    // carve the scratch
    double *sums = reinterpret_cast<double *>(base);
    int *ip = reinterpret_cast<int *>(base + NA_SUM_BYTES);
    SortPtrs S;
    for (int gr = 0; gr < 4; gr++) {
        GridSpec sp = grid_spec(g, gr);
        S.ncells[gr] = sp.rows * sp.cols;
        S.count[gr] = ip;  ip += NA_NODES + 1;
        S.cursor[gr] = ip; ip += NA_NODES + 1;
        S.start[gr] = ip;  ip += NA_NODES + 1;
        S.idx[gr] = ip;    ip += NA_MARKERS;
        S.tmp[gr] = ip;    ip += NA_MARKERS;
    }
    int8_t *tm8 = reinterpret_cast<int8_t *>(ip);
    int *err = reinterpret_cast<int *>(base + NA_BYTES - 256);

    MP M;
    for (int f = 0; f < M_COUNT; f++) M.f[f] = const_cast<double *>(static_cast<const double *>(mp[f]));
    M.f[M_tm] = nullptr;
    M.tm = tm8;
    GPtr G;
    const void *const *gp = reinterpret_cast<const void *const *>(gd);
    for (int f = 0; f < G_COUNT; f++) G.f[f] = const_cast<double *>(static_cast<const double *>(gp[f]));

    // calculate_radioactive_heating (E:1336-1357), on the host
    Heat h = {};
    if (p->hr_al) {
        double Q = p->f_al * p->ratio_al * p->E_al * exp(-timesum * (1.0 / g.tau_al)) *
                   (1.0 / g.tau_al);
        h.hrs[0] = Q * p->rhosolidm[0];
        h.hrs[1] = Q * p->rhosolidm[1];
    }
    if (p->hr_fe) {
        double Q = p->f_fe * p->ratio_fe * p->E_fe * exp(-timesum * (1.0 / g.tau_fe)) *
                   (1.0 / g.tau_fe);
        h.hrf[0] = Q * p->rhofluidm[0];
    }

    int n = (int)marknum;
    cudaMemsetAsync(err, 0, sizeof(int), st);
    for (int gr = 0; gr < 4; gr++) {
        cudaMemsetAsync(S.count[gr], 0, sizeof(int) * S.ncells[gr], st);
        cudaMemsetAsync(S.cursor[gr], 0, sizeof(int) * S.ncells[gr], st);
    }
    if (n > 0) {
        k_noalloc_tm<<<nblocks(n), kThreads, 0, st>>>(
            reinterpret_cast<const int64_t *>(mp[M_tm]), tm8, n, err);
        k_marker_props<<<nblocks(n), kThreads, 0, st>>>(*p, g, M, n, h);
        k_sort_count<<<nblocks(n), kThreads, 0, st>>>(g, M.f[M_xm], M.f[M_ym], n, S);
    }
    k_sort_scan<<<4, 1024, 0, st>>>(S);
    if (n > 0) k_sort_place<<<nblocks(n), kThreads, 0, st>>>(g, M.f[M_xm], M.f[M_ym], n, S);
    for (int gr = 0; gr < 4; gr++)
        k_sort_segments<<<nblocks((int64_t)S.ncells[gr] * 32), kThreads, 0, st>>>(S, gr);
    auto args = [&](int gr) {
        MergeArgs a = {};
        a.start = S.start[gr];
        a.idx = S.idx[gr];
        for (int f = 0; f < 10; f++) a.sums[f] = sums + (size_t)f * NA_NODES;
        return a;
    };
    auto blocks = [&](int gr) {
        GridSpec sp = grid_spec(g, gr);
        return nblocks((int64_t)sp.rows * sp.cols, 128);
    };
    k_merge<GB, MM_SCATTER><<<blocks(GB), 128, 0, st>>>(g, M, args(GB), G, 1);
    k_merge<GVX, MM_SCATTER><<<blocks(GVX), 128, 0, st>>>(g, M, args(GVX), G, 1);
    k_merge<GVY, MM_SCATTER><<<blocks(GVY), 128, 0, st>>>(g, M, args(GVY), G, 1);
    k_merge<GP, MM_SCATTER><<<blocks(GP), 128, 0, st>>>(g, M, args(GP), G, 1);
    k_insulate_rows<<<nblocks(g.Nx1), kThreads, 0, st>>>(g, G.f[G_tk1]);
    k_insulate_cols<<<nblocks(g.Ny1), kThreads, 0, st>>>(g, G.f[G_tk1]);
    int herr = 0;
    if (cudaGetLastError() != cudaSuccess) return EREBUS_ECUDA;
    if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return EREBUS_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return EREBUS_ECUDA;
    return herr ? EREBUS_EINVAL : EREBUS_OK;
}
