// bandlu.cu -- direct solver for the row-scaled banded systems.
//
// The reference factorises every system with a sparse direct LU (UMFPACK,
// E:6612, E:6736-6748, E:6925).  Here the systems keep the reference's
// unknown order (interleaved vx, vy, P, qx, qy, Pf per node, nodes
// column-major), whose half bandwidth is 6*Ny1+2 (Stokes-Darcy) or Ny1
// (heat, gravity).  The band is stored as nb x nb tiles and factorised by a
// right-looking tile LU without pivoting (the rows are scaled by their
// absolute sums first; in that order the no-pivot LU is stable for these
// systems and one step of iterative refinement reaches the residual of a
// pivoted solve).  Each step K factors the diagonal tile in one CTA and
// keeps explicit inverses of its triangular factors, turns the tiles of
// row/column K into U/L tiles with tile products, and updates the trailing
// band with tile GEMMs (FP64 FMA).  The steps run inside one persistent
// cooperative kernel separated by a grid barrier whose waits are bounded in
// time: on timeout the kernel records an error and runs to completion.
#include <cooperative_groups.h>
#include "solver.cuh"
#include "tiles.cuh"

namespace erebus {

// Invert diagonal tile (K,K), whose updated values are in registers `a`,
// and store the inverse in its place.
__device__ void invert_and_store(const BandView &B, int K, double a[4][4], FactorSmem &S,
                                 int *err) {
    tile_inverse(a, S.vec, err);
    regs_to_smem(S.Cs, a);
    __syncthreads();
    unstage_tile(tile_ptr(B, K, K), S.Cs);
    __syncthreads();
}

// Right-looking block LU without pivoting, with inverted diagonal blocks:
// A = L U with L_KK = I, L_IK = A_IK D_K^{-1}, U_KJ = A_KJ (the Schur-updated
// blocks) and D_K the Schur-updated diagonal block, whose inverse replaces
// tile (K,K).  Step K:
//   (B) L_IK <- A_IK D_K^{-1} (tile products);
//   (C) A_IJ -= L_IK A_KJ over the trailing band; CTA 0 takes (K+1,K+1) and
//       inverts it right away (look-ahead), so step K+1 starts with D^{-1}.
// Two grid barriers per step.
__global__ void __launch_bounds__(LU_THREADS, 2)
k_band_factor(BandView B, unsigned int *bar, int *err) {
    extern __shared__ __align__(16) double smem_raw[];
    FactorSmem &S = *reinterpret_cast<FactorSmem *>(smem_raw);
    const int NB = B.NB, Bb = B.Bb;
    if (blockIdx.x == 0) {
        double a[4][4];
        stage_tile(S.Cs, tile_ptr(B, 0, 0));
        __syncthreads();
        regs_from_smem(S.Cs, a);
        __syncthreads();
        invert_and_store(B, 0, a, S, err);
    }
    grid_barrier(bar, err);
    for (int K = 0; K < NB - 1; K++) {
        int nJ = min(Bb, NB - 1 - K);
        // (B) L_IK = A_IK * D_K^{-1}; CTA 0 is left free for the look-ahead
        int nw = gridDim.x > 1 ? gridDim.x - 1 : 1, w = gridDim.x > 1 ? (int)blockIdx.x - 1 : 0;
        for (int t = w; w >= 0 && t < nJ; t += nw) {
            double acc[4][4] = {};
            double *T = tile_ptr(B, K + 1 + t, K);
            stage_tile(S.As, T);
            stage_tile_t(S.Bt, tile_ptr(B, K, K));
            __syncthreads();
            gemm_acc(S.As, S.Bt, acc);
            regs_to_smem(S.Cs, acc);
            __syncthreads();
            unstage_tile(T, S.Cs);
            __syncthreads();
        }
        grid_barrier(bar, err);
        // (C) trailing update; task 0 = tile (K+1, K+1) on CTA 0
        for (int t = blockIdx.x; t < nJ * nJ; t += gridDim.x) {
            int aI = t % nJ, bJ = t / nJ;
            int I = K + 1 + aI, J = K + 1 + bJ;
            double acc[4][4];
            stage_tile(S.As, tile_ptr(B, I, K));
            stage_tile_t(S.Bt, tile_ptr(B, K, J));
            stage_tile(S.Cs, tile_ptr(B, I, J));
            __syncthreads();
            regs_from_smem(S.Cs, acc);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = -acc[i][j];
            gemm_acc(S.As, S.Bt, acc);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = -acc[i][j];
            __syncthreads();
            if (t == 0) {
                invert_and_store(B, K + 1, acc, S, err);
            } else {
                regs_to_smem(S.Cs, acc);
                __syncthreads();
                unstage_tile(tile_ptr(B, I, J), S.Cs);
                __syncthreads();
            }
        }
        grid_barrier(bar, err);
    }
}

// ---------------------------------------------------------------------------
// triangular solves: one thread-block cluster of SOLVE_P CTAs
//
// Tile row I is owned by CTA I % SOLVE_P, which keeps the partial sums of
// its rows of the current window in shared memory.  Forward sweep (L has
// identity diagonal blocks), step K: subtract L_IK y_K from the CTA's own
// rows I in (K, K+nI]; row K+1 is then final.  Backward sweep, step K:
// subtract U_IK x_K from the own rows I in [K-nI, K), and the owner of row
// K-1 applies D_{K-1}^{-1}.  The owner of the row that becomes final
// updates it first and pushes it into every CTA's row queue (DSMEM stores,
// then a remote mbarrier arrive with release semantics at cluster scope);
// each CTA waits for the rows in push order (acquire at cluster scope), so
// steps need no cluster-wide barrier.  The tiles (and the right-hand side of
// the row entering the window) a CTA needs at the next step are fetched
// with TMA bulk copies into the other buffer while the current step runs.
// Every wait is bounded in time.  Pushes run at most SOLVE_P + 1 rows ahead
// of the slowest CTA (each CTA owns every SOLVE_P-th row), below the queue
// depth SOLVE_Q, so a queue slot is never overwritten before it is read.
// ---------------------------------------------------------------------------
constexpr int SOLVE_P = 8;
constexpr int SOLVE_MAXT = 3;       // tiles per CTA and step (rows + inverse)
constexpr int SOLVE_RING = 4;       // owned-row slots
constexpr int SOLVE_Q = 16;         // pushed-row queue depth

struct SolveSmem {
    double tiles[2][SOLVE_MAXT][NB_TILE * NB_TILE];
    double rhs[2][NB_TILE];          // entering row of each buffered step
    double ring[SOLVE_RING][NB_TILE];
    double queue[SOLVE_Q][NB_TILE];  // finished rows pushed by their owners
    double wk[NB_TILE];
    double part[4][NB_TILE];
    unsigned long long mbar[2];      // TMA buffers
    unsigned long long qbar[SOLVE_Q];  // queue slots
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                             unsigned long long *b) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(smem_u32(b)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_try_cluster(unsigned long long *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(smem_u32(b)), "r"(parity) : "memory");
    return ok != 0;
}
// Remote arrive on the mbarrier at the same shared-memory offset in CTA `rank`.
__device__ __forceinline__ void mbar_arrive_remote(unsigned long long *b, uint32_t rank) {
    asm volatile(
        "{\n .reg .b32 ra;\n mapa.shared::cluster.u32 ra, %0, %1;\n"
        " mbarrier.arrive.release.cluster.shared::cluster.b64 _, [ra];\n}\n"
        ::"r"(smem_u32(b)), "r"(rank) : "memory");
}
__device__ void mbar_wait(unsigned long long *b, uint32_t parity, int *err, bool cluster) {
    if (cluster ? mbar_try_cluster(b, parity) : mbar_try(b, parity)) return;
    unsigned long long t0 = globaltimer();
    while (!(cluster ? mbar_try_cluster(b, parity) : mbar_try(b, parity))) {
        if (globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
            atomicExch(err, 3);
            return;
        }
    }
}

// What CTA `me` loads for step K of a sweep: the tiles of its rows of the
// window (forward L_IK, I in (K, K+nI]; backward U_IK, I in [K-nI, K)), the
// inverse D_{K-1}^{-1} if it owns row K-1 (backward), and the right-hand
// side of the row entering the window at step K if it owns it.  The row
// finished at this step (K+1 forward, K-1 backward) comes first.
struct StepLoad {
    int n;
    const double *src[SOLVE_MAXT];
    int row[SOLVE_MAXT];            // target row, -1 for the inverse
    int enter;                      // entering row (owned), or -1
};
__device__ __forceinline__ StepLoad step_load(const BandView &B, int K, bool fwd, int me,
                                              bool first) {
    StepLoad s;
    s.n = 0;
    s.enter = -1;
    const int NB = B.NB, Bb = B.Bb;
    if (fwd) {
        if (K >= NB - 1) return s;
        int nI = min(Bb, NB - 1 - K);
        for (int I = K + 1; I <= K + nI; I++)
            if (I % SOLVE_P == me && s.n < SOLVE_MAXT) {
                s.src[s.n] = tile_ptr(B, I, K);
                s.row[s.n++] = I;
            }
        int er = K + Bb;
        if (!first && er < NB && er % SOLVE_P == me) s.enter = er;
    } else {
        if (K <= 0) return s;
        int nI = min(Bb, K);
        for (int I = K - 1; I >= K - nI; I--)
            if (I % SOLVE_P == me && s.n < SOLVE_MAXT - 1) {
                s.src[s.n] = tile_ptr(B, I, K);
                s.row[s.n++] = I;
            }
        if ((K - 1) % SOLVE_P == me) {
            s.src[s.n] = tile_ptr(B, K - 1, K - 1);
            s.row[s.n++] = -1;
        }
        int er = K - Bb;
        if (!first && er >= 0 && er % SOLVE_P == me) s.enter = er;
    }
    return s;
}

__device__ __forceinline__ void issue_load(const double *w, SolveSmem &S, const StepLoad &sl,
                                           int stage) {
    if (threadIdx.x != 0) return;
    uint32_t bytes = sl.n * NB_TILE * NB_TILE * sizeof(double) +
                     (sl.enter >= 0 ? NB_TILE * sizeof(double) : 0);
    if (bytes == 0) return;
    mbar_expect(&S.mbar[stage], bytes);
    for (int q = 0; q < sl.n; q++)
        tma_bulk_g2s(S.tiles[stage][q], sl.src[q], NB_TILE * NB_TILE * sizeof(double),
                     &S.mbar[stage]);
    if (sl.enter >= 0)
        tma_bulk_g2s(S.rhs[stage], w + (int64_t)sl.enter * NB_TILE, NB_TILE * sizeof(double),
                     &S.mbar[stage]);
}

// y = T v (column-major tile in smem, unpadded) with all 256 threads: four
// column quarters per row, four independent chains each, reduced through
// `part`.  mode 0: y -= T v; mode 1: y = T v.
__device__ __forceinline__ void smem_gemv(const double *T, const double *v, double *y,
                                          double (*part)[NB_TILE], int mode) {
    int r = threadIdx.x & 63, q = threadIdx.x >> 6;
    const double *t = T + q * 16 * NB_TILE + r;
    const double *vv = v + q * 16;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
    for (int c = 0; c < 16; c += 4) {
        s0 = fma(t[(c + 0) * NB_TILE], vv[c + 0], s0);
        s1 = fma(t[(c + 1) * NB_TILE], vv[c + 1], s1);
        s2 = fma(t[(c + 2) * NB_TILE], vv[c + 2], s2);
        s3 = fma(t[(c + 3) * NB_TILE], vv[c + 3], s3);
    }
    part[q][r] = (s0 + s1) + (s2 + s3);
    __syncthreads();
    if (threadIdx.x < NB_TILE) {
        double s = (part[0][r] + part[1][r]) + (part[2][r] + part[3][r]);
        y[r] = mode == 0 ? y[r] - s : s;
    }
    __syncthreads();
}

// Push the finished row `src` (smem, 64 values) as queue entry `seq` into
// every CTA of the cluster, and write it to global memory.
__device__ __forceinline__ void push_row(cooperative_groups::cluster_group &cluster,
                                         SolveSmem &S, const double *src, int seq,
                                         double *wrow) {
    int slot = seq % SOLVE_Q;
    if (threadIdx.x < NB_TILE) {
        double v = src[threadIdx.x];
        wrow[threadIdx.x] = v;
#pragma unroll
        for (int c = 0; c < SOLVE_P; c++) {
            double *dst = cluster.map_shared_rank(&S.queue[slot][0], c);
            dst[threadIdx.x] = v;
        }
        asm volatile("fence.acq_rel.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x < SOLVE_P) mbar_arrive_remote(&S.qbar[slot], threadIdx.x);
}

__global__ void __cluster_dims__(SOLVE_P, 1, 1) __launch_bounds__(LU_THREADS, 1)
k_band_solve(BandView B, double *w, int *err) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(128) double smem_raw[];
    SolveSmem &S = *reinterpret_cast<SolveSmem *>(smem_raw);
    const int me = (int)cluster.block_rank();
    const int NB = B.NB, Bb = B.Bb;
    auto slot = [&](int I) { return (I / SOLVE_P) % SOLVE_RING; };
    uint32_t uses[2] = {0u, 0u};
    if (threadIdx.x == 0) {
        mbar_init(&S.mbar[0]);
        mbar_init(&S.mbar[1]);
        for (int q = 0; q < SOLVE_Q; q++) mbar_init(&S.qbar[q]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    cluster.sync();   // every queue barrier exists before the first push
    int step = 0;     // running step index over both sweeps (buffer = step & 1)
    for (int sweep = 0; sweep < 2; sweep++) {
        const bool fwd = sweep == 0;
        const int K0 = fwd ? 0 : NB - 1;
        const int seq0 = fwd ? 0 : NB;   // queue sequence of the sweep's first row
        // rows of the first window: [0, Bb] forward, [NB-1-Bb, NB-1] backward
        int lo = fwd ? 0 : max(0, NB - 1 - Bb), hi = fwd ? min(NB - 1, Bb) : NB - 1;
        for (int I = lo; I <= hi; I++)
            if (I % SOLVE_P == me && threadIdx.x < NB_TILE)
                S.ring[slot(I)][threadIdx.x] = __ldcg(&w[(int64_t)I * NB_TILE + threadIdx.x]);
        StepLoad cur = step_load(B, K0, fwd, me, true);
        issue_load(w, S, cur, step & 1);
        __syncthreads();
        if (K0 % SOLVE_P == me) {     // first row: y_0 = w_0; x_{NB-1} = D^{-1} y_{NB-1}
            double *y = S.ring[slot(K0)];
            if (!fwd) {
                const double *inv = tile_ptr(B, K0, K0);
                if (threadIdx.x < NB_TILE) S.wk[threadIdx.x] = y[threadIdx.x];
                __syncthreads();
                int r = threadIdx.x & 63, q = threadIdx.x >> 6;
                double s = 0.0;
                for (int c = q * 16; c < q * 16 + 16; c++)
                    s = fma(__ldcg(&inv[c * NB_TILE + r]), S.wk[c], s);
                S.part[q][r] = s;
                __syncthreads();
                if (threadIdx.x < NB_TILE)
                    y[r] = (S.part[0][r] + S.part[1][r]) + (S.part[2][r] + S.part[3][r]);
                __syncthreads();
            }
            push_row(cluster, S, y, seq0, w + (int64_t)K0 * NB_TILE);
        }
        const int nsteps = NB - 1;
        for (int it = 0; it < nsteps; it++, step++) {
            const int K = fwd ? it : NB - 1 - it;
            const int Kn = fwd ? K + 1 : K - 1;      // row finished at this step
            const int stage = step & 1;
            StepLoad nxt;
            nxt.n = 0;
            nxt.enter = -1;
            if (it + 1 < nsteps) {                 // prefetch the next step
                nxt = step_load(B, fwd ? K + 1 : K - 1, fwd, me, false);
                issue_load(w, S, nxt, stage ^ 1);
            }
            // the finished row K, pushed by its owner
            const int seq = seq0 + it, qs = seq % SOLVE_Q;
            mbar_wait(&S.qbar[qs], (uint32_t)(seq / SOLVE_Q) & 1u, err, true);
            if (cur.n > 0 || cur.enter >= 0) {
                mbar_wait(&S.mbar[stage], uses[stage] & 1u, err, false);
                uses[stage]++;
            }
            if (cur.enter >= 0 && threadIdx.x < NB_TILE)
                S.ring[slot(cur.enter)][threadIdx.x] = S.rhs[stage][threadIdx.x];
            __syncthreads();
            const double *yk = S.queue[qs];
            const bool owner = Kn % SOLVE_P == me;
            if (owner) {   // the row finished at this step first, then push it
                double *y = S.ring[slot(Kn)];
                if (fwd) {
                    smem_gemv(S.tiles[stage][0], yk, y, S.part, 0);
                } else {
                    for (int q = 0; q < cur.n; q++)
                        if (cur.row[q] == Kn) smem_gemv(S.tiles[stage][q], yk, y, S.part, 0);
                    if (threadIdx.x < NB_TILE) S.wk[threadIdx.x] = y[threadIdx.x];
                    __syncthreads();
                    smem_gemv(S.tiles[stage][cur.n - 1], S.wk, y, S.part, 1);
                }
                push_row(cluster, S, y, seq + 1, w + (int64_t)Kn * NB_TILE);
            }
            for (int q = 0; q < cur.n; q++)
                if (cur.row[q] >= 0 && !(owner && cur.row[q] == Kn))
                    smem_gemv(S.tiles[stage][q], yk, S.ring[slot(cur.row[q])], S.part, 0);
            cur = nxt;
            fence_proxy_async();
            __syncthreads();
        }
        // the backward sweep reads the forward result (also through TMA)
        asm volatile("fence.proxy.async.global;" ::: "memory");
        __threadfence();
        cluster.sync();
    }
    for (int s = 0; s < 2; s++)
        if (uses[s] > 0) mbar_wait(&S.mbar[s], (uses[s] - 1) & 1u, err, false);
    cluster.sync();
}

// r = rhs - A x (scaled rows, ELL)
__global__ void k_band_residual(BandView B, const double *x, double *r) {
    int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= (int64_t)B.NB * B.nb) return;
    double s = B.rhs[row];
    for (int k = 0; k < B.ell; k++) {
        int c = B.ell_cols[row * B.ell + k];
        if (c >= 0) s -= B.ell_vals[row * B.ell + k] * x[c];
    }
    r[row] = s;
}

// y = A x with the unscaled entries
__global__ void k_band_apply(BandView B, const double *x, double *y) {
    int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= B.n) return;
    double s = 0.0;
    for (int k = 0; k < B.ell; k++) {
        int c = B.ell_cols[row * B.ell + k];
        if (c >= 0) s += B.ell_vals[row * B.ell + k] * x[c];
    }
    y[row] = s / B.rscale[row];
}

// Sums of squares of a and b in a fixed order: NORM_BLOCKS blocks write
// partial sums (block k takes the k-th contiguous chunk), then one block adds
// them up in block order -> out[0], out[1].
__global__ void k_norms2_part(const double *a, const double *b, int64_t n, double *part) {
    __shared__ double sa[NORM_THREADS], sb[NORM_THREADS];
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    double xa = 0.0, xb = 0.0;
    const int64_t st = blockDim.x;
    int64_t k = lo + threadIdx.x;
    for (; k + 3 * st < hi; k += 4 * st) {   // loads in flight first, sums in order
        const double a0 = a[k], a1 = a[k + st], a2 = a[k + 2 * st], a3 = a[k + 3 * st];
        const double b0 = b[k], b1 = b[k + st], b2 = b[k + 2 * st], b3 = b[k + 3 * st];
        xa = fma(a0, a0, xa);
        xb = fma(b0, b0, xb);
        xa = fma(a1, a1, xa);
        xb = fma(b1, b1, xb);
        xa = fma(a2, a2, xa);
        xb = fma(b2, b2, xb);
        xa = fma(a3, a3, xa);
        xb = fma(b3, b3, xb);
    }
    for (; k < hi; k += st) {
        xa = fma(a[k], a[k], xa);
        xb = fma(b[k], b[k], xb);
    }
    sa[threadIdx.x] = xa;
    sb[threadIdx.x] = xb;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            sa[threadIdx.x] += sa[threadIdx.x + off];
            sb[threadIdx.x] += sb[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sa[0];
        part[2 * blockIdx.x + 1] = sb[0];
    }
}
__global__ void k_norms2_sum(const double *part, int nparts, double *out) {
    __shared__ double sa[NORM_THREADS], sb[NORM_THREADS];
    double xa = 0.0, xb = 0.0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
        xa += part[2 * k];
        xb += part[2 * k + 1];
    }
    sa[threadIdx.x] = xa;
    sb[threadIdx.x] = xb;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            sa[threadIdx.x] += sa[threadIdx.x + off];
            sb[threadIdx.x] += sb[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sa[0];
        out[1] = sb[0];
    }
}

__global__ void k_axpy(double *x, const double *d, int64_t n) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) x[k] += d[k];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
BandSystem &band_of(erebus_state *s, int kind) {
    return kind == SYS_HYDRO ? s->hydro : kind == SYS_THERMAL ? s->thermal : s->gravity;
}

BandView band_view(BandSystem &sys) {
    BandView B;
    B.n = sys.n;
    B.nb = sys.nb;
    B.NB = sys.NB;
    B.Bb = sys.Bb;
    B.ell = sys.ell;
    B.tiles = sys.tiles;
    B.rhs = sys.rhs;
    B.rscale = sys.rscale;
    B.x = sys.x;
    B.ell_cols = sys.ell_cols;
    B.ell_vals = sys.ell_vals;
    return B;
}

static size_t tiles_bytes(const BandSystem &sys) {
    return (size_t)sys.NB * (2 * sys.Bb + 1) * sys.nb * sys.nb * sizeof(double);
}

int band_alloc(erebus_state *s, BandSystem &sys, int64_t n, int b, int nb, int ell) {
    sys.n = n;
    sys.b = b;
    sys.nb = NB_TILE;
    (void)nb;
    sys.NB = (int)((n + NB_TILE - 1) / NB_TILE);
    sys.Bb = (b + NB_TILE - 1) / NB_TILE;
    sys.ell = ell;
    int64_t np = (int64_t)sys.NB * sys.nb;
    cudaError_t e = cudaMalloc(&sys.rscale, np * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sys.rhs, np * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sys.x, np * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sys.r, np * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sys.d, np * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sys.ell_vals, np * ell * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sys.ell_cols, np * ell * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sys.ell_prev, np * ell * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sys.changed, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&sys.bar, 4 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&sys.err, sizeof(int));
    if (e != cudaSuccess) {
        s->last_error = std::string("band_alloc: ") + cudaGetErrorString(e);
        return EREBUS_ENOMEM;
    }
    cudaMemset(sys.bar, 0, 4 * sizeof(unsigned int));
    cudaMemset(sys.err, 0, sizeof(int));
    cudaMemset(sys.rscale, 0, np * 8);
    cudaMemset(sys.ell_prev, 0xff, np * ell * 8);   // NaN patterns: never equal
    return EREBUS_OK;
}

// The band storage of the band LU, allocated on first use.
static int band_tiles(erebus_state *s, BandSystem &sys) {
    if (sys.tiles) return EREBUS_OK;
    cudaError_t e = cudaMalloc(&sys.tiles, tiles_bytes(sys));
    if (e != cudaSuccess) {
        sys.tiles = nullptr;
        s->last_error = std::string("band storage: ") + cudaGetErrorString(e);
        return EREBUS_ENOMEM;
    }
    return EREBUS_OK;
}

int band_free(BandSystem &sys) {
    mf_release(sys);
    krylov_free(sys);
    void *ps[] = {sys.tiles, sys.rscale, sys.rhs, sys.x, sys.r,
                  sys.d, sys.ell_vals, sys.ell_cols, sys.ell_prev, sys.changed,
                  sys.bar, sys.err};
    for (void *p : ps)
        if (p) cudaFree(p);
    sys = BandSystem();
    return EREBUS_OK;
}

int band_zero(erebus_state *s, BandSystem &sys) {
    int rc = band_tiles(s, sys);
    if (rc) return rc;
    return check_cuda(s, cudaMemsetAsync(sys.tiles, 0, tiles_bytes(sys), s->stream),
                      "band_zero");
}

static int coop_blocks(erebus_state *s, const void *func, int threads, size_t smem, int want) {
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    int maxb = per_sm * sms;
    return want < maxb ? want : maxb;
}

int mf_check_error(erebus_state *s, BandSystem &sys, const char *what) {
    int h = 0;
    int rc = check_cuda(s, cudaMemcpyAsync(&h, sys.err, sizeof(int), cudaMemcpyDeviceToHost,
                                           s->stream), what);
    if (rc) return rc;
    rc = stream_sync(s, what);
    if (rc) return rc;
    if (h) {
        s->last_error = std::string(what) +
                        (h == 1 ? ": grid barrier timed out"
                         : h == 2 ? ": zero pivot"
                         : h == 3 ? ": wait timed out"
                                  : ": matrix pattern changed since the analysis");
        cudaMemsetAsync(sys.err, 0, sizeof(int), s->stream);
        mf_clear_counts(s, sys);
        if (h == 4) mf_release(sys);   // analysed again at the next factorisation
        return h == 2 ? EREBUS_ENOCONV : EREBUS_ECUDA;
    }
    return EREBUS_OK;
}

void band_stats(const BandSystem &sys, ErebusFactorStats *o) {
    double tiles = 0.0;
    for (int K = 0; K < sys.NB; K++) {
        int nJ = std::min(sys.Bb, sys.NB - 1 - K);
        tiles += 1 + nJ + (double)nJ * nJ;
    }
    o->fronts = 0;
    o->levels = sys.NB;
    o->storage_bytes = (int64_t)tiles_bytes(sys);
    o->flops = tiles * 2.0 * NB_TILE * NB_TILE * NB_TILE;
    o->solve_bytes = (double)tiles_bytes(sys);
}

bool use_multifrontal(const erebus_state *s) {
    return s->opt.direct_solver != EREBUS_SOLVER_BAND;
}

int band_factor(erebus_state *s, BandSystem &sys) {
    if (use_multifrontal(s)) return mf_factor(s, sys, s->opt.factor_fp32 != 0);
    int trc = band_tiles(s, sys);
    if (trc) return trc;
    size_t smem = sizeof(FactorSmem);
    cudaFuncSetAttribute(k_band_factor, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    int want = 1 + (sys.Bb * sys.Bb > 2 * sys.Bb ? sys.Bb * sys.Bb : 2 * sys.Bb);
    int blocks = coop_blocks(s, (const void *)k_band_factor, LU_THREADS, smem, want);
    if (blocks < 1) {
        s->last_error = "band_factor: kernel does not fit";
        return EREBUS_ECUDA;
    }
    BandView B = band_view(sys);
    unsigned int *bar = sys.bar;
    int *err = sys.err;
    void *args[] = {&B, &bar, &err};
    cudaMemsetAsync(sys.bar, 0, 4 * sizeof(unsigned int), s->stream);
    int rc = coop_launch(s, (const void *)k_band_factor, blocks, LU_THREADS, args, smem, "band_factor launch");
    s->launches++;
    if (rc) return rc;
    sys.factored = true;
    sys.factorizations++;
    return EREBUS_OK;
}

// In-place solve L U w = w with the cluster kernel.
static int band_solve_inplace(erebus_state *s, BandSystem &sys, double *w) {
    if (use_multifrontal(s)) return mf_solve(s, sys, w);
    if (sys.Bb > 2 * SOLVE_P) {
        s->last_error = "band_solve: band too wide for the cluster solve";
        return EREBUS_EINVAL;
    }
    size_t smem = sizeof(SolveSmem);
    cudaFuncSetAttribute(k_band_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    BandView B = band_view(sys);
    k_band_solve<<<SOLVE_P, LU_THREADS, smem, s->stream>>>(B, w, sys.err);
    s->launches++;
    return check_cuda(s, cudaGetLastError(), "band_solve launch");
}

// Solves accepted at a system's measured residual floor before refinement is
// run to the stall again.
constexpr int kFloorUses = 8;

int band_solve_refined(erebus_state *s, BandSystem &sys, double rtol, int max_ir,
                       ErebusSolveStats *st) {
    int rc;
    if (!sys.factored) {
        timer_begin(s, sys.ph_factor);
        rc = band_factor(s, sys);
        timer_end(s, sys.ph_factor);
        if (rc) return rc;
    }
    timer_begin(s, sys.ph_solve);
    int64_t np = (int64_t)sys.NB * sys.nb;
    BandView B = band_view(sys);
    // Iterative refinement x <- x + (LU)^{-1} (b - A x), started from the
    // previous solution of this system when there is one (the matrix or the
    // right-hand side changed little since), else from zero.
    bool cold = !sys.have_x;
    if (cold) cudaMemsetAsync(sys.x, 0, np * 8, s->stream);
    double rel = 0.0, prev = INFINITY;
    int solves = 0;
    bool escalated = false;
    // When the last solve of this system needed corrections, the first one is
    // made here before any norm is read back (one host round trip less); the
    // starting residual's norms are still computed and come back with the
    // first check, so a system whose starting points become good enough
    // (a state at rest) returns to checking first.
    double *part = s->norm_part;   // 2 * NORM_BLOCKS partial sums
    const bool forced = !sys.warm_ok;
    bool start_ok = false;
    if (forced) {
        EREBUS_LAUNCH(s, k_band_residual, nblocks(np), kThreads, 0, B, sys.x, sys.r);
        EREBUS_LAUNCH(s, k_norms2_part, NORM_BLOCKS, NORM_THREADS, 0, sys.r, sys.rhs, np, part);
        EREBUS_LAUNCH(s, k_norms2_sum, 1, NORM_THREADS, 0, part, NORM_BLOCKS, &s->dsc->norms0[0]);
        rc = band_solve_inplace(s, sys, sys.r);
        if (rc) return rc;
        EREBUS_LAUNCH(s, k_axpy, nblocks(np), kThreads, 0, sys.x, sys.r, np);
        solves = 1;
    }
    bool first_check = true;
    bool stalled = false, at_floor = false;
refine:
    for (;;) {
        EREBUS_LAUNCH(s, k_band_residual, nblocks(np), kThreads, 0, B, sys.x, sys.r);
        EREBUS_LAUNCH(s, k_norms2_part, NORM_BLOCKS, NORM_THREADS, 0, sys.r, sys.rhs, np, part);
        EREBUS_LAUNCH(s, k_norms2_sum, 1, NORM_THREADS, 0, part, NORM_BLOCKS, &s->dsc->norms[0]);
        rc = check_cuda(s, cudaMemcpyAsync(&s->hsc->norms[0], &s->dsc->norms[0],
                                           forced && first_check ? 32 : 16,
                                           cudaMemcpyDeviceToHost, s->stream), "norms");
        if (rc) return rc;
        rc = mf_check_error(s, sys, "LU");
        if (rc) return rc;
        double rr = s->hsc->norms[0], bb = s->hsc->norms[1];
        rel = bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
        if (forced && first_check) {
            const double r0 = s->hsc->norms0[0], b0 = s->hsc->norms0[1];
            start_ok = (b0 > 0.0 ? sqrt(r0 / b0) : sqrt(r0)) <= rtol;
        }
        first_check = false;
        if (rel <= rtol) break;
        if (!(rel < INFINITY)) {            // NaN/Inf: restart once from zero
            if (cold) break;
            cudaMemsetAsync(sys.x, 0, np * 8, s->stream);
            cold = true;
            prev = INFINITY;
            continue;
        }
        // refinement has reached the accuracy the factors allow: the last
        // correction did not halve the residual
        if (solves > 0 && rel > 0.5 * prev) { stalled = true; break; }
        // Within a factor 2 of the residual at which this system's refinement
        // last stalled, one more correction could at most halve it, and
        // refinement would stop after it.  Stop now, after at least one
        // correction; every kFloorUses-th solve refines to the stall again, so
        // the floor is measured afresh.
        if (solves > 0 && sys.floor_rel > 0.0 && rel <= 2.0 * sys.floor_rel &&
            sys.floor_uses < kFloorUses) {
            sys.floor_uses++;
            at_floor = true;
            break;
        }
        if (solves > max_ir) break;
        prev = rel;
        cudaMemcpyAsync(sys.d, sys.r, np * 8, cudaMemcpyDeviceToDevice, s->stream);
        rc = band_solve_inplace(s, sys, sys.d);
        if (rc) return rc;
        EREBUS_LAUNCH(s, k_axpy, nblocks(np), kThreads, 0, sys.x, sys.d, np);
        solves++;
    }
    // Mixed precision: when refinement with the FP32 factors stalls above the
    // target, factor this matrix again in FP64 and go on refining from the
    // current solution.
    if (!(rel <= rtol) && !at_floor && !escalated && use_multifrontal(s) && mf_is_fp32(sys)) {
        escalated = true;
        timer_end(s, sys.ph_solve);
        timer_begin(s, sys.ph_factor);
        rc = mf_factor(s, sys, false);
        timer_end(s, sys.ph_factor);
        if (rc) return rc;
        sys.fp64_refactorizations++;
        timer_begin(s, sys.ph_solve);
        prev = INFINITY;
        stalled = false;
        if (!(rel < INFINITY)) {
            cudaMemsetAsync(sys.x, 0, np * 8, s->stream);
            cold = true;
        }
        goto refine;
    }
    timer_end(s, sys.ph_solve);
    if (rel <= rtol) {
        sys.floor_rel = 0.0;
    } else if (stalled) {
        sys.floor_rel = rel;
        sys.floor_uses = 0;
    }
    sys.have_x = rel < 1e-6;   // good enough to start the next solve from
    sys.warm_ok = sys.have_x && (forced ? start_ok : solves == 0);
    if (st) {
        st->iterations = solves;
        st->converged = rel <= rtol;
        st->rel_residual = rel;
    }
    if (!(rel <= rtol) && !(rel < 1e-6)) {
        char msg[160];
        snprintf(msg, sizeof msg,
                 "%s solve did not reach tolerance: relative residual %.3e after %d "
                 "refinement steps (previous %.3e)", sys.name, rel, solves, prev);
        s->last_error = msg;
        return EREBUS_ENOCONV;
    }
    return EREBUS_OK;
}

int band_apply_unscaled(erebus_state *s, BandSystem &sys, const double *x, double *y) {
    BandView B = band_view(sys);
    EREBUS_LAUNCH(s, k_band_apply, nblocks(sys.n), kThreads, 0, B, x, y);
    return check_cuda(s, cudaGetLastError(), "band_apply");
}

}  // namespace erebus
