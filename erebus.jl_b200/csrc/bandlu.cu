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

namespace erebus {

constexpr int NB_TILE = 64;       // tile size
constexpr int LU_THREADS = 256;
constexpr unsigned long long BARRIER_TIMEOUT_NS = 2000000000ull;   // 2 s

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Sense-reversing grid barrier over all CTAs of a cooperative launch.
// bar[0] = arrival count, bar[1] = generation.  A wait that exceeds the
// timeout sets *err and returns.
__device__ void grid_barrier(unsigned int *bar, int *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *vgen = bar + 1;
        unsigned int gen = *vgen;
        __threadfence();
        unsigned int arrived = atomicAdd(bar, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned long long t0 = globaltimer();
            while (*vgen == gen) {
                if (globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// tile kernels (one CTA, 256 threads, nb = 64)
// ---------------------------------------------------------------------------
// mode 0: C -= A * B; mode 1: C = A * B (C may alias A or B).
// Shared memory: As[k][r] and Bt[k][c], 2 * 64 * 64 doubles.
__device__ void tile_gemm(const double *A, const double *Bm, double *C, int mode,
                          double *smem) {
    constexpr int nb = NB_TILE;
    double *As = smem, *Bt = smem + nb * nb;
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
        As[e] = A[e];                          // As[k*nb + r] = A(r,k)
        int k = e % nb, c = e / nb;            // B(k,c) at e
        Bt[k * nb + c] = Bm[e];
    }
    __syncthreads();
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
#pragma unroll 8
    for (int k = 0; k < nb; k++) {
        double2 a01 = *reinterpret_cast<const double2 *>(&As[k * nb + ty * 4]);
        double2 a23 = *reinterpret_cast<const double2 *>(&As[k * nb + ty * 4 + 2]);
        double2 b01 = *reinterpret_cast<const double2 *>(&Bt[k * nb + tx * 4]);
        double2 b23 = *reinterpret_cast<const double2 *>(&Bt[k * nb + tx * 4 + 2]);
        double av[4] = {a01.x, a01.y, a23.x, a23.y};
        double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int b = 0; b < 4; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
        for (int a = 0; a < 4; a++) {
            int r = ty * 4 + a, c = tx * 4 + b;
            double *p = &C[c * nb + r];
            *p = mode == 0 ? *p - acc[a][b] : acc[a][b];
        }
}

// LU (no pivoting) of the tile at T in place, and the inverses of its unit
// lower factor (Li) and upper factor (Ui).  Shared memory: 3 * nb * nb.
__device__ void tile_lu_inv(double *T, double *Li, double *Ui, double *smem, int *err) {
    constexpr int nb = NB_TILE;
    double *A = smem, *X = smem + nb * nb, *Y = smem + 2 * nb * nb;
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) A[e] = T[e];
    __syncthreads();
    for (int k = 0; k < nb; k++) {
        double piv = A[k * nb + k];
        if (threadIdx.x == 0 && !(piv != 0.0)) atomicExch(err, 2);
        for (int r = k + 1 + threadIdx.x; r < nb; r += blockDim.x) A[k * nb + r] /= piv;
        __syncthreads();
        int m = nb - k - 1;
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            int r = k + 1 + e % m, c = k + 1 + e / m;
            A[c * nb + r] -= A[k * nb + r] * A[c * nb + k];
        }
        __syncthreads();
    }
    // inverses: one thread per column
    int c = threadIdx.x;
    if (c < nb) {
        // X = U^{-1}: U X = I, back substitution in column c
        for (int r = nb - 1; r >= 0; r--) {
            double s = (r == c) ? 1.0 : 0.0;
            for (int k = r + 1; k < nb; k++) s -= A[k * nb + r] * X[c * nb + k];
            X[c * nb + r] = r > c ? 0.0 : s / A[r * nb + r];
        }
    } else if (c < 2 * nb) {
        c -= nb;
        // Y = L^{-1} (unit lower): forward substitution in column c
        for (int r = 0; r < nb; r++) {
            double s = (r == c) ? 1.0 : 0.0;
            for (int k = 0; k < r; k++) s -= A[k * nb + r] * Y[c * nb + k];
            Y[c * nb + r] = r < c ? 0.0 : s;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
        T[e] = A[e];
        Ui[e] = X[e];
        Li[e] = Y[e];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(LU_THREADS)
k_band_factor(BandView B, unsigned int *bar, int *err) {
    extern __shared__ double smem[];
    constexpr int nb = NB_TILE;
    const int NB = B.NB, Bb = B.Bb;
    const int64_t t2 = (int64_t)nb * nb;
    for (int K = 0; K < NB; K++) {
        if (blockIdx.x == 0)
            tile_lu_inv(tile_ptr(B, K, K), B.invL + K * t2, B.invU + K * t2, smem, err);
        grid_barrier(bar, err);
        int nJ = min(Bb, NB - 1 - K);
        for (int t = blockIdx.x; t < 2 * nJ; t += gridDim.x) {
            if (t < nJ) {   // U tile: A_KJ <- L_KK^{-1} A_KJ
                double *T = tile_ptr(B, K, K + 1 + t);
                tile_gemm(B.invL + K * t2, T, T, 1, smem);
            } else {        // L tile: A_IK <- A_IK U_KK^{-1}
                double *T = tile_ptr(B, K + 1 + (t - nJ), K);
                tile_gemm(T, B.invU + K * t2, T, 1, smem);
            }
            __syncthreads();
        }
        grid_barrier(bar, err);
        for (int t = blockIdx.x; t < nJ * nJ; t += gridDim.x) {
            int a = t % nJ, b = t / nJ;
            int I = K + 1 + a, J = K + 1 + b;
            tile_gemm(tile_ptr(B, I, K), tile_ptr(B, K, J), tile_ptr(B, I, J), 0, smem);
            __syncthreads();
        }
        grid_barrier(bar, err);
    }
}

// y (+)= T * x for one nb x nb tile; 4 threads per row.  mode 0: y -= Tx,
// mode 1: y = Tx.  x must not alias y.
__device__ __forceinline__ void tile_gemv(const double *T, const double *x, double *y,
                                          int mode) {
    constexpr int nb = NB_TILE;
    int r = threadIdx.x >> 2, q = threadIdx.x & 3;
    double s = 0.0;
#pragma unroll 4
    for (int c = q * 16; c < q * 16 + 16; c++) s = fma(T[c * nb + r], x[c], s);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (q == 0) y[r] = mode == 0 ? y[r] - s : s;
}

// Forward (L, unit) then backward (U) substitution of b -> x in place on
// `w` (length NB*nb).  CTA a of step K updates block K+1+a; the CTA that
// updates block K+1 also solves it, so one grid barrier per step suffices.
__global__ void __launch_bounds__(LU_THREADS)
k_band_solve(BandView B, double *w, unsigned int *bar, int *err) {
    __shared__ double xs[NB_TILE], ys[NB_TILE];
    constexpr int nb = NB_TILE;
    const int NB = B.NB, Bb = B.Bb;
    const int64_t t2 = (int64_t)nb * nb;
    // forward: w_K <- L_KK^{-1} (w_K - sum L_KJ w_J)
    if (blockIdx.x == 0) {
        if (threadIdx.x < nb) xs[threadIdx.x] = w[threadIdx.x];
        __syncthreads();
        tile_gemv(B.invL, xs, ys, 1);
        __syncthreads();
        if (threadIdx.x < nb) w[threadIdx.x] = ys[threadIdx.x];
    }
    grid_barrier(bar, err);
    for (int K = 0; K < NB - 1; K++) {
        int nI = min(Bb, NB - 1 - K);
        for (int a = blockIdx.x; a < nI; a += gridDim.x) {
            int I = K + 1 + a;
            if (threadIdx.x < nb) xs[threadIdx.x] = w[(int64_t)K * nb + threadIdx.x];
            __syncthreads();
            tile_gemv(tile_ptr(B, I, K), xs, w + (int64_t)I * nb, 0);
            __syncthreads();
            if (a == 0) {
                if (threadIdx.x < nb) xs[threadIdx.x] = w[(int64_t)I * nb + threadIdx.x];
                __syncthreads();
                tile_gemv(B.invL + I * t2, xs, ys, 1);
                __syncthreads();
                if (threadIdx.x < nb) w[(int64_t)I * nb + threadIdx.x] = ys[threadIdx.x];
            }
            __syncthreads();
        }
        grid_barrier(bar, err);
    }
    // backward: w_K <- U_KK^{-1} (w_K - sum U_KJ w_J)
    if (blockIdx.x == 0) {
        int K = NB - 1;
        if (threadIdx.x < nb) xs[threadIdx.x] = w[(int64_t)K * nb + threadIdx.x];
        __syncthreads();
        tile_gemv(B.invU + K * t2, xs, ys, 1);
        __syncthreads();
        if (threadIdx.x < nb) w[(int64_t)K * nb + threadIdx.x] = ys[threadIdx.x];
    }
    grid_barrier(bar, err);
    for (int K = NB - 1; K > 0; K--) {
        int nI = min(Bb, K);
        for (int a = blockIdx.x; a < nI; a += gridDim.x) {
            int I = K - 1 - a;
            if (threadIdx.x < nb) xs[threadIdx.x] = w[(int64_t)K * nb + threadIdx.x];
            __syncthreads();
            tile_gemv(tile_ptr(B, I, K), xs, w + (int64_t)I * nb, 0);
            __syncthreads();
            if (a == 0) {
                if (threadIdx.x < nb) xs[threadIdx.x] = w[(int64_t)I * nb + threadIdx.x];
                __syncthreads();
                tile_gemv(B.invU + I * t2, xs, ys, 1);
                __syncthreads();
                if (threadIdx.x < nb) w[(int64_t)I * nb + threadIdx.x] = ys[threadIdx.x];
            }
            __syncthreads();
        }
        grid_barrier(bar, err);
    }
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

// sum of squares of a and b in fixed order (single block) -> out[0], out[1]
__global__ void k_norms2(const double *a, const double *b, int64_t n, double *out) {
    __shared__ double sa[1024], sb[1024];
    int t = threadIdx.x, T = blockDim.x;
    int64_t chunk = (n + T - 1) / T, lo = t * chunk, hi = min(n, lo + chunk);
    double xa = 0.0, xb = 0.0;
    for (int64_t k = lo; k < hi; k++) {
        xa = fma(a[k], a[k], xa);
        xb = fma(b[k], b[k], xb);
    }
    sa[t] = xa;
    sb[t] = xb;
    __syncthreads();
    for (int off = T / 2; off > 0; off >>= 1) {
        if (t < off) {
            sa[t] += sa[t + off];
            sb[t] += sb[t + off];
        }
        __syncthreads();
    }
    if (t == 0) {
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
    B.invL = sys.invL;
    B.invU = sys.invU;
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
    size_t t2 = (size_t)NB_TILE * NB_TILE * sizeof(double);
    cudaError_t e = cudaMalloc(&sys.tiles, tiles_bytes(sys));
    if (e == cudaSuccess) e = cudaMalloc(&sys.invL, sys.NB * t2);
    if (e == cudaSuccess) e = cudaMalloc(&sys.invU, sys.NB * t2);
    if (e == cudaSuccess) e = cudaMalloc(&sys.rscale, np * 8);
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

int band_free(BandSystem &sys) {
    void *ps[] = {sys.tiles, sys.invL, sys.invU, sys.rscale, sys.rhs, sys.x, sys.r,
                  sys.d, sys.ell_vals, sys.ell_cols, sys.ell_prev, sys.changed,
                  sys.bar, sys.err};
    for (void *p : ps)
        if (p) cudaFree(p);
    sys = BandSystem();
    return EREBUS_OK;
}

int band_zero(erebus_state *s, BandSystem &sys) {
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

static int lu_error(erebus_state *s, BandSystem &sys, const char *what) {
    int h = 0;
    int rc = check_cuda(s, cudaMemcpyAsync(&h, sys.err, sizeof(int), cudaMemcpyDeviceToHost,
                                           s->stream), what);
    if (rc) return rc;
    rc = check_cuda(s, cudaStreamSynchronize(s->stream), what);
    if (rc) return rc;
    if (h) {
        s->last_error = std::string(what) +
                        (h == 1 ? ": grid barrier timed out" : ": zero pivot");
        cudaMemsetAsync(sys.err, 0, sizeof(int), s->stream);
        return h == 1 ? EREBUS_ECUDA : EREBUS_ENOCONV;
    }
    return EREBUS_OK;
}

int band_factor(erebus_state *s, BandSystem &sys) {
    size_t smem = 3 * NB_TILE * NB_TILE * sizeof(double);
    cudaFuncSetAttribute(k_band_factor, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    int want = sys.Bb * sys.Bb > 2 * sys.Bb ? sys.Bb * sys.Bb : 2 * sys.Bb;
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
    int rc = check_cuda(s, cudaLaunchCooperativeKernel((const void *)k_band_factor, blocks,
                                                       LU_THREADS, args, smem, s->stream),
                        "band_factor launch");
    s->launches++;
    if (rc) return rc;
    sys.factored = true;
    sys.factorizations++;
    return EREBUS_OK;
}

static int band_solve_inplace(erebus_state *s, BandSystem &sys, double *w) {
    int blocks = coop_blocks(s, (const void *)k_band_solve, LU_THREADS, 0, sys.Bb);
    BandView B = band_view(sys);
    unsigned int *bar = sys.bar;
    int *err = sys.err;
    void *args[] = {&B, &w, &bar, &err};
    cudaMemsetAsync(sys.bar, 0, 4 * sizeof(unsigned int), s->stream);
    int rc = check_cuda(s, cudaLaunchCooperativeKernel((const void *)k_band_solve, blocks,
                                                       LU_THREADS, args, 0, s->stream),
                        "band_solve launch");
    s->launches++;
    return rc;
}

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
    cudaMemcpyAsync(sys.x, sys.rhs, np * 8, cudaMemcpyDeviceToDevice, s->stream);
    rc = band_solve_inplace(s, sys, sys.x);
    if (rc) return rc;
    double rel = 0.0;
    int it = 0;
    for (;;) {
        EREBUS_LAUNCH(s, k_band_residual, nblocks(np), kThreads, 0, B, sys.x, sys.r);
        EREBUS_LAUNCH(s, k_norms2, 1, 1024, 0, sys.r, sys.rhs, np, &s->dsc->norms[0]);
        rc = check_cuda(s, cudaMemcpyAsync(&s->hsc->norms[0], &s->dsc->norms[0], 16,
                                           cudaMemcpyDeviceToHost, s->stream), "norms");
        if (rc) return rc;
        rc = lu_error(s, sys, "band LU");
        if (rc) return rc;
        double rr = s->hsc->norms[0], bb = s->hsc->norms[1];
        rel = bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
        if (!(rel > rtol) || it >= max_ir) break;
        cudaMemcpyAsync(sys.d, sys.r, np * 8, cudaMemcpyDeviceToDevice, s->stream);
        rc = band_solve_inplace(s, sys, sys.d);
        if (rc) return rc;
        EREBUS_LAUNCH(s, k_axpy, nblocks(np), kThreads, 0, sys.x, sys.d, np);
        it++;
    }
    timer_end(s, sys.ph_solve);
    if (st) {
        st->iterations = it;
        st->converged = rel <= rtol;
        st->rel_residual = rel;
    }
    if (!(rel <= rtol) && !(rel < 1e-6)) {
        s->last_error = "linear solve did not reach tolerance";
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
