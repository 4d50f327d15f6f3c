// tiles.cuh -- 64 x 64 FP64 tile primitives shared by the dense LU kernels
// (the block-banded LU of bandlu.cu and the multifrontal LU of mfront.cu),
// and the bounded grid barrier of their persistent cooperative kernels.
#pragma once
#include "solver.cuh"

namespace erebus {

constexpr int NB_TILE = 64;       // tile size
constexpr int LU_THREADS = 256;
constexpr unsigned long long BARRIER_TIMEOUT_NS = 2000000000ull;   // 2 s

static __device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Sense-reversing grid barrier over all CTAs of a cooperative launch.
// bar[0] = arrival count, bar[1] = generation.  A wait that exceeds the
// timeout sets *err and returns.
static __device__ void grid_barrier(unsigned int *bar, int *err) {
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
// tile primitives (one CTA of 256 threads, 64 x 64 FP64 tiles)
//
// Register layout of a tile held by the CTA: thread (ty, tx) = (tid/16,
// tid%16) owns rows r = ty + 16 i and columns c = tx + 16 j, i, j = 0..3.
// Shared-memory tiles are column-major with leading dimension LDS = 65
// (conflict-free staging).  Data another CTA wrote during this kernel is
// read with ld.global.cg (L2), never through the non-coherent L1.
// ---------------------------------------------------------------------------
constexpr int LDS = NB_TILE + 1;
constexpr int STILE = NB_TILE * LDS;            // doubles per staged tile

static __device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// global column-major tile -> smem column-major (ld LDS)
static __device__ __forceinline__ void stage_tile(double *dst, const double *src) {
    const double2 *s2 = reinterpret_cast<const double2 *>(src);
    double2 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = __ldcg(&s2[threadIdx.x + 256 * q]);
#pragma unroll
    for (int q = 0; q < 8; q++) {
        int e = 2 * (threadIdx.x + 256 * q), r = e % NB_TILE, c = e / NB_TILE;
        dst[c * LDS + r] = v[q].x;
        dst[c * LDS + r + 1] = v[q].y;
    }
}
// global column-major tile -> smem transposed (Bt[k*LDS + c] = B(k, c))
static __device__ __forceinline__ void stage_tile_t(double *dst, const double *src) {
    const double2 *s2 = reinterpret_cast<const double2 *>(src);
    double2 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = __ldcg(&s2[threadIdx.x + 256 * q]);
#pragma unroll
    for (int q = 0; q < 8; q++) {
        int e = 2 * (threadIdx.x + 256 * q), k = e % NB_TILE, c = e / NB_TILE;
        dst[k * LDS + c] = v[q].x;
        dst[(k + 1) * LDS + c] = v[q].y;
    }
}
// smem column-major (ld LDS) -> global column-major
static __device__ __forceinline__ void unstage_tile(double *dst, const double *src) {
    double2 *d2 = reinterpret_cast<double2 *>(dst);
#pragma unroll
    for (int q = 0; q < 8; q++) {
        int e = 2 * (threadIdx.x + 256 * q), r = e % NB_TILE, c = e / NB_TILE;
        d2[threadIdx.x + 256 * q] = make_double2(src[c * LDS + r], src[c * LDS + r + 1]);
    }
}
static __device__ __forceinline__ void regs_from_smem(const double *S, double a[4][4]) {
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) a[i][j] = S[(tx + 16 * j) * LDS + ty + 16 * i];
}
static __device__ __forceinline__ void regs_to_smem(double *S, const double a[4][4]) {
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) S[(tx + 16 * j) * LDS + ty + 16 * i] = a[i][j];
}
// acc (+)= A * B with As column-major (ld LDS) and Bt transposed (ld LDS)
static __device__ __forceinline__ void gemm_acc(const double *As, const double *Bt, double acc[4][4]) {
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll 4
    for (int k = 0; k < NB_TILE; k++) {
        double av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) av[i] = As[k * LDS + ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; j++) bv[j] = Bt[k * LDS + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
}

// In-place Gauss-Jordan inverse (no pivoting) of the tile held in registers
// `a` (the layout above): step k publishes column k and row k, then every
// thread updates its 16 elements branch-free; one barrier per step
// (broadcast vectors double-buffered).  A zero or non-finite pivot raises
// *err = 2.
static __device__ void tile_inverse(double a[4][4], double *vec, int *err) {
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll
    for (int kq = 0; kq < 4; kq++)
        for (int kk = 0; kk < 16; kk++) {
            const int k = kq * 16 + kk;
            double *col = vec + (k & 1) * 2 * NB_TILE, *row = col + NB_TILE;
            if (tx == kk) {
#pragma unroll
                for (int i = 0; i < 4; i++) col[ty + 16 * i] = a[i][kq];
            }
            if (ty == kk) {
#pragma unroll
                for (int j = 0; j < 4; j++) row[tx + 16 * j] = a[kq][j];
            }
            __syncthreads();
            double piv = row[k];
            if (threadIdx.x == 0 && !(fabs(piv) > 0.0 && fabs(piv) < INFINITY)) atomicExch(err, 2);
            double ip = 1.0 / piv;
            double f[4], rk[4];
#pragma unroll
            for (int i = 0; i < 4; i++) f[i] = col[ty + 16 * i] * ip;
#pragma unroll
            for (int j = 0; j < 4; j++) rk[j] = row[tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) a[i][j] = fma(-f[i], rk[j], a[i][j]);
            // column k (rows != k), then row k, then the pivot
            if (tx == kk) {
#pragma unroll
                for (int i = 0; i < 4; i++) a[i][kq] = -f[i];
            }
            if (ty == kk) {
#pragma unroll
                for (int j = 0; j < 4; j++) a[kq][j] = rk[j] * ip;
                if (tx == kk) a[kq][kq] = ip;
            }
        }
    __syncthreads();
}

struct FactorSmem {
    double As[STILE], Bt[STILE], Cs[STILE];
    double vec[2 * 2 * NB_TILE];
};

}  // namespace erebus
