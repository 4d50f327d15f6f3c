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
// timeout sets *err and returns.  Thread 0 of each CTA arrives with an
// acquire-release add after the CTA barrier (the release carries the whole
// CTA's earlier writes), the last arrival bumps the generation with a
// release, and the others spin on it with acquire loads: 2.05 us per barrier
// over 296 CTAs on a B200, against 2.45-2.7 us with full fences around
// relaxed atomics (a two-level arrival tree measured 2.8 us: the cost is
// round trips, not contention on the counter).
static __device__ void grid_barrier(unsigned int *bar, int *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int gen, arrived;
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(gen) : "l"(bar + 1) : "memory");
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                     : "=r"(arrived)
                     : "l"(bar)
                     : "memory");
        if (arrived == gridDim.x - 1) {
            asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(bar), "r"(0u) : "memory");
            asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar + 1) : "memory");
        } else {
            const unsigned long long t0 = globaltimer();
            for (;;) {
                unsigned int g;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];"
                             : "=r"(g)
                             : "l"(bar + 1)
                             : "memory");
                if (g != gen) break;
                if (globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
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

// In-place Gauss-Jordan inverse (no pivoting) of the tile held in registers
// `a` (FFMA layout), eliminating two unknowns per step with the inverse of
// their 2 x 2 pivot block: for pivot rows/columns K = {k, k+1},
//   A_ij -= A_iK P^{-1} A_Kj,  A_iK <- -A_iK P^{-1},  A_Kj <- P^{-1} A_Kj,
//   A_KK <- P^{-1}.
// One barrier per step (32 steps); `vec` holds 2 x 4 x 64 doubles.  A zero
// or non-finite pivot determinant raises *err = 2.
static __device__ void tile_inverse2(double a[4][4], double *vec, int *err) {
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll
    for (int kq = 0; kq < 4; kq++)
        for (int kk = 0; kk < 16; kk += 2) {
            const int k = kq * 16 + kk;
            double *buf = vec + ((k >> 1) & 1) * 4 * NB_TILE;
            double *col0 = buf, *col1 = buf + NB_TILE, *row0 = buf + 2 * NB_TILE,
                   *row1 = buf + 3 * NB_TILE;
            if (tx == kk || tx == kk + 1) {
                double *cd = tx == kk ? col0 : col1;
#pragma unroll
                for (int i = 0; i < 4; i++) cd[ty + 16 * i] = a[i][kq];
            }
            if (ty == kk || ty == kk + 1) {
                double *rd = ty == kk ? row0 : row1;
#pragma unroll
                for (int j = 0; j < 4; j++) rd[tx + 16 * j] = a[kq][j];
            }
            __syncthreads();
            const double p00 = row0[k], p01 = row0[k + 1], p10 = row1[k], p11 = row1[k + 1];
            const double det = p00 * p11 - p01 * p10;
            if (threadIdx.x == 0 && !(fabs(det) > 0.0 && fabs(det) < INFINITY)) atomicExch(err, 2);
            const double id = 1.0 / det;
            const double q00 = p11 * id, q01 = -p01 * id, q10 = -p10 * id, q11 = p00 * id;
            double u0[4], u1[4], r0[4], r1[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                double c0 = col0[ty + 16 * i], c1 = col1[ty + 16 * i];
                u0[i] = c0 * q00 + c1 * q10;
                u1[i] = c0 * q01 + c1 * q11;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                r0[j] = row0[tx + 16 * j];
                r1[j] = row1[tx + 16 * j];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    a[i][j] = fma(-u0[i], r0[j], fma(-u1[i], r1[j], a[i][j]));
            // pivot columns, then pivot rows, then the pivot block
            if (tx == kk || tx == kk + 1) {
#pragma unroll
                for (int i = 0; i < 4; i++) a[i][kq] = tx == kk ? -u0[i] : -u1[i];
            }
            if (ty == kk || ty == kk + 1) {
#pragma unroll
                for (int j = 0; j < 4; j++)
                    a[kq][j] = ty == kk ? q00 * r0[j] + q01 * r1[j] : q10 * r0[j] + q11 * r1[j];
                if (tx == kk || tx == kk + 1)
                    a[kq][kq] = ty == kk ? (tx == kk ? q00 : q01) : (tx == kk ? q10 : q11);
            }
        }
    __syncthreads();
}

struct FactorSmem {
    double As[STILE], Bt[STILE], Cs[STILE];
    double vec[2 * 2 * NB_TILE];
};

// ---------------------------------------------------------------------------
// FP64 tensor-core tile products (mma.sync m16n8k16 .f64)
//
// A 64 x 64 result tile is held in registers by the 8 warps of the CTA:
// warp w owns rows 32 (w & 1) .. +32 and columns 16 (w >> 1) .. +16 as
// 2 x 2 fragments of 16 x 8; fragment element q of thread (g = lane / 4,
// t = lane % 4) is row g + 8 (q / 2), column 2 t + q % 2.  Operand tiles
// stream through shared memory in K-chunks of 32 with cp.async (16-byte
// copies that bypass L1, so data other CTAs wrote is read from L2), three
// stages deep: A chunks column-major with leading dimension 68, B chunks
// column-major with leading dimension 36, both chosen so that the fragment
// loads of a warp hit every bank pair exactly twice.
// ---------------------------------------------------------------------------
constexpr int MMA_LA = 68, MMA_LB = 36, MMA_KC = 32, MMA_NSTAGE = 3;
constexpr int MMA_STAGE = MMA_KC * MMA_LA + NB_TILE * MMA_LB;   // doubles per stage

struct MmaSmem {
    double stage[MMA_NSTAGE][MMA_STAGE];
    double vec[2 * 4 * NB_TILE];   // pivot rows/columns of tile_inverse2, double-buffered
};
static_assert(MMA_STAGE >= STILE, "a stage holds a padded tile");

typedef double MmaAcc[2][2][4];

static __device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
static __device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
                 : "memory");
}
static __device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
static __device__ __forceinline__ void cp_async_wait1() {
    asm volatile("cp.async.wait_group 1;" ::: "memory");
}
static __device__ __forceinline__ void cp_async_wait0() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Copies K-chunk h (columns 32 h .. 32 h + 31 of A, rows of B) of the
// column-major 64 x 64 tiles A and B into stage `st`.
static __device__ __forceinline__ void mma_load_chunk(double *st, const double *A, const double *B,
                                                      int h) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int e = threadIdx.x + 256 * q;
        int col = e >> 5, rp = (e & 31) * 2;
        cp_async16(st + col * MMA_LA + rp, A + (h * MMA_KC + col) * NB_TILE + rp);
    }
    double *sb = st + MMA_KC * MMA_LA;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int e = threadIdx.x + 256 * q;
        int c = e >> 4, kp = (e & 15) * 2;
        cp_async16(sb + c * MMA_LB + kp, B + c * NB_TILE + h * MMA_KC + kp);
    }
}

static __device__ __forceinline__ void mma_16816(double c[4], const double a[8], const double b[4]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
        "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]),
          "d"(a[7]), "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// acc += (chunk's A part) * (chunk's B part)
static __device__ __forceinline__ void mma_chunk(const double *st, MmaAcc acc) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int rb = (w & 1) * 32, cb = (w >> 1) * 16;
    const double *sa = st, *sb = st + MMA_KC * MMA_LA;
#pragma unroll
    for (int ks = 0; ks < MMA_KC; ks += 16) {
        double a[2][8], b[2][4];
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int i = 0; i < 8; i++)
                a[mi][i] = sa[(ks + t + 4 * (i >> 1)) * MMA_LA + rb + mi * 16 + g + 8 * (i & 1)];
#pragma unroll
        for (int ni = 0; ni < 2; ni++)
#pragma unroll
            for (int i = 0; i < 4; i++) b[ni][i] = sb[(cb + ni * 8 + g) * MMA_LB + ks + t + 4 * i];
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int ni = 0; ni < 2; ni++) mma_16816(acc[mi][ni], a[mi], b[ni]);
    }
}

// acc += sum_{p < np} tileA(p) * tileB(p) (global column-major tiles),
// three-stage cp.async pipeline.  Ends with the stages free.
// `pre()` runs once the first copies are in flight (e.g. loading the
// accumulator), so its latency overlaps theirs.
template <class TA, class TB, class Pre>
static __device__ void mma_tiles(MmaSmem &S, int np, TA tileA, TB tileB, MmaAcc acc, Pre pre) {
    const int nq = 2 * np;
#pragma unroll 1
    for (int q = 0; q < 2; q++) {
        if (q < nq) mma_load_chunk(S.stage[q], tileA(q >> 1), tileB(q >> 1), q & 1);
        cp_async_commit();
    }
    pre();
#pragma unroll 1
    for (int q = 0; q < nq; q++) {
        cp_async_wait1();
        __syncthreads();
        if (q + 2 < nq)
            mma_load_chunk(S.stage[(q + 2) % MMA_NSTAGE], tileA((q + 2) >> 1), tileB((q + 2) >> 1),
                           (q + 2) & 1);
        cp_async_commit();
        mma_chunk(S.stage[q % MMA_NSTAGE], acc);
    }
    cp_async_wait0();
    __syncthreads();
}

// fragment element (mi, ni, q) -> (row, column) of the tile
static __device__ __forceinline__ int frag_row(int mi, int q) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    return (w & 1) * 32 + mi * 16 + (lane >> 2) + 8 * (q >> 1);
}
static __device__ __forceinline__ int frag_col(int ni, int q) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    return (w >> 1) * 16 + ni * 8 + 2 * (lane & 3) + (q & 1);
}
template <class A>
static __device__ __forceinline__ void frag_zero(A acc[2][2][4]) {
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 2; ni++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[mi][ni][q] = A(0);
}
// acc = sign * C (global column-major tile, read through L2)
template <class T, class A>
static __device__ __forceinline__ void frag_load(const T *C, A acc[2][2][4], A sign) {
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 2; ni++)
#pragma unroll
            for (int q = 0; q < 4; q++)
                acc[mi][ni][q] = sign * (A)__ldcg(&C[frag_col(ni, q) * NB_TILE + frag_row(mi, q)]);
}
template <class T, class A>
static __device__ __forceinline__ void frag_store(T *C, const A acc[2][2][4], A sign) {
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 2; ni++)
#pragma unroll
            for (int q = 0; q < 4; q++)
                C[frag_col(ni, q) * NB_TILE + frag_row(mi, q)] = (T)(sign * acc[mi][ni][q]);
}
// fragments -> shared-memory FP64 tile (column-major, ld LDS)
template <class A>
static __device__ __forceinline__ void frag_to_smem(double *T, const A acc[2][2][4], double sign) {
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 2; ni++)
#pragma unroll
            for (int q = 0; q < 4; q++)
                T[frag_col(ni, q) * LDS + frag_row(mi, q)] = sign * (double)acc[mi][ni][q];
}

// ---------------------------------------------------------------------------
// FP32 tiles (mixed-precision factor): 64 x 64 float tiles, products on the
// tensor cores with three TF32 products per FP32 product (x = hi + lo with
// hi, lo TF32; a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi), which keeps about
// FP32 accuracy; accumulation in FP32.  A stage holds a whole tile pair:
// A column-major with leading dimension 72, B column-major with leading
// dimension 68 (fragment loads hit every bank once); the same bytes as an
// FP64 stage.
// ---------------------------------------------------------------------------
constexpr int MMAF_LA = 72, MMAF_LB = 68;
static_assert((NB_TILE * MMAF_LA + NB_TILE * MMAF_LB) * 4 <= MMA_STAGE * 8, "float stage fits");
typedef float MmaAccF[2][2][4];

static __device__ __forceinline__ void mma_load_pair_f(float *st, const float *A, const float *B) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int e = threadIdx.x + 256 * q;
        int col = e >> 4, rq = (e & 15) * 4;
        cp_async16(st + col * MMAF_LA + rq, A + col * NB_TILE + rq);
    }
    float *sb = st + NB_TILE * MMAF_LA;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int e = threadIdx.x + 256 * q;
        int c = e >> 4, kq = (e & 15) * 4;
        cp_async16(sb + c * MMAF_LB + kq, B + c * NB_TILE + kq);
    }
}

static __device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo) {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
    float r = x - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}
static __device__ __forceinline__ void mma_tf32(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// acc += (pair's A) * (pair's B), K = 64 in steps of 8
static __device__ __forceinline__ void mma_pair_f(const float *st, MmaAccF acc) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int rb = (w & 1) * 32, cb = (w >> 1) * 16;
    const float *sa = st, *sb = st + NB_TILE * MMAF_LA;
#pragma unroll 2
    for (int ks = 0; ks < NB_TILE; ks += 8) {
        uint32_t ah[2][4], al[2][4], bh[2][2], bl[2][2];
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int i = 0; i < 4; i++)
                tf32_split(sa[(ks + t + 4 * (i >> 1)) * MMAF_LA + rb + mi * 16 + g + 8 * (i & 1)],
                           ah[mi][i], al[mi][i]);
#pragma unroll
        for (int ni = 0; ni < 2; ni++)
#pragma unroll
            for (int i = 0; i < 2; i++)
                tf32_split(sb[(cb + ni * 8 + g) * MMAF_LB + ks + t + 4 * i], bh[ni][i], bl[ni][i]);
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int ni = 0; ni < 2; ni++) {
                mma_tf32(acc[mi][ni], al[mi], bh[ni]);
                mma_tf32(acc[mi][ni], ah[mi], bl[ni]);
                mma_tf32(acc[mi][ni], ah[mi], bh[ni]);
            }
    }
}

// acc += sum_{p < np} tileA(p) * tileB(p) for float tiles; three-stage
// cp.async pipeline over the tile pairs; `pre()` as in mma_tiles.
template <class TA, class TB, class Pre>
static __device__ void mma_tiles(MmaSmem &S, int np, TA tileA, TB tileB, MmaAccF acc, Pre pre) {
#pragma unroll 1
    for (int q = 0; q < 2; q++) {
        if (q < np) mma_load_pair_f(reinterpret_cast<float *>(S.stage[q]), tileA(q), tileB(q));
        cp_async_commit();
    }
    pre();
#pragma unroll 1
    for (int q = 0; q < np; q++) {
        cp_async_wait1();
        __syncthreads();
        if (q + 2 < np)
            mma_load_pair_f(reinterpret_cast<float *>(S.stage[(q + 2) % MMA_NSTAGE]),
                            tileA(q + 2), tileB(q + 2));
        cp_async_commit();
        mma_pair_f(reinterpret_cast<const float *>(S.stage[q % MMA_NSTAGE]), acc);
    }
    cp_async_wait0();
    __syncthreads();
}

// float tile (global, column-major) <-> FP64 shared-memory tile (ld LDS)
static __device__ __forceinline__ void stage_tile(double *dst, const float *src) {
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
    float4 v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) v[q] = __ldcg(&s4[threadIdx.x + 256 * q]);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int e = 4 * (threadIdx.x + 256 * q), r = e % NB_TILE, c = e / NB_TILE;
        dst[c * LDS + r] = v[q].x;
        dst[c * LDS + r + 1] = v[q].y;
        dst[c * LDS + r + 2] = v[q].z;
        dst[c * LDS + r + 3] = v[q].w;
    }
}
static __device__ __forceinline__ void unstage_tile(float *dst, const double *src) {
    float4 *d4 = reinterpret_cast<float4 *>(dst);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        int e = 4 * (threadIdx.x + 256 * q), r = e % NB_TILE, c = e / NB_TILE;
        d4[threadIdx.x + 256 * q] =
            make_float4((float)src[c * LDS + r], (float)src[c * LDS + r + 1],
                        (float)src[c * LDS + r + 2], (float)src[c * LDS + r + 3]);
    }
}

}  // namespace erebus
