// mfront.cu -- nested-dissection multifrontal LU of the row-scaled systems.
//
// The reference factorises each system with a sparse direct LU (UMFPACK,
// E:6612, E:6736-6748, E:6925).  Here the unknowns are ordered by nested
// dissection of the P-node grid (mf_plan.h) and the LU runs front by front,
// level by level from the leaves to the root, without pivoting:
//
//   assembly   the scaled ELL entries are stored into the fronts that
//              eliminate them (k_mf_scatter), padding unknowns become
//              identity rows (k_mf_pad);
//   factor     (k_mf_factor, one persistent cooperative kernel) per level:
//              extend-add of the children's Schur complements, then for each
//              64-column block K of the eliminated part the inverse of the
//              diagonal tile D_K (Gauss-Jordan), L_IK = A_IK D_K^{-1}, and
//              the rank-64 update of the eliminated rows and columns; last
//              the Schur complement of the update block with inner dimension
//              Kp (tile products on the FP64 tensor cores, operands streamed
//              through a cp.async pipeline);
//   solve      (k_mf_solve) forward over the levels from the leaves, backward
//              from the root; each front gathers its children's update
//              vectors and its ring solution through index maps.
//
// Levels with many small fronts run one front per CTA with no grid barrier
// inside; levels with few large fronts spread each step's tile tasks over
// all CTAs, separated by the bounded grid barrier.  Results do not depend
// on the number of CTAs: every tile is computed by one CTA in a fixed order.
#include <cooperative_groups.h>

#include <type_traits>
#include <vector>

#include "mf_plan.h"
#include "mf_tasks.h"
#include "solver.cuh"
#include "tiles.cuh"

namespace erebus {

constexpr int T2 = NB_TILE * NB_TILE;
static_assert(MF_TILE == NB_TILE, "front tiles are the LU tiles");

struct MfView {
    const MfFront *fr;
    void *F;            // front storage (double, or float for the mixed-precision factor)
    double *vec;        // front vectors (solve)
    const int *vars;    // local -> global unknown
    const int *eamap;   // local -> children's update index
    const int *lvl;     // level ranges (nlev + 1)
    const int *lvl_kt;  // max Kt per level
    const int *lvl_mode;  // per level: MF_FACTOR_LOCAL, MF_SOLVE_LOCAL, ... bits
    int *flags;         // per 64-row block of the front vectors: the solve epoch it is final in
    int *done;          // per front (at its first row block), F1 and B1 tasks counted done
    double *vec2;       // pivot part of the forward solution (levels with inverted pivot blocks)
    double *part;       // partial sums of the backward ring products (MfFront::poff)
    int inv;            // cooperative solve levels hold inverted pivot blocks
    int nlev;
    const long long *target;   // ELL entry -> storage offset
    const int *expect;         // ELL column pattern the targets were built from
    long long n;
    int ell;
};

struct MfDevice {
    MfPlan plan;
    bool fp32 = false;   // the current factors are the float ones
    bool solve32 = false;   // solves read F32, an FP32 copy of the FP64 factors in F64
    MfFront *fr = nullptr;
    void *F64 = nullptr, *F32 = nullptr;   // front storage of each precision, on first use
    double *vec = nullptr;
    int *vars = nullptr, *eamap = nullptr, *lvl = nullptr, *lvl_kt = nullptr;
    int *lvl_mode = nullptr;
    int *flags = nullptr;   // row-block flags of the cooperative solve levels
    int *done = nullptr;    // per-front counts of the inverted form's F1 and B1 tasks
    int epoch = 0;          // solves launched so far
    // inverted pivot blocks of the cooperative solve levels
    bool inv = false;
    double *vec2 = nullptr, *part = nullptr;
    int2 *inv_list = nullptr;   // (front, Kt) of the fronts k_mf_invert works on
    int n_inv = 0, inv_ktmax = 0;
    longlong2 *cvt = nullptr;   // storage ranges the FP32 copy converts
    int n_cvt = 0;
    long long *target = nullptr;
    int *expect = nullptr;
    int nlev = 0;
};

template <class T>
__device__ __forceinline__ T *ftile(const MfView &V, const MfFront &f, int I, int J) {
    return (T *)V.F + f.off + ((long long)J * f.Mt + I) * T2;
}
// accumulator fragments of a tile product with T-valued tiles
template <class T> struct MfAccT { typedef double type[2][2][4]; };
template <> struct MfAccT<float> { typedef float type[2][2][4]; };
__device__ __forceinline__ long long felem(const MfFront &f, int a, int b) {
    return f.off + ((long long)(b >> 6) * f.Mt + (a >> 6)) * T2 + (b & 63) * 64 + (a & 63);
}

// ---------------------------------------------------------------------------
// assembly
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_mf_scatter(MfView V, const int *cols, const double *vals, int *err) {
    long long row = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= V.n) return;
    for (int s = 0; s < V.ell; s++) {
        long long e = row * V.ell + s;
        int c = cols[e];
        if (c != V.expect[e]) {
            atomicExch(err, 4);
            continue;
        }
        long long t = V.target[e];
        if (t >= 0) ((T *)V.F)[t] += (T)vals[e];
    }
}

template <class T>
__global__ void k_mf_pad(MfView V, int nfronts) {
    int f = blockIdx.x;
    if (f >= nfronts) return;
    MfFront fr = V.fr[f];
    for (int a = fr.k + threadIdx.x; a < fr.Kp; a += blockDim.x) ((T *)V.F)[felem(fr, a, a)] = T(1);
}

// ---------------------------------------------------------------------------
// factor: CTA-wide tile operations (256 threads)
// ---------------------------------------------------------------------------

// Tile (I, J) of front f += the children's Schur complement entries that
// map onto it (child 0 first, then child 1).  The tile's row and column maps
// are staged in shared memory; a child that maps onto no row or no column
// of the tile is skipped, and so is the whole tile when neither child does.
template <class T>
__device__ void mf_extend_add_tile(const MfView &V, const MfFront &f, int I, int J,
                                   int (*emap)[64]) {
    const int *map = V.eamap + f.map_off;
    const int tid = threadIdx.x;
    if (tid < 128) {
        int a = (tid < 64 ? I : J) * 64 + (tid & 63);
        emap[tid < 64 ? 0 : 2][tid & 63] = __ldg(&map[2 * a]);
        emap[tid < 64 ? 1 : 3][tid & 63] = __ldg(&map[2 * a + 1]);
    }
    __syncthreads();
    const bool h0 = f.c0 >= 0, h1 = f.c1 >= 0;
    const int lane64 = tid & 63, which = tid >> 6;   // 4 groups of 64 threads
    int any = which < 4 && emap[which][lane64] >= 0;
    int r0 = __syncthreads_or(which == 0 && any), c0 = __syncthreads_or(which == 2 && any);
    int r1 = __syncthreads_or(which == 1 && any), c1 = __syncthreads_or(which == 3 && any);
    const bool u0 = h0 && r0 && c0, u1 = h1 && r1 && c1;
    if (u0 || u1) {
        T *Tt = ftile<T>(V, f, I, J);
        const T *F = (const T *)V.F;
        MfFront C0, C1;
        if (u0) C0 = V.fr[f.c0];
        if (u1) C1 = V.fr[f.c1];
        // all loads of a batch are issued before any store (the stores could
        // alias the children's storage as far as the compiler knows)
#pragma unroll 1
        for (int q0 = 0; q0 < 16; q0 += 8) {
            T t[8], x0[8], x1[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                int e = tid + 256 * (q0 + q), r = e & 63, c = e >> 6;
                t[q] = __ldcg(&Tt[c * 64 + r]);
                x0[q] = T(0);
                x1[q] = T(0);
                if (u0) {
                    int ia = emap[0][r], ib = emap[2][c];
                    if (ia >= 0 && ib >= 0) x0[q] = __ldcg(F + felem(C0, C0.Kp + ia, C0.Kp + ib));
                }
                if (u1) {
                    int ia = emap[1][r], ib = emap[3][c];
                    if (ia >= 0 && ib >= 0) x1[q] = __ldcg(F + felem(C1, C1.Kp + ia, C1.Kp + ib));
                }
            }
#pragma unroll
            for (int q = 0; q < 8; q++) {
                int e = tid + 256 * (q0 + q), r = e & 63, c = e >> 6;
                Tt[c * 64 + r] = (t[q] + x0[q]) + x1[q];
            }
        }
    }
    __syncthreads();
}

// Inverts tile T in place (Gauss-Jordan in FP64 registers, FFMA layout).
template <class T>
__device__ void mf_invert_tile(T *Tt, MmaSmem &S, int *err) {
    double a[4][4];
    double *P = S.stage[0];
    stage_tile(P, Tt);
    __syncthreads();
    regs_from_smem(P, a);
    __syncthreads();
    tile_inverse(a, S.vec, err);
    regs_to_smem(P, a);
    __syncthreads();
    unstage_tile(Tt, P);
    __syncthreads();
}

// L_IK = A_IK D_K^{-1} (tile (K,K) holds D_K^{-1})
template <class T>
__device__ void mf_l_tile(const MfView &V, const MfFront &f, int I, int K, MmaSmem &S) {
    typename MfAccT<T>::type acc;
    typedef typename std::remove_reference<decltype(acc[0][0][0])>::type A;
    const T *At = ftile<T>(V, f, I, K), *Bt = ftile<T>(V, f, K, K);
    mma_tiles(
        S, 1, [&](int) { return At; }, [&](int) { return Bt; }, acc, [&] { frag_zero(acc); });
    frag_store(ftile<T>(V, f, I, K), acc, A(1));
    __syncthreads();
}

// A_IJ -= sum_{K in [k0, k1)} L_IK A_KJ; optionally invert the result.
template <class T>
__device__ void mf_update_tile(const MfView &V, const MfFront &f, int I, int J, int k0,
                               int k1, MmaSmem &S, int *err, bool invert) {
    typedef typename MfAccT<T>::type Acc;
    Acc acc;
    typedef typename std::remove_reference<decltype(acc[0][0][0])>::type A;
    T *C = ftile<T>(V, f, I, J);
    mma_tiles(
        S, k1 - k0, [&](int p) { return (const T *)ftile<T>(V, f, I, k0 + p); },
        [&](int p) { return (const T *)ftile<T>(V, f, k0 + p, J); }, acc,
        [&] { frag_load(C, acc, A(-1)); });
    if (invert) {
        double a[4][4];
        double *P = S.stage[0];
        frag_to_smem(P, acc, -1.0);
        __syncthreads();
        regs_from_smem(P, a);
        __syncthreads();
        tile_inverse(a, S.vec, err);
        regs_to_smem(P, a);
        __syncthreads();
        unstage_tile(C, P);
    } else {
        frag_store(C, acc, A(-1));
    }
    __syncthreads();
}

// Fronts of a level whose tile counts a CTA keeps in shared memory; levels
// with more fronts run one front per CTA.
constexpr int MF_KM_MAX = 256;
// Bits of MfView::lvl_mode: the level runs one front per CTA in the factor /
// in the solve (else cooperatively, tile tasks dealt over all CTAs).
constexpr int MF_FACTOR_LOCAL = 1, MF_SOLVE_LOCAL = 2;
// ... and every front of the level keeps its vector in shared memory
// (M <= MF_VS_MAX), so the level's sweeps stream all of a CTA's fronts
// through one tile pipeline.
constexpr int MF_SOLVE_VS = 4;
// Cooperative solve levels whose update rows (F2) or pivot rows (B2) run in
// 8-tile chunks: set where a front has rows of more than 12 tiles and the
// chunked tasks of the phase still fit one wave of the grid (more tasks per
// CTA cost more than the shorter rows save).
constexpr int MF_CHUNK_F2 = 8, MF_CHUNK_B2 = 16;

struct MfFactorSmem {
    MmaSmem m;
    int emap[4][64];
    int2 km[MF_KM_MAX];   // (Kt, Mt) of the level's fronts
};

// Number of update tasks of step K: rows/cols K+1..Mt-1 except the block
// of update rows and update columns (deferred to the Schur phase).
__device__ __forceinline__ int mf_nupd(int Kt, int Mt, int K) {
    if (K >= Kt) return 0;
    int R = Mt - K - 1, e = Kt - K - 1;
    return e * R + (Mt - Kt) * e;
}
__device__ __forceinline__ void mf_upd_ij(const MfFront &f, int K, int u, int &I, int &J) {
    int R = f.Mt - K - 1, e = f.Kt - K - 1;
    if (u < e * R) {           // eliminated rows, all columns
        I = K + 1 + u % e;
        J = K + 1 + u / e;
    } else {                   // update rows, eliminated columns
        u -= e * R;
        int ru = f.Mt - f.Kt;
        I = f.Kt + u % ru;
        J = K + 1 + u / ru;
    }
}

// The whole partial LU of one front by one CTA.
template <class T>
__device__ void mf_factor_local(const MfView &V, const MfFront &f, MfFactorSmem &FS,
                                int *err) {
    MmaSmem &S = FS.m;
    if (f.c0 >= 0 || f.c1 >= 0) {
        for (int t = 0; t < f.Mt * f.Mt; t++)
            mf_extend_add_tile<T>(V, f, t % f.Mt, t / f.Mt, FS.emap);
        __threadfence_block();
        __syncthreads();
    }
    for (int K = 0; K < f.Kt; K++) {
        if (K == 0) mf_invert_tile(ftile<T>(V, f, 0, 0), S, err);
        for (int I = K + 1; I < f.Mt; I++) mf_l_tile<T>(V, f, I, K, S);
        int nu = mf_nupd(f.Kt, f.Mt, K);
        for (int u = 0; u < nu; u++) {
            int I, J;
            mf_upd_ij(f, K, u, I, J);
            mf_update_tile<T>(V, f, I, J, K, K + 1, S, err, I == K + 1 && J == K + 1);
        }
    }
    for (int J = f.Kt; J < f.Mt; J++)
        for (int I = f.Kt; I < f.Mt; I++) mf_update_tile<T>(V, f, I, J, 0, f.Kt, S, err, false);
}

// Runs task(f, u) for the tasks u in [0, count(Kt, Mt)) of the fronts
// [fb, fe), numbered consecutively across the fronts and dealt round-robin
// to the CTAs.  km holds (Kt, Mt) of the fronts in shared memory; a front's
// descriptor is read only when this CTA has one of its tasks.
template <class Count, class Task>
__device__ void mf_for_tasks(const MfView &V, int fb, int fe, const int2 *km, Count count,
                             Task task) {
    const int G = gridDim.x;
    // first = (blockIdx.x - tasks of the earlier fronts) mod G, kept in 32
    // bits and updated per front: every thread runs this loop over all the
    // level's fronts, so it must stay a few instructions per front
    int first = blockIdx.x;
    for (int fi = fb; fi < fe; fi++) {
        int2 q = km[fi - fb];
        int cnt = count(q.x, q.y);
        if (cnt <= 0) continue;
        if (first < cnt) {
            const MfFront f = V.fr[fi];
            for (int u = first; u < cnt; u += G) task(f, u);
        }
        first -= cnt;
        if (first < 0) first = first % G + (first % G < 0 ? G : 0);
    }
}

// (Kt, Mt) of the fronts [fb, fe) into shared memory.
__device__ __forceinline__ void mf_load_km(const MfView &V, int fb, int fe, int2 *km) {
    for (int i = threadIdx.x; i < fe - fb; i += blockDim.x) {
        const MfFront &f = V.fr[fb + i];
        km[i] = make_int2(f.Kt, f.Mt);
    }
    __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(LU_THREADS, 2)
k_mf_factor(MfView V, unsigned int *bar, int *err) {
    extern __shared__ __align__(16) double smem_raw[];
    MfFactorSmem &FS = *reinterpret_cast<MfFactorSmem *>(smem_raw);
    MmaSmem &S = FS.m;
    const int G = gridDim.x;
    for (int p = 0; p < V.nlev; p++) {
        const int fb = V.lvl[p], fe = V.lvl[p + 1];
        if (V.lvl_mode[p] & MF_FACTOR_LOCAL) {
            for (int fi = fb + blockIdx.x; fi < fe; fi += G) {
                const MfFront f = V.fr[fi];
                mf_factor_local<T>(V, f, FS, err);
            }
            grid_barrier(bar, err);
            continue;
        }
        mf_load_km(V, fb, fe, FS.km);
        // extend-add; the task of tile (0,0) also inverts it
        mf_for_tasks(
            V, fb, fe, FS.km, [](int, int Mt) { return Mt * Mt; },
            [&](const MfFront &f, int u) {
                int I = u % f.Mt, J = u / f.Mt;
                if (f.c0 >= 0 || f.c1 >= 0) mf_extend_add_tile<T>(V, f, I, J, FS.emap);
                if (u == 0 && f.Kt > 0) mf_invert_tile(ftile<T>(V, f, 0, 0), S, err);
            });
        grid_barrier(bar, err);
        const int ktmax = V.lvl_kt[p];
        for (int K = 0; K < ktmax; K++) {
            mf_for_tasks(
                V, fb, fe, FS.km, [K](int Kt, int Mt) { return K < Kt ? Mt - K - 1 : 0; },
                [&](const MfFront &f, int u) { mf_l_tile<T>(V, f, K + 1 + u, K, S); });
            grid_barrier(bar, err);
            // the last step has no update tasks in any front (mf_nupd is 0 for
            // K = Kt - 1); ktmax is the same in every CTA, so all skip it
            if (K + 1 == ktmax) break;
            mf_for_tasks(
                V, fb, fe, FS.km, [K](int Kt, int Mt) { return mf_nupd(Kt, Mt, K); },
                [&](const MfFront &f, int u) {
                    int I, J;
                    mf_upd_ij(f, K, u, I, J);
                    mf_update_tile<T>(V, f, I, J, K, K + 1, S, err, I == K + 1 && J == K + 1);
                });
            grid_barrier(bar, err);
        }
        mf_for_tasks(
            V, fb, fe, FS.km, [](int Kt, int Mt) { return (Mt - Kt) * (Mt - Kt); },
            [&](const MfFront &f, int u) {
                int ru = f.Mt - f.Kt;
                mf_update_tile<T>(V, f, f.Kt + u % ru, f.Kt + u / ru, 0, f.Kt, S, err, false);
            });
        grid_barrier(bar, err);
    }
}

// ---------------------------------------------------------------------------
// inverted pivot blocks (fronts of the cooperative solve levels)
// ---------------------------------------------------------------------------
// After the factorisation, the pivot block of a front holds the block-unit-
// lower L (tiles (I,K), I > K), the diagonal inverses D_K^{-1} (tiles (K,K))
// and the block-upper U's off-diagonal tiles (K,J), K < J.  k_mf_invert
// replaces them in place by
//   Y = I - L^{-1}                      below the diagonal,
//   Z_KJ = -(U^{-1})_KJ = Y'_KJ D_J^{-1}  above it (Y' = I - (I + D^{-1} N)^{-1},
//                                         N the strictly upper part of U),
// keeping D_K^{-1} on the diagonal, so that the triangular solves of the
// pivot block become products whose row blocks are independent:
//   y = v_P - Y v_P,   x_K = D_K^{-1} t_K - sum_{J > K} Z_KJ t_J.
// Right-looking, in place, on the tile products of the factorisation:
//   step 0:           U~_KJ = D_K^{-1} U_KJ                 (K < J)
//   step s, 1..Kt-2:  Y_IK  -= L_Is Y_sK   (I > s > K)
//                     Y'_KJ -= Y'_Ks U~_sJ (K < s < J)
//   step Kt-1:        Z_KJ = Y'_KJ D_J^{-1}                 (K < J)
// Step s reads row and column s only and writes neither, and a tile's last
// update comes before the step that reads it.

// the (K, J), K < J, of triangular index u (column J holds J entries)
__device__ __forceinline__ void mf_tri(int u, int &K, int &J) {
    J = 1;
    while ((J + 1) * J / 2 <= u) J++;
    K = u - J * (J - 1) / 2;
}

__device__ __forceinline__ int mf_inv_count(int s, int Kt) {
    if (Kt < 2) return 0;
    if (s == 0 || s == Kt - 1) return Kt * (Kt - 1) / 2;
    if (s < Kt - 1) return 2 * s * (Kt - 1 - s);
    return 0;
}

// tile C = tile A * tile B (C may be A or B)
template <class T>
__device__ void mf_tile_mul(T *C, const T *At, const T *Bt, MmaSmem &S) {
    typename MfAccT<T>::type acc;
    typedef typename std::remove_reference<decltype(acc[0][0][0])>::type A;
    mma_tiles(
        S, 1, [&](int) { return At; }, [&](int) { return Bt; }, acc, [&] { frag_zero(acc); });
    frag_store(C, acc, A(1));
    __syncthreads();
}

// tile C -= tile A * tile B
template <class T>
__device__ void mf_tile_sub_mul(T *C, const T *At, const T *Bt, MmaSmem &S) {
    typename MfAccT<T>::type acc;
    typedef typename std::remove_reference<decltype(acc[0][0][0])>::type A;
    mma_tiles(
        S, 1, [&](int) { return At; }, [&](int) { return Bt; }, acc,
        [&] { frag_load(C, acc, A(-1)); });
    frag_store(C, acc, A(-1));
    __syncthreads();
}

template <class T>
__device__ void mf_inv_task(const MfView &V, const MfFront &f, int s, int u, MmaSmem &S) {
    const int Kt = f.Kt;
    auto t = [&](int I, int J) { return ftile<T>(V, f, I, J); };
    int I, J, K;
    if (s == 0) {
        mf_tri(u, K, J);
        mf_tile_mul<T>(t(K, J), t(K, K), t(K, J), S);
    } else if (s == Kt - 1) {
        mf_tri(u, K, J);
        mf_tile_mul<T>(t(K, J), t(K, J), t(J, J), S);
    } else {
        const int e = Kt - 1 - s;
        if (u < s * e) {
            I = s + 1 + u % e;
            K = u / e;
            mf_tile_sub_mul<T>(t(I, K), t(I, s), t(s, K), S);
        } else {
            u -= s * e;
            K = u % s;
            J = s + 1 + u / s;
            mf_tile_sub_mul<T>(t(K, J), t(K, s), t(s, J), S);
        }
    }
}

// All listed fronts at once: step s of every front, then a grid barrier.
// Tasks are numbered across the fronts and dealt round-robin, as in
// mf_for_tasks.
template <class T>
__global__ void __launch_bounds__(LU_THREADS, 2)
k_mf_invert(MfView V, const int2 *list, int nlist, int ktmax, unsigned int *bar, int *err) {
    extern __shared__ __align__(16) double smem_raw[];
    MfFactorSmem &FS = *reinterpret_cast<MfFactorSmem *>(smem_raw);
    const int G = gridDim.x;
    for (int s = 0; s < ktmax; s++) {
        int first = blockIdx.x;
        for (int q = 0; q < nlist; q++) {
            const int2 e = list[q];
            const int cnt = mf_inv_count(s, e.y);
            if (cnt <= 0) continue;
            if (first < cnt) {
                const MfFront f = V.fr[e.x];
                for (int u = first; u < cnt; u += G) mf_inv_task<T>(V, f, s, u, FS.m);
            }
            first -= cnt;
            if (first < 0) first = first % G + (first % G < 0 ? G : 0);
        }
        if (s + 1 < ktmax) grid_barrier(bar, err);
    }
}

// ---------------------------------------------------------------------------
// solve
// ---------------------------------------------------------------------------
// The solve streams factor tiles into shared memory with bulk async copies
// (one 32 KB copy per tile, MF_SLOTS tiles in flight per CTA) and computes
// from there: the sweeps read every tile once, so their speed is the rate at
// which a CTA keeps HBM reads in flight.
constexpr int MF_SLOTS = 3;

// A front of a one-front-per-CTA level whose vector has at most MF_VS_MAX
// entries keeps it in shared memory for the whole sweep, so a tile costs
// one CTA barrier and no round trip to L2 (20 row blocks: level 6 of the
// 401 x 401 Stokes-Darcy tree has fronts of 18).
constexpr int MF_VS_MAX = 1280;

// What the one-front-per-CTA sweeps read of a front's descriptor.  A CTA
// loads the records of up to MF_LF_MAX of its fronts of a level at once (one
// thread per front, its children's descriptors too) instead of each front's
// descriptor, then its children's, when the front starts.
struct MfLf {
    long long off, var_off, map_off, vec_off;
    long long c0v, c1v;   // children's update parts in V.vec (-1: no child)
    int M, Kp, k, Kt, Mt, pad;
};
constexpr int MF_LF_MAX = MF_KM_MAX * (int)sizeof(int2) / (int)sizeof(MfLf);

struct MfSolveSmem {
    double tile[MF_SLOTS][T2];
    unsigned long long bar[MF_SLOTS];
    double part[2][4][64];  // quarter partial sums (two buffers, alternating tiles)
    double x[64];          // vector piece the current tile multiplies
    double vs[MF_VS_MAX];  // the front vector of a front swept by one CTA
    union {
        int2 km[MF_KM_MAX];   // cooperative levels: (Kt, Mt) of the level's fronts
        MfLf lf[MF_LF_MAX];   // one-front-per-CTA levels: a batch of this CTA's fronts
    };
    int last;              // this CTA's chunk of a row arrived last
};
// two CTAs per SM
static_assert(sizeof(MfSolveSmem) <= 113 * 1024, "solve shared memory");

__device__ __forceinline__ uint32_t mf_smem(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Vector piece of the sweeps that keep the front vector in global memory:
// the second partial-sum buffer, which only the shared-memory sweeps'
// one-barrier reductions (mf_reduce_rows1) use.
__device__ __forceinline__ double *mf_y(MfSolveSmem &S) { return S.part[1][0]; }

// Tile slots in flight per CTA (three for either element type: six FP32
// slots in the same storage measured no faster) and slot sl's tile.
template <class T> struct MfSlots {
    static constexpr int n = MF_SLOTS;
};
template <class T>
__device__ __forceinline__ const T *mf_slot(MfSolveSmem &S, int sl) {
    return reinterpret_cast<const T *>(S.tile[sl]);
}

// Issues the copy of one 64 x 64 tile into slot `sl` (thread 0).
template <class T>
__device__ __forceinline__ void mf_fetch(MfSolveSmem &S, int sl, const T *src) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                         mf_smem(&S.bar[sl])),
                     "r"((uint32_t)(T2 * sizeof(T)))
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(mf_smem(S.tile[sl])),
            "l"(src), "r"((uint32_t)(T2 * sizeof(T))), "r"(mf_smem(&S.bar[sl]))
            : "memory");
    }
}

// Waits (bounded, 2 s) for phase `parity` of slot `sl`; on timeout *err = 3.
__device__ __forceinline__ void mf_slot_wait(MfSolveSmem &S, int sl, uint32_t parity, int *err) {
    uint32_t ok;
    unsigned long long t0 = 0;
    for (int spin = 0;; spin++) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(mf_smem(&S.bar[sl])), "r"(parity)
            : "memory");
        if (ok) return;
        if (spin == 0) t0 = globaltimer();
        else if (globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
            atomicExch(err, 3);
            return;
        }
    }
}

// Streams the n tiles src(0..n-1) through the slots and calls use(i, tile)
// with all threads once tile i is in shared memory.  uses[] counts the
// phases of each slot's barrier (identical in every thread).  With
// `released`, use() itself ends every thread's reads of the tile before a
// CTA barrier it passes, so the slot is refilled without another one.
template <bool released = false, class Src, class Use>
__device__ void mf_stream(MfSolveSmem &S, uint32_t *uses, int n, Src src, Use use, int *err) {
    mf_stream<released>(S, uses, n, src, use, [](int) {}, err);
}
// The same with pre(i) called by all threads before tile i is waited for
// (after the previous tile's use), so its work overlaps the copies in flight.
template <bool released = false, class Src, class Use, class Pre>
__device__ void mf_stream(MfSolveSmem &S, uint32_t *uses, int n, Src src, Use use, Pre pre,
                          int *err) {
    for (int i = 0; i < n && i < MF_SLOTS; i++) mf_fetch(S, i, src(i));
    for (int i = 0; i < n; i++) {
        const int sl = i % MF_SLOTS;
        pre(i);
        mf_slot_wait(S, sl, uses[sl] & 1u, err);
        uses[sl]++;
        use(i, (const decltype(src(0)))S.tile[sl]);
        if (!released) __syncthreads();
        if (i + MF_SLOTS < n) mf_fetch(S, sl, src(i + MF_SLOTS));
    }
}

// Thread (r, q) = (tid % 64, tid / 64): its share of row r of T x, columns
// 16 q .. 16 q + 15 (T in shared memory, column-major; x in shared memory).
template <class T>
__device__ __forceinline__ double mf_quarter(const T *Tt, const double *x) {
    const int r = threadIdx.x & 63, q = threadIdx.x >> 6;
    const T *t = Tt + q * 16 * 64 + r;
    const double *xx = x + q * 16;
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int c = 0; c < 16; c += 2) {
        s0 = fma((double)t[c * 64], xx[c], s0);
        s1 = fma((double)t[(c + 1) * 64], xx[c + 1], s1);
    }
    return s0 + s1;
}

// Reduces the quarter sums s of all threads: returns the row total in
// threads 0..63 (row = tid).  Ends with a barrier.
__device__ __forceinline__ double mf_reduce_rows(MfSolveSmem &S, double s) {
    S.part[0][threadIdx.x >> 6][threadIdx.x & 63] = s;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 64) {
        const int r = threadIdx.x;
        t = (S.part[0][0][r] + S.part[0][1][r]) + (S.part[0][2][r] + S.part[0][3][r]);
    }
    __syncthreads();
    return t;
}

// The same sum through buffer `b` with one barrier: consecutive calls
// alternate the buffers, so a buffer is written again only after the
// barrier of the call in between, when its readers (threads 0..63, right
// after the barrier of their own call) are done with it.
__device__ __forceinline__ double mf_reduce_rows1(MfSolveSmem &S, double s, int b) {
    S.part[b][threadIdx.x >> 6][threadIdx.x & 63] = s;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 64) {
        const int r = threadIdx.x;
        t = (S.part[b][0][r] + S.part[b][1][r]) + (S.part[b][2][r] + S.part[b][3][r]);
    }
    return t;
}

// Gathers the front vector: the right-hand side of the eliminated unknowns
// plus the children's update vectors.
__device__ void mf_gather_fwd(const MfView &V, const MfFront &f, const double *w, double *v) {
    const int *var = V.vars + f.var_off, *map = V.eamap + f.map_off;
    MfFront C0, C1;
    bool h0 = f.c0 >= 0, h1 = f.c1 >= 0;
    if (h0) C0 = V.fr[f.c0];
    if (h1) C1 = V.fr[f.c1];
    for (int a = threadIdx.x; a < f.M; a += blockDim.x) {
        int g = var[a];
        double s = (a < f.Kp && g >= 0) ? __ldcg(&w[g]) : 0.0;
        if (h0) {
            int i = map[2 * a];
            if (i >= 0) s += __ldcg(&V.vec[C0.vec_off + C0.Kp + i]);
        }
        if (h1) {
            int i = map[2 * a + 1];
            if (i >= 0) s += __ldcg(&V.vec[C1.vec_off + C1.Kp + i]);
        }
        __stcg(&v[a], s);
    }
    __syncthreads();
}

// Forward elimination inside a front: for each block column K < Kt, rows
// I in (K, iend) get v_I -= L_IK y_K, with y_K = v_K final once column K
// starts.  The tiles stream in column order.
template <class T>
__device__ void mf_fwd_front(const MfView &V, const MfFront &f, double *v, int iend,
                             MfSolveSmem &S, uint32_t *uses, int *err) {
    // tile i -> (K, I): columns K = 0.. with iend - K - 1 tiles each
    int n = 0;
    for (int K = 0; K < f.Kt; K++) n += max(0, iend - K - 1);
    int K = 0, I = 1;     // position of the next tile handed to use()
    int fk = 0, fi = 1;   // position of the next tile fetched by src()
    auto src = [&](int) {
        while (fi >= iend) {
            fk++;
            fi = fk + 1;
        }
        const T *t = ftile<T>(V, f, fi, fk);
        fi++;
        return t;
    };
    mf_stream(
        S, uses, n, src,
        [&](int, const T *Tt) {
            while (I >= iend) {
                K++;
                I = K + 1;
            }
            if (I == K + 1) {   // first tile of column K: y_K
                if (threadIdx.x < 64) mf_y(S)[threadIdx.x] = __ldcg(&v[K * 64 + threadIdx.x]);
                __syncthreads();
            }
            double t = mf_reduce_rows(S, mf_quarter(Tt, mf_y(S)));
            if (threadIdx.x < 64) {
                double *d = &v[I * 64 + threadIdx.x];
                __stcg(d, __ldcg(d) - t);
            }
            I++;
        },
        err);
}

// v_I -= sum_{K in [k0, k1)} T(I, K) x_K for one tile row I; xsrc(K, c)
// gives element c of the vector piece K.
template <class T, class Xsrc>
__device__ void mf_row_gemv(const MfView &V, const MfFront &f, double *v, int I, int k0, int k1,
                            Xsrc xsrc, MfSolveSmem &S, uint32_t *uses, int *err) {
    double acc = 0.0;
    mf_stream(
        S, uses, k1 - k0, [&](int i) { return (const T *)ftile<T>(V, f, I, k0 + i); },
        [&](int i, const T *Tt) {
            if (threadIdx.x < 64) S.x[threadIdx.x] = xsrc(k0 + i, threadIdx.x);
            __syncthreads();
            acc += mf_quarter(Tt, S.x);
        },
        err);
    double t = mf_reduce_rows(S, acc);
    if (threadIdx.x < 64) {
        double *d = &v[I * 64 + threadIdx.x];
        __stcg(d, __ldcg(d) - t);
    }
    __syncthreads();
}

// Backward substitution inside a front (the update part already
// subtracted): for K = Kt-1 .. 0, x_K = D_K^{-1} v_K, then v_I -= U_IK x_K
// for I < K.  The solution goes to v and to w.  Tiles stream as (K,K),
// (0,K), (1,K), ..., (K-1,K) for K descending.
template <class T>
__device__ void mf_bwd_front(const MfView &V, const MfFront &f, double *v, double *wout,
                             MfSolveSmem &S, uint32_t *uses, int *err) {
    const int *var = V.vars + f.var_off;
    const int n = f.Kt * (f.Kt + 1) / 2;
    int K = f.Kt - 1, j = 0;     // use position: j == 0 -> (K,K), else row j-1
    int fk = f.Kt - 1, fj = 0;   // fetch position
    auto src = [&](int) {
        if (fj > fk) {
            fk--;
            fj = 0;
        }
        const T *t = fj == 0 ? ftile<T>(V, f, fk, fk) : ftile<T>(V, f, fj - 1, fk);
        fj++;
        return t;
    };
    mf_stream(
        S, uses, n, src,
        [&](int, const T *Tt) {
            if (j > K) {
                K--;
                j = 0;
            }
            if (j == 0) {   // x_K = D_K^{-1} v_K
                if (threadIdx.x < 64) mf_y(S)[threadIdx.x] = __ldcg(&v[K * 64 + threadIdx.x]);
                __syncthreads();
                double x = mf_reduce_rows(S, mf_quarter(Tt, mf_y(S)));
                if (threadIdx.x < 64) {
                    const int r = threadIdx.x, a = K * 64 + r;
                    S.x[r] = x;
                    __stcg(&v[a], x);
                    if (a < f.k) __stcg(&wout[var[a]], x);
                }
                __syncthreads();
            } else {        // v_I -= U_IK x_K, I = j - 1
                double t = mf_reduce_rows(S, mf_quarter(Tt, S.x));
                if (threadIdx.x < 64) {
                    double *d = &v[(j - 1) * 64 + threadIdx.x];
                    __stcg(d, __ldcg(d) - t);
                }
            }
            j++;
        },
        err);
}

// ---- one front per CTA, the front vector in shared memory ------------------
// The same arithmetic as mf_gather_fwd + mf_fwd_front and mf_row_gemv +
// mf_bwd_front, in the same order, for fronts with M <= MF_VS_MAX.

// Forward sweep of front f: gather into S.vs, eliminate, write the vector
// (pivot part for the backward sweep, update part for the parent) to V.vec.
template <class T>
__device__ void mf_fwd_front_s(const MfView &V, const MfFront &f, const double *w,
                               MfSolveSmem &S, uint32_t *uses, int *err) {
    double *vs = S.vs;
    {
        const int *var = V.vars + f.var_off, *map = V.eamap + f.map_off;
        MfFront C0, C1;
        const bool h0 = f.c0 >= 0, h1 = f.c1 >= 0;
        if (h0) C0 = V.fr[f.c0];
        if (h1) C1 = V.fr[f.c1];
        for (int a = threadIdx.x; a < f.M; a += blockDim.x) {
            int g = var[a];
            double s = (a < f.Kp && g >= 0) ? __ldcg(&w[g]) : 0.0;
            if (h0) {
                int i = map[2 * a];
                if (i >= 0) s += __ldcg(&V.vec[C0.vec_off + C0.Kp + i]);
            }
            if (h1) {
                int i = map[2 * a + 1];
                if (i >= 0) s += __ldcg(&V.vec[C1.vec_off + C1.Kp + i]);
            }
            vs[a] = s;
        }
    }
    int n = 0;
    for (int K = 0; K < f.Kt; K++) n += f.Mt - K - 1;
    int K = 0, I = 1, b = 0;
    int fk = 0, fi = 1;
    auto src = [&](int) {
        while (fi >= f.Mt) {
            fk++;
            fi = fk + 1;
        }
        const T *t = ftile<T>(V, f, fi, fk);
        fi++;
        return t;
    };
    __syncthreads();
    mf_stream<true>(
        S, uses, n, src,
        [&](int, const T *Tt) {
            while (I >= f.Mt) {
                K++;
                I = K + 1;
            }
            if (I == K + 1) __syncthreads();   // row K is final
            double t = mf_reduce_rows1(S, mf_quarter(Tt, vs + K * 64), b);
            b ^= 1;
            if (threadIdx.x < 64) vs[I * 64 + threadIdx.x] -= t;
            I++;
        },
        err);
    __syncthreads();
    double *v = V.vec + f.vec_off;
    for (int a = threadIdx.x; a < f.M; a += blockDim.x) __stcg(&v[a], vs[a]);
    __syncthreads();
}

// Backward sweep of front f: the ring solution (from w) and the pivot part
// of the forward sweep into S.vs; rows K < Kt subtract the ring products
// (all ring tiles streamed row after row), then the block substitution.
// The solution goes to V.vec and to w.
template <class T>
__device__ void mf_bwd_front_s(const MfView &V, const MfFront &f, double *w, MfSolveSmem &S,
                               uint32_t *uses, int *err) {
    double *vs = S.vs, *v = V.vec + f.vec_off;
    const int *var = V.vars + f.var_off;
    for (int a = threadIdx.x; a < f.M; a += blockDim.x) {
        if (a < f.Kp) {
            vs[a] = __ldcg(&v[a]);
        } else {
            int g = var[a];
            vs[a] = g >= 0 ? __ldcg(&w[g]) : 0.0;
        }
    }
    __syncthreads();
    const int nr = f.Mt - f.Kt;
    if (nr > 0) {
        double acc = 0.0;
        mf_stream(
            S, uses, f.Kt * nr,
            [&](int i) { return (const T *)ftile<T>(V, f, i / nr, f.Kt + i % nr); },
            [&](int i, const T *Tt) {
                acc += mf_quarter(Tt, vs + (f.Kt + i % nr) * 64);
                if (i % nr == nr - 1) {
                    double t = mf_reduce_rows(S, acc);
                    if (threadIdx.x < 64) vs[(i / nr) * 64 + threadIdx.x] -= t;
                    acc = 0.0;
                }
            },
            err);
    }
    const int n = f.Kt * (f.Kt + 1) / 2;
    int K = f.Kt - 1, j = 0, b = 0;
    int fk = f.Kt - 1, fj = 0;
    auto src = [&](int) {
        if (fj > fk) {
            fk--;
            fj = 0;
        }
        const T *t = fj == 0 ? ftile<T>(V, f, fk, fk) : ftile<T>(V, f, fj - 1, fk);
        fj++;
        return t;
    };
    __syncthreads();
    mf_stream<true>(
        S, uses, n, src,
        [&](int, const T *Tt) {
            if (j > K) {
                K--;
                j = 0;
            }
            if (j == 0) {   // x_K = D_K^{-1} v_K
                __syncthreads();   // row K is final
                double x = mf_reduce_rows1(S, mf_quarter(Tt, vs + K * 64), b);
                if (threadIdx.x < 64) {
                    const int r = threadIdx.x, a = K * 64 + r;
                    S.x[r] = x;
                    vs[a] = x;
                    __stcg(&v[a], x);
                    if (a < f.k) __stcg(&w[var[a]], x);
                }
                __syncthreads();   // S.x is complete
            } else {        // v_I -= U_IK x_K, I = j - 1
                double t = mf_reduce_rows1(S, mf_quarter(Tt, S.x), b);
                if (threadIdx.x < 64) vs[(j - 1) * 64 + threadIdx.x] -= t;
            }
            b ^= 1;
            j++;
        },
        err);
    __syncthreads();
}

// ---- one front per CTA, a level at a time -----------------------------------
// The sweeps of mf_fwd_front_s / mf_bwd_front_s (same arithmetic, same
// order) over all of this CTA's fronts of a level (fronts fb + blockIdx.x +
// k G) through one tile pipeline: thread 0 keeps a fetch cursor that runs
// MfSlots<T>::n tiles ahead across the fronts, so the next front's first
// tiles are in flight while the current front finishes and the next one is
// gathered.

// Records of this CTA's fronts fi, fi + G, ... (at most MF_LF_MAX, below
// fe) into lf; `children` adds the children's update-part offsets.  Called
// by all threads; ends with a barrier.
template <bool children>
__device__ void mf_load_lf(const MfView &V, int fi, int G, int fe, MfLf *lf) {
    const int q = threadIdx.x, f_i = fi + q * G;
    if (q < MF_LF_MAX && f_i < fe) {
        const MfFront f = V.fr[f_i];
        MfLf r;
        r.off = f.off;
        r.var_off = f.var_off;
        r.map_off = f.map_off;
        r.vec_off = f.vec_off;
        r.M = f.M;
        r.Kp = f.Kp;
        r.k = f.k;
        r.Kt = f.Kt;
        r.Mt = f.Mt;
        r.pad = 0;
        r.c0v = r.c1v = -1;
        if (children) {
            if (f.c0 >= 0) r.c0v = V.fr[f.c0].vec_off + V.fr[f.c0].Kp;
            if (f.c1 >= 0) r.c1v = V.fr[f.c1].vec_off + V.fr[f.c1].Kp;
        }
        lf[q] = r;
    }
    __syncthreads();
}

// (off, Kt, Mt) of front fi for a fetch cursor (thread 0): from the batch
// of records in lf that starts at front lf0 when fi is in it, else from the
// descriptor in global memory.
__device__ __forceinline__ void mf_cursor_front(const MfView &V, const MfLf *lf, int lf0,
                                                int lfn, int G, int fi, long long &off,
                                                int &Kt, int &Mt) {
    const int q = (fi - lf0) / G;
    if (fi >= lf0 && q < lfn) {
        off = lf[q].off;
        Kt = lf[q].Kt;
        Mt = lf[q].Mt;
    } else {
        const MfFront &F = V.fr[fi];
        off = F.off;
        Kt = F.Kt;
        Mt = F.Mt;
    }
}

// Fetch cursor of the forward sweep: tiles (I, K), K < Kt, I = K+1..Mt-1.
template <class T>
struct MfFwdCursor {
    int fi, fe, G, K, I, Kt, Mt;
    long long off;
    const MfLf *lf;
    int lf0, lfn;   // the batch of records in lf: fronts lf0, lf0 + G, ... (lfn of them)
    __device__ void load(const MfView &V) {
        if (fi < fe) {
            mf_cursor_front(V, lf, lf0, lfn, G, fi, off, Kt, Mt);
            K = 0;
            I = 1;
        }
    }
    __device__ const T *next(const MfView &V) {
        while (fi < fe) {
            while (K < Kt && I >= Mt) {
                K++;
                I = K + 1;
            }
            if (K < Kt) return (const T *)V.F + off + ((long long)K * Mt + I++) * T2;
            fi += G;
            load(V);
        }
        return nullptr;
    }
};

// Fetch cursor of the backward sweep: the ring tiles (K, Kt + j) row by row,
// then (K, K), (0, K), ..., (K-1, K) for K = Kt-1 .. 0.
template <class T>
struct MfBwdCursor {
    int fi, fe, G, K, j, ring, Kt, Mt;
    long long off;
    const MfLf *lf;
    int lf0, lfn;   // as in MfFwdCursor
    __device__ void load(const MfView &V) {
        if (fi < fe) {
            mf_cursor_front(V, lf, lf0, lfn, G, fi, off, Kt, Mt);
            ring = Mt > Kt;
            K = ring ? 0 : Kt - 1;
            j = 0;
        }
    }
    __device__ const T *next(const MfView &V) {
        while (fi < fe) {
            if (ring) {
                const int nr = Mt - Kt;
                if (j >= nr) {
                    j = 0;
                    K++;
                }
                if (K < Kt) {
                    const int J = Kt + j++;
                    return (const T *)V.F + off + ((long long)J * Mt + K) * T2;
                }
                ring = 0;
                K = Kt - 1;
                j = 0;
            }
            if (K >= 0 && j > K) {
                K--;
                j = 0;
            }
            if (K >= 0) {
                const int I = j == 0 ? K : j - 1;
                j++;
                return (const T *)V.F + off + ((long long)K * Mt + I) * T2;
            }
            fi += G;
            load(V);
        }
        return nullptr;
    }
};

// The next front's gather (this CTA's front fi + G, when its record is in
// the batch) is prefetched into registers while the current front's tiles
// stream: its index loads right after the current front's gather, its value
// loads after the first tile, and the sums, in the gather's order, when it
// starts.  Thread t holds elements t + j LU_THREADS, j < MF_PF: fronts of
// up to MF_PF LU_THREADS entries (the levels with several fronts per CTA have
// at most 640) are prefetched, larger ones gathered when they start.
constexpr int MF_PF = 3;

template <class T>
__device__ void mf_fwd_level_s(const MfView &V, int fb, int fe, const double *w, MfSolveSmem &S,
                               uint32_t *uses, int *err) {
    constexpr int NS = MfSlots<T>::n;
    const int G = gridDim.x;
    double *vs = S.vs;
    const int fi0 = fb + blockIdx.x;
    mf_load_lf<true>(V, fi0, G, fe, S.lf);
    MfFwdCursor<T> cur;
    if (threadIdx.x == 0) {
        cur.fi = fi0;
        cur.fe = fe;
        cur.G = G;
        cur.lf = S.lf;
        cur.lf0 = fi0;
        cur.lfn = MF_LF_MAX;
        cur.load(V);
        for (int q = 0; q < NS; q++) {
            const T *p = cur.next(V);
            if (!p) break;
            mf_fetch(S, q, p);
        }
    }
    int pg[MF_PF], pm0[MF_PF], pm1[MF_PF];   // next front: indices
    double pw[MF_PF], pc0[MF_PF], pc1[MF_PF];  // next front: values
    bool have = false;   // the current front's gather is in the registers
    int sl = 0, q = 0;
    for (int fi = fi0; fi < fe; fi += G, q++) {
        if (q == MF_LF_MAX) {   // every thread is past the batch's last front
            q = 0;
            mf_load_lf<true>(V, fi, G, fe, S.lf);
            if (threadIdx.x == 0) cur.lf0 = fi;
        }
        const MfLf &f = S.lf[q];
        if (have) {
#pragma unroll
            for (int j = 0; j < MF_PF; j++) {
                const int a = threadIdx.x + j * LU_THREADS;
                if (a < f.M) {
                    double s = pw[j];
                    if (pm0[j] >= 0) s += pc0[j];
                    if (pm1[j] >= 0) s += pc1[j];
                    vs[a] = s;
                }
            }
        } else {
            const int *var = V.vars + f.var_off, *map = V.eamap + f.map_off;
            const long long c0v = f.c0v, c1v = f.c1v;
            for (int a = threadIdx.x; a < f.M; a += blockDim.x) {
                int g = var[a];
                double s = (a < f.Kp && g >= 0) ? __ldcg(&w[g]) : 0.0;
                if (c0v >= 0) {
                    int i = map[2 * a];
                    if (i >= 0) s += __ldcg(&V.vec[c0v + i]);
                }
                if (c1v >= 0) {
                    int i = map[2 * a + 1];
                    if (i >= 0) s += __ldcg(&V.vec[c1v + i]);
                }
                vs[a] = s;
            }
        }
        __syncthreads();
        // the next front's indices
        const bool next =
            q + 1 < MF_LF_MAX && fi + G < fe && S.lf[q + 1].M <= MF_PF * LU_THREADS;
        if (next) {
            const MfLf &nf = S.lf[q + 1];
            const int *var = V.vars + nf.var_off, *map = V.eamap + nf.map_off;
#pragma unroll
            for (int j = 0; j < MF_PF; j++) {
                const int a = threadIdx.x + j * LU_THREADS;
                pg[j] = pm0[j] = pm1[j] = -1;
                if (a < nf.M) {
                    pg[j] = a < nf.Kp ? var[a] : -1;
                    if (nf.c0v >= 0) pm0[j] = map[2 * a];
                    if (nf.c1v >= 0) pm1[j] = map[2 * a + 1];
                }
            }
        }
        auto values = [&]() {   // the next front's value loads
            const MfLf &nf = S.lf[q + 1];
#pragma unroll
            for (int j = 0; j < MF_PF; j++) {
                pw[j] = pg[j] >= 0 ? __ldcg(&w[pg[j]]) : 0.0;
                pc0[j] = pm0[j] >= 0 ? __ldcg(&V.vec[nf.c0v + pm0[j]]) : 0.0;
                pc1[j] = pm1[j] >= 0 ? __ldcg(&V.vec[nf.c1v + pm1[j]]) : 0.0;
            }
        };
        int n = 0;
        for (int K = 0; K < f.Kt; K++) n += f.Mt - K - 1;
        int K = 0, I = 1, b = 0;
        for (int t = 0; t < n; t++) {
            while (I >= f.Mt) {
                K++;
                I = K + 1;
            }
            if (I == K + 1) __syncthreads();   // row K is final
            mf_slot_wait(S, sl, uses[sl] & 1u, err);
            uses[sl]++;
            const double r = mf_reduce_rows1(S, mf_quarter(mf_slot<T>(S, sl), vs + K * 64), b);
            b ^= 1;
            if (threadIdx.x < 64) vs[I * 64 + threadIdx.x] -= r;
            if (threadIdx.x == 0) {   // every thread has read the slot (the barrier above)
                const T *p = cur.next(V);
                if (p) mf_fetch(S, sl, p);
            }
            sl = sl + 1 == NS ? 0 : sl + 1;
            I++;
            if (next && t == 0) values();
        }
        if (next && n == 0) values();
        have = next;
        __syncthreads();
        double *v = V.vec + f.vec_off;
        for (int a = threadIdx.x; a < f.M; a += blockDim.x) __stcg(&v[a], vs[a]);
        __syncthreads();
    }
}

template <class T>
__device__ void mf_bwd_level_s(const MfView &V, int fb, int fe, double *w, MfSolveSmem &S,
                               uint32_t *uses, int *err) {
    constexpr int NS = MfSlots<T>::n;
    const int G = gridDim.x;
    double *vs = S.vs;
    const int fi0 = fb + blockIdx.x;
    mf_load_lf<false>(V, fi0, G, fe, S.lf);
    MfBwdCursor<T> cur;
    if (threadIdx.x == 0) {
        cur.fi = fi0;
        cur.fe = fe;
        cur.G = G;
        cur.lf = S.lf;
        cur.lf0 = fi0;
        cur.lfn = MF_LF_MAX;
        cur.load(V);
        for (int q = 0; q < NS; q++) {
            const T *p = cur.next(V);
            if (!p) break;
            mf_fetch(S, q, p);
        }
    }
    int sl = 0;
    auto refill = [&]() {   // call after a barrier that follows every read of slot sl
        if (threadIdx.x == 0) {
            const T *p = cur.next(V);
            if (p) mf_fetch(S, sl, p);
        }
        sl = sl + 1 == NS ? 0 : sl + 1;
    };
    // the next front's vector, prefetched as in mf_fwd_level_s
    int pg[MF_PF];
    double pv[MF_PF];
    bool have = false;
    int q = 0;
    for (int fi = fi0; fi < fe; fi += G, q++) {
        if (q == MF_LF_MAX) {   // every thread is past the batch's last front
            q = 0;
            mf_load_lf<false>(V, fi, G, fe, S.lf);
            if (threadIdx.x == 0) cur.lf0 = fi;
        }
        const MfLf &f = S.lf[q];
        double *v = V.vec + f.vec_off;
        const int *var = V.vars + f.var_off;
        if (have) {
#pragma unroll
            for (int j = 0; j < MF_PF; j++) {
                const int a = threadIdx.x + j * LU_THREADS;
                if (a < f.M) vs[a] = pv[j];
            }
        } else {
            for (int a = threadIdx.x; a < f.M; a += blockDim.x) {
                if (a < f.Kp) {
                    vs[a] = __ldcg(&v[a]);
                } else {
                    int g = var[a];
                    vs[a] = g >= 0 ? __ldcg(&w[g]) : 0.0;
                }
            }
        }
        __syncthreads();
        // the next front's ring indices (-2: a pivot-part entry, -1: none)
        const bool next =
            q + 1 < MF_LF_MAX && fi + G < fe && S.lf[q + 1].M <= MF_PF * LU_THREADS;
        if (next) {
            const MfLf &nf = S.lf[q + 1];
            const int *nvar = V.vars + nf.var_off;
#pragma unroll
            for (int j = 0; j < MF_PF; j++) {
                const int a = threadIdx.x + j * LU_THREADS;
                pg[j] = a >= nf.M ? -1 : a < nf.Kp ? -2 : nvar[a];
            }
        }
        bool fetched = !next;
        auto values = [&]() {   // the next front's value loads
            if (fetched) return;
            fetched = true;
            const MfLf &nf = S.lf[q + 1];
            const double *nv = V.vec + nf.vec_off;
#pragma unroll
            for (int j = 0; j < MF_PF; j++) {
                const int a = threadIdx.x + j * LU_THREADS;
                pv[j] = pg[j] == -2 ? __ldcg(&nv[a]) : pg[j] >= 0 ? __ldcg(&w[pg[j]]) : 0.0;
            }
        };
        const int nr = f.Mt - f.Kt;
        if (nr > 0) {   // rows K < Kt minus the ring products
            for (int K = 0; K < f.Kt; K++) {
                double acc = 0.0;
                for (int j = 0; j < nr; j++) {
                    mf_slot_wait(S, sl, uses[sl] & 1u, err);
                    uses[sl]++;
                    acc += mf_quarter(mf_slot<T>(S, sl), vs + (f.Kt + j) * 64);
                    __syncthreads();
                    refill();
                    values();
                }
                const double t = mf_reduce_rows(S, acc);
                if (threadIdx.x < 64) vs[K * 64 + threadIdx.x] -= t;
            }
        }
        int b = 0;
        for (int K = f.Kt - 1; K >= 0; K--) {
            for (int j = 0; j <= K; j++) {
                mf_slot_wait(S, sl, uses[sl] & 1u, err);
                uses[sl]++;
                const T *Tt = mf_slot<T>(S, sl);
                if (j == 0) {   // x_K = D_K^{-1} v_K
                    __syncthreads();   // row K is final
                    const double x = mf_reduce_rows1(S, mf_quarter(Tt, vs + K * 64), b);
                    if (threadIdx.x < 64) {
                        const int r = threadIdx.x, a = K * 64 + r;
                        S.x[r] = x;
                        vs[a] = x;
                        __stcg(&v[a], x);
                        if (a < f.k) __stcg(&w[var[a]], x);
                    }
                    refill();
                    __syncthreads();   // S.x is complete
                } else {        // v_I -= U_IK x_K, I = j - 1
                    const double t = mf_reduce_rows1(S, mf_quarter(Tt, S.x), b);
                    if (threadIdx.x < 64) vs[(j - 1) * 64 + threadIdx.x] -= t;
                    refill();
                }
                b ^= 1;
                values();
            }
        }
        values();
        have = next;
        __syncthreads();
    }
}

// ---- cooperative levels: one task per 64-row block of a front --------------
// Row block I of front f is final in solve `epoch` once its flag holds
// 2 epoch (forward) or 2 epoch + 1 (backward); epochs grow, so older marks
// are smaller.  Writers: every thread fences its own stores, then thread 0
// raises the flag; readers: thread 0 waits (bounded, 2 s; on timeout *err = 3)
// and the block reads through L2.
__device__ __forceinline__ int *mf_flag(const MfView &V, const MfFront &f, int I) {
    return V.flags + f.vec_off / 64 + I;
}
__device__ __forceinline__ void mf_wait_flag(const int *flag, int want, int *err) {
    if (threadIdx.x == 0) {
        unsigned long long t0 = 0;
        for (int spin = 0;; spin++) {
            if (*(volatile const int *)flag >= want) break;
            // once a wait of this launch has given up, the launch ends quickly
            if (*(volatile const int *)err) break;
            if (spin == 0) {
                t0 = globaltimer();
            } else if (globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
                atomicExch(err, 3);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
    }
    __syncthreads();
}
__device__ __forceinline__ void mf_raise_flag(int *flag, int val) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicExch(flag, val);
}

// Element a of front f's vector before elimination: the right-hand side of
// an eliminated unknown plus the children's update entries (child 0, then
// child 1).
__device__ __forceinline__ double mf_gather_elem(const MfView &V, const MfFront &f,
                                                 const double *w, int a, bool h0,
                                                 const MfFront &C0, bool h1,
                                                 const MfFront &C1) {
    const int *var = V.vars + f.var_off, *map = V.eamap + f.map_off;
    int g = var[a];
    double s = (a < f.Kp && g >= 0) ? __ldcg(&w[g]) : 0.0;
    if (h0) {
        int i = map[2 * a];
        if (i >= 0) s += __ldcg(&V.vec[C0.vec_off + C0.Kp + i]);
    }
    if (h1) {
        int i = map[2 * a + 1];
        if (i >= 0) s += __ldcg(&V.vec[C1.vec_off + C1.Kp + i]);
    }
    return s;
}

// Forward, row block I: v_I = gather_I - sum_{K < min(I, Kt)} L_IK y_K, the
// y_K taken as their rows finish; pivot rows then publish.
template <class T>
__device__ void mf_fwd_row(const MfView &V, const MfFront &f, const double *w, int I, int epoch,
                           MfSolveSmem &S, uint32_t *uses, int *err) {
    double *v = V.vec + f.vec_off;
    const bool h0 = f.c0 >= 0, h1 = f.c1 >= 0;
    MfFront C0, C1;
    if (h0) C0 = V.fr[f.c0];
    if (h1) C1 = V.fr[f.c1];
    double gath = 0.0;
    if (threadIdx.x < 64) gath = mf_gather_elem(V, f, w, I * 64 + threadIdx.x, h0, C0, h1, C1);
    const int nK = I < f.Kt ? I : f.Kt;
    double acc = 0.0;
    mf_stream(
        S, uses, nK, [&](int K) { return (const T *)ftile<T>(V, f, I, K); },
        [&](int K, const T *Tt) {
            mf_wait_flag(mf_flag(V, f, K), 2 * epoch, err);
            if (threadIdx.x < 64) S.x[threadIdx.x] = __ldcg(&v[K * 64 + threadIdx.x]);
            __syncthreads();
            acc += mf_quarter(Tt, S.x);
        },
        err);
    double t = mf_reduce_rows(S, acc);
    if (threadIdx.x < 64) __stcg(&v[I * 64 + threadIdx.x], gath - t);
    if (I < f.Kt) mf_raise_flag(mf_flag(V, f, I), 2 * epoch);
    __syncthreads();
}

// Backward, row block K of the pivot part:
// x_K = D_K^{-1} (v_K - sum_{J >= Kt} U_KJ x_J - sum_{K < J < Kt} U_KJ x_J),
// the ring solution from w, the pivot ones taken as their rows finish.
template <class T>
__device__ void mf_bwd_row(const MfView &V, const MfFront &f, double *w, int K, int epoch,
                           MfSolveSmem &S, uint32_t *uses, int *err) {
    double *v = V.vec + f.vec_off;
    const int *var = V.vars + f.var_off;
    const int nr = f.Mt - f.Kt, np = f.Kt - 1 - K;
    double acc = 0.0;
    mf_stream(
        S, uses, nr + np + 1,
        [&](int i) {
            const int J = i < nr ? f.Kt + i : i < nr + np ? f.Kt - 1 - (i - nr) : K;
            return (const T *)ftile<T>(V, f, K, J);
        },
        [&](int i, const T *Tt) {
            if (i < nr) {
                const int J = f.Kt + i;
                if (threadIdx.x < 64) {
                    int g = var[J * 64 + threadIdx.x];
                    S.x[threadIdx.x] = g >= 0 ? __ldcg(&w[g]) : 0.0;
                }
                __syncthreads();
                acc += mf_quarter(Tt, S.x);
            } else if (i < nr + np) {
                const int J = f.Kt - 1 - (i - nr);
                mf_wait_flag(mf_flag(V, f, J), 2 * epoch + 1, err);
                if (threadIdx.x < 64) S.x[threadIdx.x] = __ldcg(&v[J * 64 + threadIdx.x]);
                __syncthreads();
                acc += mf_quarter(Tt, S.x);
            } else {   // the diagonal tile holds D_K^{-1}
                double t = mf_reduce_rows(S, acc);
                if (threadIdx.x < 64) mf_y(S)[threadIdx.x] = __ldcg(&v[K * 64 + threadIdx.x]) - t;
                __syncthreads();
                double x = mf_reduce_rows(S, mf_quarter(Tt, mf_y(S)));
                if (threadIdx.x < 64) {
                    const int a = K * 64 + threadIdx.x;
                    __stcg(&v[a], x);
                    if (a < f.k) __stcg(&w[var[a]], x);
                }
            }
        },
        err);
    mf_raise_flag(mf_flag(V, f, K), 2 * epoch + 1);
    __syncthreads();
}

// ---- cooperative levels with inverted pivot blocks -------------------------
// Per level, forward: (F1) pivot rows y_I = v_I - sum_{K<I} Y_IK v_K into
// vec2, (F2) update rows v_I -= sum_{K<Kt} L_IK y_K; backward: (B1) partial
// ring products sum_{J in chunk} U_KJ x_J of the pivot rows, (B2)
// x_K = D_K^{-1} t_K - sum_{J>K} Z_KJ t_J with t_J = y_J minus its partials.
// v is gathered where it is read (children's update parts and the right-
// hand side), so each sweep of a level takes two phases, and every task is
// one row block or a chunk of one: no task waits for another inside a phase.
constexpr int MF_XG = 16;                // vector pieces staged in shared memory at a time
static_assert(MF_XG * 64 == 4 * LU_THREADS, "staging: four elements per thread");
static_assert(MF_XG * 64 <= MF_VS_MAX, "staging area");
static_assert(MF_RING_CHUNK == MF_XG, "a B1 task stages its ring pieces once");

// The task maps, chunk sizes and partial-sum offsets are in mf_tasks.h.
// element c of y_K
__device__ __forceinline__ double mf_inv_y(const MfView &V, const MfFront &f, int K, int c) {
    double y = __ldcg(&V.vec2[f.vec_off + K * 64 + c]);
    const int nc = mf_f1_chunks(K);
    for (int ch = 1; ch < nc; ch++) y -= __ldcg(&V.part[mf_f1_part(f, K, ch) + c]);
    return y;
}

// Update rows (F2, Kt tiles each) and pivot rows (B2, Kt - K tiles) of more
// than MF_F1_CHUNK tiles are split into chunks of MF_F1_CHUNK tiles on the
// levels that chunk long rows, each chunk a task of its own (the root's first
// pivot row would stream 38 tiles through one CTA).  Every chunk stores its
// partial row product; the chunk that arrives last (a count per row block, in
// V.flags, which the inverted form does not otherwise use) adds the partials
// in chunk order and writes the row, so the result does not depend on which
// CTA finishes last.
// Called by all threads after threads 0..63 stored their chunk's partial:
// counts the chunk in *cnt and returns, in every thread, whether it was the
// last of the row's nch.  The last one resets the count for the next solve
// and may then read the other chunks' partials through L2.
__device__ __forceinline__ bool mf_chunk_arrive(int *cnt, int nch, MfSolveSmem &S) {
    __threadfence();   // this thread's partial before the count
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool last = atomicAdd(cnt, 1) + 1 == nch;
        if (last) {
            atomicExch(cnt, 0);
            __threadfence();
        }
        S.last = last;
    }
    __syncthreads();
    return S.last;
}

// Inside a cooperative level the F2 tasks of a front read only that front's
// F1 results, and its B2 tasks only its B1 partials, so instead of a grid
// barrier between the phases each F1 (B1) task counts itself done in the
// front's count, V.done[2 r] (V.done[2 r + 1]) with r the front's first row
// block, and an F2 (B2) task waits for its front's count.  The counts grow
// by the front's task count every solve: solve `epoch` waits for epoch x
// tasks (compared modulo 2^32).  Every CTA runs all its F1 (B1) tasks before
// any F2 (B2) task and those wait for nothing, so every wait ends; waits are
// bounded (2 s; on timeout *err = 3) all the same.
__device__ __forceinline__ int *mf_done(const MfView &V, const MfFront &f, int phase) {
    return V.done + 2 * (f.vec_off / 64) + phase;
}
// Called by all threads after their outputs are stored.
__device__ __forceinline__ void mf_count_done(int *cnt) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(cnt, 1);
}
// Called by all threads; returns once *cnt has reached `want` (mod 2^32).
__device__ __forceinline__ void mf_wait_done(const int *cnt, unsigned int want, int *err) {
    if (threadIdx.x == 0) {
        unsigned long long t0 = 0;
        for (int spin = 0;; spin++) {
            const unsigned int c = (unsigned int)*(volatile const int *)cnt;
            if ((int)(c - want) >= 0) break;
            if (*(volatile const int *)err) break;   // the launch is giving up
            if (spin == 0) {
                t0 = globaltimer();
            } else if (globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
                atomicExch(err, 3);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
    }
    __syncthreads();
}

// Per-thread quarter sums of sum_{i<n} sign(i) T_i x_i: tile(i) points to
// T_i, piece(i, c) gives element c of x_i; the pieces are staged in
// S.vs MF_XG at a time while the tiles stream.  wait() runs in all threads
// once, after the first tiles' copies are issued and before any piece is
// read; first() once, after the first pieces' loads are issued, so the
// task's own gather overlaps them.
template <class T, class Tile, class Piece, class Sign, class Wait, class First>
__device__ double mf_row_tiles(MfSolveSmem &S, uint32_t *uses, int n, Tile tile, Piece piece,
                               Sign sign, Wait wait, First first, int *err) {
    double acc = 0.0;
    if (n == 0) first();
    mf_stream(
        S, uses, n, tile,
        [&](int i, const T *Tt) { acc += sign(i) * mf_quarter(Tt, S.vs + (i % MF_XG) * 64); },
        [&](int i) {
            if (i == 0) wait();
            if (i % MF_XG == 0) {   // staged while the tiles' copies are in flight; the
                                    // previous tile's barrier has passed
                const int m = min(n - i, MF_XG) * 64;
                double v[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int e = threadIdx.x + q * LU_THREADS;
                    v[q] = e < m ? piece(i + (e >> 6), e & 63) : 0.0;
                }
                if (i == 0) first();
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int e = threadIdx.x + q * LU_THREADS;
                    if (e < m) S.vs[e] = v[q];
                }
                __syncthreads();
            }
        },
        err);
    return acc;
}

// F1 task u of front f: chunk ch of pivot row block I (tiles K in
// [8 ch, min(I, 8 ch + 8))).
template <class T>
__device__ void mf_inv_f1(const MfView &V, const MfFront &f, const double *w, int u,
                          MfSolveSmem &S, uint32_t *uses, int *err) {
    int I, ch, k0, n;
    mf_f1_task(f.Kt, u, I, ch, k0, n);
    const bool h0 = f.c0 >= 0, h1 = f.c1 >= 0;
    MfFront C0, C1;
    if (h0) C0 = V.fr[f.c0];
    if (h1) C1 = V.fr[f.c1];
    double g = 0.0;
    const double acc = mf_row_tiles<T>(
        S, uses, n, [&](int i) { return (const T *)ftile<T>(V, f, I, k0 + i); },
        [&](int i, int c) {
            return mf_gather_elem(V, f, w, (k0 + i) * 64 + c, h0, C0, h1, C1);
        },
        [](int) { return 1.0; }, []() {},
        [&]() {
            if (ch == 0 && threadIdx.x < 64)
                g = mf_gather_elem(V, f, w, I * 64 + threadIdx.x, h0, C0, h1, C1);
        },
        err);
    const double t = mf_reduce_rows(S, acc);
    if (threadIdx.x < 64) {
        if (ch == 0) __stcg(&V.vec2[f.vec_off + I * 64 + threadIdx.x], g - t);
        else __stcg(&V.part[mf_f1_part(f, I, ch) + threadIdx.x], t);
    }
    mf_count_done(mf_done(V, f, 0));
}

// F2 task u of front f with nrc chunks per row: chunk ch of update row block
// I (>= Kt), tiles K in [8 ch, 8 ch + 8) (all Kt when nrc = 1): v_I =
// gathered entries minus sum_K L_IK y_K.  Chunk 0's partial holds the
// gathered entries minus its products, the later ones their products.
template <class T>
__device__ void mf_inv_f2(const MfView &V, const MfFront &f, const double *w, int u, int nrc,
                          int epoch, MfSolveSmem &S, uint32_t *uses, int *err) {
    int I, ch, k0, n;
    mf_f2_task(f.Kt, nrc, u, I, ch, k0, n);
    const bool h0 = f.c0 >= 0, h1 = f.c1 >= 0;
    MfFront C0, C1;
    if (h0) C0 = V.fr[f.c0];
    if (h1) C1 = V.fr[f.c1];
    double g = 0.0;
    const double acc = mf_row_tiles<T>(
        S, uses, n, [&](int i) { return (const T *)ftile<T>(V, f, I, k0 + i); },
        [&](int i, int c) { return mf_inv_y(V, f, k0 + i, c); }, [](int) { return 1.0; },
        [&]() {   // the front's pivot rows (F1)
            mf_wait_done(mf_done(V, f, 0), (unsigned)epoch * (unsigned)mf_f1_tasks(f.Kt), err);
        },
        [&]() {
            if (ch == 0 && threadIdx.x < 64)
                g = mf_gather_elem(V, f, w, I * 64 + threadIdx.x, h0, C0, h1, C1);
        },
        err);
    const double t = mf_reduce_rows(S, acc);
    double *v = V.vec + f.vec_off + I * 64;
    if (nrc == 1) {
        if (threadIdx.x < 64) __stcg(&v[threadIdx.x], g - t);
        return;
    }
    if (threadIdx.x < 64)
        __stcg(&V.part[mf_row_part(f, I, ch) + threadIdx.x], ch == 0 ? g - t : t);
    if (!mf_chunk_arrive(mf_flag(V, f, I), nrc, S)) return;
    if (threadIdx.x < 64) {
        double r = __ldcg(&V.part[mf_row_part(f, I, 0) + threadIdx.x]);
        for (int c = 1; c < nrc; c++) r -= __ldcg(&V.part[mf_row_part(f, I, c) + threadIdx.x]);
        __stcg(&v[threadIdx.x], r);
    }
}

// B1 task u of front f: ring tiles [Kt + 16 ch, ...) of pivot row block K.
template <class T>
__device__ void mf_inv_b1(const MfView &V, const MfFront &f, const double *w, int u,
                          MfSolveSmem &S, uint32_t *uses, int *err) {
    int K, ch, j0, n;
    mf_b1_task(f.Kt, f.Mt, u, K, ch, j0, n);
    const int *var = V.vars + f.var_off;
    const double acc = mf_row_tiles<T>(
        S, uses, n, [&](int j) { return (const T *)ftile<T>(V, f, K, j0 + j); },
        [&](int j, int c) {
            const int g = var[(j0 + j) * 64 + c];
            return g >= 0 ? __ldcg(&w[g]) : 0.0;
        },
        [](int) { return 1.0; }, []() {}, []() {}, err);
    const double t = mf_reduce_rows(S, acc);
    if (threadIdx.x < 64) __stcg(&V.part[mf_ring_part(f, K, ch) + threadIdx.x], t);
    mf_count_done(mf_done(V, f, 1));
}

// B2 task u of front f: chunk ch of pivot row block K, tiles (K, K + i) for i
// in [8 ch, 8 ch + 8) (all Kt - K when the row has one chunk or the level is
// not `chunked`); the solution x_K = D_K^{-1} t_K - sum_{J>K} Z_KJ t_J goes
// to w.
template <class T>
__device__ void mf_inv_b2(const MfView &V, const MfFront &f, double *w, int u, bool chunked,
                          int epoch, MfSolveSmem &S, uint32_t *uses, int *err) {
    const int nch = mf_ring_chunks(f.Mt - f.Kt);
    const int *var = V.vars + f.var_off;
    int K, ch, nrc, i0, n;
    mf_b2_task(f.Kt, chunked, u, K, ch, nrc, i0, n);
    const double acc = mf_row_tiles<T>(
        S, uses, n, [&](int i) { return (const T *)ftile<T>(V, f, K, K + i0 + i); },
        [&](int i, int c) {
            const int J = K + i0 + i;
            double t = mf_inv_y(V, f, J, c);
            if (nch > 0) {
                const double *pp = V.part + mf_ring_part(f, J, 0) + c;
                for (int q = 0; q < nch; q++) t -= __ldcg(&pp[q * 64]);
            }
            return t;
        },
        [=](int i) { return i0 + i == 0 ? 1.0 : -1.0; },
        [&]() {   // the front's ring partials (B1)
            if (nch > 0)
                mf_wait_done(mf_done(V, f, 1),
                             (unsigned)epoch * (unsigned)mf_b1_tasks(f.Kt, f.Mt), err);
        },
        []() {}, err);
    double x = mf_reduce_rows(S, acc);
    if (nrc > 1) {
        if (threadIdx.x < 64) __stcg(&V.part[mf_row_part(f, K, ch) + threadIdx.x], x);
        if (!mf_chunk_arrive(mf_flag(V, f, K), nrc, S)) return;
        if (threadIdx.x < 64) {
            x = __ldcg(&V.part[mf_row_part(f, K, 0) + threadIdx.x]);
            for (int c = 1; c < nrc; c++) x += __ldcg(&V.part[mf_row_part(f, K, c) + threadIdx.x]);
        }
    }
    if (threadIdx.x < 64) {
        const int a = K * 64 + threadIdx.x;
        if (a < f.k) __stcg(&w[var[a]], x);
    }
}

// Solves L U x = w in place (w: n values; rows >= n untouched).
template <class T>
__global__ void __launch_bounds__(LU_THREADS, 2)
k_mf_solve(MfView V, double *w, unsigned int *bar, int *err, int epoch) {
    extern __shared__ __align__(128) double smem_raw[];
    MfSolveSmem &S = *reinterpret_cast<MfSolveSmem *>(smem_raw);
    const int G = gridDim.x;
    uint32_t uses[MF_SLOTS];
    for (int i = 0; i < MF_SLOTS; i++) uses[i] = 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < MF_SLOTS; i++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mf_smem(&S.bar[i]))
                         : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    // forward: leaves to root
    for (int p = 0; p < V.nlev; p++) {
        const int fb = V.lvl[p], fe = V.lvl[p + 1];
        const bool local = V.lvl_mode[p] & MF_SOLVE_LOCAL;
        if (!local) mf_load_km(V, fb, fe, S.km);
        if (local && (V.lvl_mode[p] & MF_SOLVE_VS)) {
            mf_fwd_level_s<T>(V, fb, fe, w, S, uses, err);
        } else if (local) {
            for (int fi = fb + blockIdx.x; fi < fe; fi += G) {
                const MfFront f = V.fr[fi];
                if (f.M <= MF_VS_MAX) {
                    mf_fwd_front_s<T>(V, f, w, S, uses, err);
                    continue;
                }
                double *v = V.vec + f.vec_off;
                mf_gather_fwd(V, f, w, v);
                mf_fwd_front<T>(V, f, v, f.Mt, S, uses, err);
            }
        } else if (V.inv) {
            mf_for_tasks(
                V, fb, fe, S.km, [](int Kt, int) { return mf_f1_tasks(Kt); },
                [&](const MfFront &f, int u) { mf_inv_f1<T>(V, f, w, u, S, uses, err); });
            // no grid barrier: an F2 task waits for its own front's F1 tasks
            const bool cf = V.lvl_mode[p] & MF_CHUNK_F2;
            mf_for_tasks(
                V, fb, fe, S.km,
                [cf](int Kt, int Mt) { return mf_f2_tasks(Kt, Mt, cf ? mf_row_chunks(Kt) : 1); },
                [&](const MfFront &f, int u) {
                    mf_inv_f2<T>(V, f, w, u, cf ? mf_row_chunks(f.Kt) : 1, epoch, S, uses,
                                 err);
                });
        } else {
            // one task per row block, in increasing order within each front
            mf_for_tasks(
                V, fb, fe, S.km, [](int, int Mt) { return Mt; },
                [&](const MfFront &f, int I) { mf_fwd_row<T>(V, f, w, I, epoch, S, uses, err); });
        }
        grid_barrier(bar, err);
    }
    // backward: root to leaves
    for (int p = V.nlev - 1; p >= 0; p--) {
        const int fb = V.lvl[p], fe = V.lvl[p + 1];
        const bool local = V.lvl_mode[p] & MF_SOLVE_LOCAL;
        if (!local) mf_load_km(V, fb, fe, S.km);
        auto ring_x = [&](const MfFront &f) {
            const int *var = V.vars + f.var_off;
            return [=](int J, int c) {
                int g = var[J * 64 + c];
                return g >= 0 ? __ldcg(&w[g]) : 0.0;
            };
        };
        if (local && (V.lvl_mode[p] & MF_SOLVE_VS)) {
            mf_bwd_level_s<T>(V, fb, fe, w, S, uses, err);
        } else if (local) {
            for (int fi = fb + blockIdx.x; fi < fe; fi += G) {
                const MfFront f = V.fr[fi];
                if (f.M <= MF_VS_MAX) {
                    mf_bwd_front_s<T>(V, f, w, S, uses, err);
                    continue;
                }
                double *v = V.vec + f.vec_off;
                for (int K = 0; K < f.Kt && f.Mt > f.Kt; K++)
                    mf_row_gemv<T>(V, f, v, K, f.Kt, f.Mt, ring_x(f), S, uses, err);
                mf_bwd_front<T>(V, f, v, w, S, uses, err);
            }
        } else if (V.inv) {
            mf_for_tasks(
                V, fb, fe, S.km, [](int Kt, int Mt) { return mf_b1_tasks(Kt, Mt); },
                [&](const MfFront &f, int u) { mf_inv_b1<T>(V, f, w, u, S, uses, err); });
            // no grid barrier: a B2 task waits for its own front's B1 tasks
            const bool cb = V.lvl_mode[p] & MF_CHUNK_B2;
            mf_for_tasks(
                V, fb, fe, S.km, [cb](int Kt, int) { return mf_b2_count(Kt, cb); },
                [&](const MfFront &f, int u) {
                    mf_inv_b2<T>(V, f, w, u, cb, epoch, S, uses, err);
                });
        } else {
            // one task per pivot row block, the last first
            mf_for_tasks(
                V, fb, fe, S.km, [](int Kt, int) { return Kt; },
                [&](const MfFront &f, int u) {
                    mf_bwd_row<T>(V, f, w, f.Kt - 1 - u, epoch, S, uses, err);
                });
        }
        grid_barrier(bar, err);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static MfView mf_view(const MfDevice &D, const BandSystem &sys) {
    MfView V;
    V.fr = D.fr;
    V.F = (D.fp32 || D.solve32) ? D.F32 : D.F64;
    V.vec = D.vec;
    V.vars = D.vars;
    V.eamap = D.eamap;
    V.lvl = D.lvl;
    V.lvl_kt = D.lvl_kt;
    V.lvl_mode = D.lvl_mode;
    V.flags = D.flags;
    V.done = D.done;
    V.vec2 = D.vec2;
    V.part = D.part;
    V.inv = D.inv ? 1 : 0;
    V.nlev = D.nlev;
    V.target = D.target;
    V.expect = D.expect;
    V.n = sys.n;
    V.ell = sys.ell;
    return V;
}

bool mf_is_fp32(const BandSystem &sys) { return sys.mf && sys.mf->fp32; }

// Zeroes the row-block flags (the chunk counts of the inverted form) and the
// per-front task counts, and restarts the epochs: after a solve that gave
// up, counts of tasks that never finished must not carry over into the next
// solve.
void mf_clear_counts(erebus_state *s, BandSystem &sys) {
    MfDevice *D = sys.mf;
    if (!D || !D->flags) return;
    cudaMemsetAsync(D->flags, 0, (D->plan.vec / MF_TILE + 1) * sizeof(int), s->stream);
    if (D->done)
        cudaMemsetAsync(D->done, 0, 2 * (D->plan.vec / MF_TILE + 1) * sizeof(int), s->stream);
    D->epoch = 0;   // the counts restart with the epochs
}

void mf_release(BandSystem &sys) {
    MfDevice *D = sys.mf;
    if (!D) return;
    void *ps[] = {D->fr, D->F64, D->F32, D->vec, D->vars, D->eamap, D->lvl, D->lvl_kt,
                  D->lvl_mode, D->flags, D->done, D->target, D->expect, D->vec2, D->part,
                  D->inv_list,
                  D->cvt};
    for (void *p : ps)
        if (p) cudaFree(p);
    delete D;
    sys.mf = nullptr;
    sys.has_factor = false;
    sys.refactor_cost = 0.0;   // the next plan may differ
    sys.cyc_solves = 0;
    sys.cyc_iters = 0;
}

template <class T>
static cudaError_t upload(T **dst, const std::vector<T> &src, cudaStream_t st) {
    cudaError_t e = cudaMalloc(dst, std::max<size_t>(1, src.size()) * sizeof(T));
    if (e == cudaSuccess && !src.empty())
        e = cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st);
    return e;
}

// CTAs of the cooperative factor and solve launches (2 per SM).
static int mf_grid(const erebus_state *s) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    return 2 * sms;
}

// How each level is processed.  A level with at least G/2 fronts (or more
// than fit the shared-memory table) runs one front per CTA.  Otherwise the
// choice weighs the serial chain of one CTA doing a whole front against the
// fixed cost of the cooperative phases (a grid barrier and a pass over the
// level's fronts each): the factor runs a front per CTA when that front's
// tile operations are few, the solve when its tile sweeps are short.  The
// thresholds come from timing whole timesteps of the 141x141 and 401x401
// workloads on a B200 (erebus_b200.autotune): with inverted pivot blocks at
// the cooperative levels, 64 tiles per sweep beat 24 by 0.7-1.5%.
constexpr int kLocalFactorOps = 8;    // tile operations per CTA
constexpr int kLocalSolveTiles = 64;  // tiles streamed per CTA and sweep
static std::vector<int> mf_level_modes(const MfPlan &P, int G, int factor_ops,
                                       int solve_tiles) {
    std::vector<int> mode;
    for (size_t p = 0; p + 1 < P.level_begin.size(); p++) {
        const int fb = P.level_begin[p], fe = P.level_begin[p + 1], F = fe - fb;
        const int waves = (F + G - 1) / G;
        long long ops = 0, tiles = 0;
        for (int fi = fb; fi < fe; fi++) {
            const MfFront &f = P.fronts[fi];
            long long o = (f.c0 >= 0 || f.c1 >= 0 ? (long long)f.Mt * f.Mt : 0) + 2LL * f.Kt +
                          (long long)(f.Mt - f.Kt) * (f.Mt - f.Kt) * f.Kt;
            long long fwd = 0;
            for (int K = 0; K < f.Kt; K++) {
                const int e = f.Kt - K - 1, R = f.Mt - K - 1;
                o += R + (long long)e * R + (long long)(f.Mt - f.Kt) * e;
                fwd += R;
            }
            const long long bwd = (long long)f.Kt * (f.Kt + 1) / 2 + (long long)f.Kt * (f.Mt - f.Kt);
            ops = std::max(ops, o);
            tiles = std::max(tiles, std::max(fwd, bwd));
        }
        const bool forced = F >= G / 2 || F > MF_KM_MAX;
        int m = 0;
        bool vs = true;
        for (int fi = fb; fi < fe; fi++) vs = vs && P.fronts[fi].M <= MF_VS_MAX;
        if (vs) m |= MF_SOLVE_VS;
        if (forced || waves * ops <= factor_ops) m |= MF_FACTOR_LOCAL;
        if (forced || waves * tiles <= solve_tiles) m |= MF_SOLVE_LOCAL;
        long long f2 = 0, b2 = 0;
        bool longrows = false;
        for (int fi = fb; fi < fe; fi++) {
            const MfFront &f = P.fronts[fi];
            f2 += (long long)(f.Mt - f.Kt) * mf_row_chunks(f.Kt);
            b2 += mf_b2_tasks(f.Kt);
            // a row of 9-12 tiles gains less than a chunk's count and
            // partial-sum reads cost
            longrows = longrows || f.Kt > MF_F1_CHUNK + MF_F1_CHUNK / 2;
        }
        if (longrows && f2 <= G) m |= MF_CHUNK_F2;
        if (longrows && b2 <= G) m |= MF_CHUNK_B2;
        mode.push_back(m);
    }
    return mode;
}

// Leaves of at most 32 nodes for the 6-unknown system (at 141 x 141 the
// bisection stops at regions of 21-32 nodes: 126-192 unknowns, two or three
// 64-wide pivot tiles), 64 nodes for the scalar ones.  Measured at 141 x 141 against 8, 16 and 24
// nodes (Stokes-Darcy) and 32 and 128 (scalar): 16 -> 32 takes one tree
// level off and the timestep from 10.24 to 9.97 ms.
static int mf_leaf(const erebus_state *s, int dofs) {
    const int o = dofs >= 4 ? s->opt.mf_leaf_vector : s->opt.mf_leaf_scalar;
    return o > 0 ? o : dofs >= 4 ? 32 : 64;
}

// Builds the plan of `sys` from the column pattern of its assembled ELL
// matrix (on the device) and uploads it.
static int mf_prepare(erebus_state *s, BandSystem &sys, int dofs) {
    mf_release(sys);
    MfDevice *D = new MfDevice();
    sys.mf = D;
    int64_t rows = (int64_t)sys.NB * sys.nb;
    std::vector<int> cols(rows * sys.ell);
    int rc = check_cuda(s, cudaMemcpyAsync(cols.data(), sys.ell_cols, cols.size() * 4,
                                           cudaMemcpyDeviceToHost, s->stream), "mf pattern");
    if (!rc) rc = stream_sync(s, "mf pattern");
    if (rc) return rc;
    MfPlan &P = D->plan;
    if (!mf_analyse(P, dofs, s->g.Ny1, s->g.Nx1, mf_leaf(s, dofs)) || P.n != sys.n) {
        s->last_error = "multifrontal analysis failed";
        return EREBUS_EINVAL;
    }
    std::vector<long long> target;
    if (!mf_targets(P, cols.data(), rows, sys.ell, target)) {
        s->last_error = "multifrontal analysis: matrix pattern outside the fronts";
        return EREBUS_EINVAL;
    }
    std::vector<int> expect(cols.begin(), cols.begin() + sys.n * sys.ell);
    target.resize(sys.n * sys.ell);
    std::vector<int> lvl_kt;
    for (size_t p = 0; p + 1 < P.level_begin.size(); p++) {
        int m = 0;
        for (int f = P.level_begin[p]; f < P.level_begin[p + 1]; f++) m = std::max(m, P.fronts[f].Kt);
        lvl_kt.push_back(m);
    }
    D->nlev = (int)P.level_begin.size() - 1;
    const int fops = s->opt.mf_local_factor_ops > 0 ? s->opt.mf_local_factor_ops
                                                     : kLocalFactorOps;
    const int stiles = s->opt.mf_local_solve_tiles > 0 ? s->opt.mf_local_solve_tiles
                                                        : kLocalSolveTiles;
    const std::vector<int> modes = mf_level_modes(P, mf_grid(s), fops, stiles);
    // cooperative solve levels: inverted pivot blocks, partial-sum storage
    D->inv = s->opt.mf_block_substitution == 0;
    std::vector<int2> inv;
    long long poff = 0;
    for (int p = 0; D->inv && p < D->nlev; p++) {
        if (modes[p] & MF_SOLVE_LOCAL) continue;
        for (int fi = P.level_begin[p]; fi < P.level_begin[p + 1]; fi++) {
            MfFront &F = P.fronts[fi];
            const long long slots = mf_part_slots(F.Kt, F.Mt);
            if (slots > 0 && F.Kt > 0) {   // ring partials, F1 partials, chunked rows
                F.poff = poff;
                poff += slots * 64;
            }
            if (F.Kt >= 2) {
                inv.push_back(make_int2(fi, F.Kt));
                D->inv_ktmax = std::max(D->inv_ktmax, F.Kt);
            }
        }
    }
    D->n_inv = (int)inv.size();
    cudaError_t e = upload(&D->fr, P.fronts, s->stream);
    if (e == cudaSuccess) e = upload(&D->vars, P.vars, s->stream);
    if (e == cudaSuccess) e = upload(&D->eamap, P.eamap, s->stream);
    if (e == cudaSuccess) e = upload(&D->lvl, P.level_begin, s->stream);
    if (e == cudaSuccess) e = upload(&D->lvl_kt, lvl_kt, s->stream);
    if (e == cudaSuccess) e = upload(&D->lvl_mode, modes, s->stream);
    if (e == cudaSuccess && D->inv) e = upload(&D->inv_list, inv, s->stream);
    if (e == cudaSuccess && D->inv) e = cudaMalloc(&D->vec2, P.vec * sizeof(double));
    if (e == cudaSuccess && D->inv)
        e = cudaMalloc(&D->part, std::max<long long>(poff, 1) * sizeof(double));
    if (e == cudaSuccess) e = upload(&D->target, target, s->stream);
    if (e == cudaSuccess) e = upload(&D->expect, expect, s->stream);
    if (e == cudaSuccess) e = cudaMalloc(&D->vec, P.vec * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&D->flags, (P.vec / MF_TILE + 1) * sizeof(int));
    if (e == cudaSuccess && D->inv)
        e = cudaMalloc(&D->done, 2 * (P.vec / MF_TILE + 1) * sizeof(int));
    if (e == cudaSuccess && D->inv)
        e = cudaMemsetAsync(D->done, 0, 2 * (P.vec / MF_TILE + 1) * sizeof(int), s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(D->flags, 0, (P.vec / MF_TILE + 1) * sizeof(int),
                                              s->stream);
    if (e != cudaSuccess) {
        s->last_error = std::string("multifrontal allocation: ") + cudaGetErrorString(e);
        return EREBUS_ENOMEM;
    }
    return stream_sync(s, "mf upload");
}

static int mf_blocks(erebus_state *s, const void *func, size_t smem) {
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, LU_THREADS, smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    return std::min(per_sm, 2) * sms;
}

template <class T>
static int mf_factor_t(erebus_state *s, BandSystem &sys) {
    MfDevice &D = *sys.mf;
    void *&F = sizeof(T) == 4 ? D.F32 : D.F64;
    if (!F) {
        cudaError_t e = cudaMalloc(&F, D.plan.storage * sizeof(T));
        if (e != cudaSuccess) {
            F = nullptr;
            s->last_error = std::string("multifrontal factor storage: ") + cudaGetErrorString(e);
            return EREBUS_ENOMEM;
        }
    }
    D.fp32 = sizeof(T) == 4;
    D.solve32 = false;
    MfView V = mf_view(D, sys);
    int rc = check_cuda(s, cudaMemsetAsync(F, 0, D.plan.storage * sizeof(T), s->stream),
                        "mf zero");
    if (rc) return rc;
    EREBUS_LAUNCH(s, k_mf_scatter<T>, nblocks(sys.n), kThreads, 0, V, sys.ell_cols,
                  sys.ell_vals, sys.err);
    int nf = (int)D.plan.fronts.size();
    EREBUS_LAUNCH(s, k_mf_pad<T>, nf, 64, 0, V, nf);
    size_t smem = sizeof(MfFactorSmem);
    const void *fn = (const void *)k_mf_factor<T>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int blocks = mf_blocks(s, fn, smem);
    if (blocks < 1) {
        s->last_error = "mf_factor: kernel does not fit";
        return EREBUS_ECUDA;
    }
    unsigned int *bar = sys.bar;
    int *err = sys.err;
    void *args[] = {&V, &bar, &err};
    cudaMemsetAsync(sys.bar, 0, 4 * sizeof(unsigned int), s->stream);
    rc = coop_launch(s, fn, blocks, LU_THREADS, args, smem, "mf_factor launch");
    s->launches++;
    if (rc || !D.inv || D.n_inv == 0) return rc;
    const void *fi = (const void *)k_mf_invert<T>;
    cudaFuncSetAttribute(fi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    blocks = mf_blocks(s, fi, smem);
    if (blocks < 1) {
        s->last_error = "mf_invert: kernel does not fit";
        return EREBUS_ECUDA;
    }
    const int2 *list = D.inv_list;
    int nlist = D.n_inv, ktmax = D.inv_ktmax;
    void *iargs[] = {&V, &list, &nlist, &ktmax, &bar, &err};
    cudaMemsetAsync(sys.bar, 0, 4 * sizeof(unsigned int), s->stream);
    rc = coop_launch(s, fi, blocks, LU_THREADS, iargs, smem, "mf_invert launch");
    s->launches++;
    return rc;
}

int mf_factor(erebus_state *s, BandSystem &sys, bool fp32) {
    int rc;
    if (!sys.mf) {
        rc = mf_prepare(s, sys, sys.dofs);
        if (rc) return rc;
    }
    rc = fp32 ? mf_factor_t<float>(s, sys) : mf_factor_t<double>(s, sys);
    if (rc) return rc;
    sys.factored = true;
    sys.has_factor = true;
    sys.factorizations++;
    return EREBUS_OK;
}

// The FP32 copy holds only what the triangular solves read: per front the
// pivot columns (tile columns J < Kt) and the pivot rows of the other
// columns (tiles (I, J), I < Kt <= J).  The Schur complement block, which
// the parent consumed in the extend-add, is not copied.  One CTA per range
// (x: first element, y: element count, both multiples of 4096).
__global__ void k_f64_to_f32(const double *__restrict__ src, float *__restrict__ dst,
                             const longlong2 *__restrict__ ranges) {
    const longlong2 r = ranges[blockIdx.x];
    const double2 *s2 = reinterpret_cast<const double2 *>(src + r.x);
    float2 *d2 = reinterpret_cast<float2 *>(dst + r.x);
    for (long long k = threadIdx.x; k < r.y / 2; k += blockDim.x) {
        const double2 v = __ldcs(&s2[k]);
        d2[k] = make_float2((float)v.x, (float)v.y);
    }
}

int mf_convert_fp32(erebus_state *s, BandSystem &sys) {
    MfDevice *D = sys.mf;
    if (!D || !D->F64 || D->fp32) {
        s->last_error = "mf_convert_fp32: no FP64 factors";
        return EREBUS_EINVAL;
    }
    if (!D->F32) {
        cudaError_t e = cudaMalloc(&D->F32, D->plan.storage * sizeof(float));
        if (e != cudaSuccess) {
            D->F32 = nullptr;
            s->last_error = std::string("multifrontal FP32 copy: ") + cudaGetErrorString(e);
            return EREBUS_ENOMEM;
        }
    }
    if (!D->cvt) {
        std::vector<longlong2> r;
        for (const MfFront &F : D->plan.fronts)
            for (int J = 0; J < F.Mt; J++) {
                const long long n = J < F.Kt ? F.Mt : F.Kt;
                if (n > 0)
                    r.push_back(make_longlong2(F.off + (long long)J * F.Mt * T2, n * T2));
            }
        cudaError_t e = upload(&D->cvt, r, s->stream);
        if (e != cudaSuccess) {
            s->last_error = std::string("multifrontal FP32 ranges: ") + cudaGetErrorString(e);
            return EREBUS_ENOMEM;
        }
        D->n_cvt = (int)r.size();
    }
    if (D->n_cvt > 0)
        EREBUS_LAUNCH(s, k_f64_to_f32, D->n_cvt, 256, 0, (const double *)D->F64, (float *)D->F32,
                      (const longlong2 *)D->cvt);
    D->solve32 = true;
    return check_cuda(s, cudaGetLastError(), "mf_convert_fp32");
}

void mf_stats(const erebus_state *s, const BandSystem &sys, ErebusFactorStats *o) {
    MfPlan P;
    mf_analyse(P, sys.dofs, s->g.Ny1, s->g.Nx1, mf_leaf(s, sys.dofs));
    double tiles = 0.0, rd = 0.0;
    if (s->opt.mf_block_substitution == 0) {   // inversion of the cooperative levels' pivot blocks
        const int fops = s->opt.mf_local_factor_ops > 0 ? s->opt.mf_local_factor_ops
                                                         : kLocalFactorOps;
        const int stiles = s->opt.mf_local_solve_tiles > 0 ? s->opt.mf_local_solve_tiles
                                                            : kLocalSolveTiles;
        const std::vector<int> modes = mf_level_modes(P, mf_grid(s), fops, stiles);
        for (size_t p = 0; p < modes.size(); p++) {
            if (modes[p] & MF_SOLVE_LOCAL) continue;
            for (int fi = P.level_begin[p]; fi < P.level_begin[p + 1]; fi++) {
                const double kt = P.fronts[fi].Kt;
                if (kt >= 2) tiles += kt * (kt - 1) + (kt - 2) * (kt - 1) * kt / 3.0;
            }
        }
    }
    for (const MfFront &F : P.fronts) {
        tiles += F.Kt;   // inverses
        for (int K = 0; K < F.Kt; K++) {
            int R = F.Mt - K - 1, e = F.Kt - K - 1;
            tiles += R + e * R + (F.Mt - F.Kt) * e;
        }
        tiles += (double)(F.Mt - F.Kt) * (F.Mt - F.Kt) * F.Kt;
        rd += 2.0 * F.Kt * F.Mt - (double)F.Kt * F.Kt;
    }
    o->fronts = (int32_t)P.fronts.size();
    o->levels = (int32_t)P.level_begin.size() - 1;
    const int es = s->opt.factor_fp32 ? sizeof(float) : sizeof(double);
    const int ss = (s->opt.factor_fp32 ||
                    (s->opt.krylov && s->opt.precond_fp32 && sys.dofs > 1))
                       ? sizeof(float) : sizeof(double);
    o->storage_bytes = P.storage * (int64_t)es;
    o->flops = tiles * 2.0 * T2 * NB_TILE;
    o->solve_bytes = rd * T2 * ss;
}

int mf_solve(erebus_state *s, BandSystem &sys, double *w) {
    if (!sys.mf) {
        s->last_error = "mf_solve: system not factored";
        return EREBUS_EINVAL;
    }
    MfDevice &D = *sys.mf;
    MfView V = mf_view(D, sys);
    size_t smem = sizeof(MfSolveSmem);
    const void *fn = (D.fp32 || D.solve32) ? (const void *)k_mf_solve<float>
                                           : (const void *)k_mf_solve<double>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int blocks = mf_blocks(s, fn, smem);
    if (blocks < 1) {
        s->last_error = "mf_solve: kernel does not fit";
        return EREBUS_ECUDA;
    }
    unsigned int *bar = sys.bar;
    int *err = sys.err;
    int epoch = ++D.epoch;
    void *args[] = {&V, &w, &bar, &err, &epoch};
    cudaMemsetAsync(sys.bar, 0, 4 * sizeof(unsigned int), s->stream);
    timer_begin(s, sys.ph_precond);
    int rc = coop_launch(s, fn, blocks, LU_THREADS, args, smem, "mf_solve launch");
    timer_end(s, sys.ph_precond);
    s->launches++;
    return rc;
}

}  // namespace erebus
