// krylov.cu -- mixed-precision Krylov solves with a lagged LU preconditioner.
//
// The reference solves its three linear systems with a sparse direct LU at
// every call (UMFPACK through LinearSolve / `\`, src/Erebus.jl:6612,
// E:6736-6748, E:6925).  The plain path of this library does the same with
// the multifrontal LU plus FP64 iterative refinement (bandlu.cu).  This file
// is the library's mixed-precision form of those solves:
//
//  * flexible GMRES (right preconditioned, restarted) in FP64: residuals,
//    matrix products with the assembled rows, Gram-Schmidt (two passes) and
//    the solution update are FP64;
//  * the preconditioner is the multifrontal LU of an earlier matrix of the
//    same system; with precond_fp32 set, the Stokes-Darcy system applies it
//    from an FP32 copy of its FP64 factors (a triangular solve then reads
//    half the bytes);
//  * the factors are kept while the matrix changes, and computed again (in
//    FP64) when they stop paying: by default when the previous solve's cost
//    reached the average cost per solve since the last factorisation, the
//    factorisation included (the renewal rule for the cheapest long-run
//    cost per solve while iterations grow with the preconditioner's age;
//    the factorisation's cost in iterations comes from a fixed cost model of
//    the plan, so the decisions, and the results, are the same run to run);
//    with refactor_iterations = n > 0, when the previous solve needed more
//    than n iterations.  A solve that reaches three times the break-even
//    count without converging refactors on the spot.
//
// Every reduction is summed in a fixed order (block partials, then the blocks
// in order), so a solve is reproducible run to run.  The residual targets are
// the plain path's (hydro_rtol and friends).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "solver.cuh"

namespace erebus {

namespace {

constexpr int KB = 296;   // blocks of the partial dot products (2 per SM)
constexpr int KT = 256;
constexpr int kFloorUses = 8;   // solves accepted at a measured residual floor

// part[i * KB + b] = block b's share of dot(V_i, w), i < nv.  Block b takes
// the b-th contiguous chunk; inside a block lanes stride by KT and the KT
// lane sums are reduced in a fixed tree.
__global__ void __launch_bounds__(KT) k_mdot_part(const double *__restrict__ V, int64_t ld,
                                                  int nv, const double *__restrict__ w,
                                                  int64_t n, double *__restrict__ part) {
    __shared__ double red[KT / 32];
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = 0; i < nv; i++) {
        const double *v = V + (int64_t)i * ld;
        double acc = 0.0;
        // four elements' loads in flight before their multiply-adds, which
        // keep the lane's order k, k + KT, k + 2 KT, ...
        int64_t k = lo + threadIdx.x;
        for (; k + 3 * KT < hi; k += 4 * KT) {
            const double a0 = v[k], a1 = v[k + KT], a2 = v[k + 2 * KT], a3 = v[k + 3 * KT];
            const double b0 = w[k], b1 = w[k + KT], b2 = w[k + 2 * KT], b3 = w[k + 3 * KT];
            acc = fma(a0, b0, acc);
            acc = fma(a1, b1, acc);
            acc = fma(a2, b2, acc);
            acc = fma(a3, b3, acc);
        }
        for (; k < hi; k += KT) acc = fma(v[k], w[k], acc);
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) red[warp] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int q = 0; q < KT / 32; q++) t += red[q];
            part[(int64_t)i * KB + blockIdx.x] = t;
        }
        __syncthreads();
    }
}

// out[i] = sum_b part[i * KB + b] in block order (one block per i); with
// `acc`, acc[i] += out[i] as well.
__global__ void __launch_bounds__(KT) k_mdot_sum(const double *__restrict__ part,
                                                 double *__restrict__ out,
                                                 double *__restrict__ acc) {
    __shared__ double red[KT];
    const int i = blockIdx.x;
    red[threadIdx.x] = threadIdx.x < KB ? part[(int64_t)i * KB + threadIdx.x] : 0.0;
    if (threadIdx.x + KT < KB) red[threadIdx.x] += part[(int64_t)i * KB + threadIdx.x + KT];
    __syncthreads();
    for (int off = KT / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[i] = red[0];
        if (acc) acc[i] += red[0];
    }
}

// w += sign * sum_i c_i V_i (i in increasing order), c on the device
__global__ void k_maxpy(double *__restrict__ w, const double *__restrict__ V, int64_t ld,
                        int nv, const double *__restrict__ c, double sign, int64_t n) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double s = 0.0;
    int i = 0;
    for (; i + 3 < nv; i += 4) {   // four loads in flight, summed in order
        const double v0 = V[(int64_t)i * ld + k], v1 = V[(int64_t)(i + 1) * ld + k];
        const double v2 = V[(int64_t)(i + 2) * ld + k], v3 = V[(int64_t)(i + 3) * ld + k];
        s = fma(c[i], v0, s);
        s = fma(c[i + 1], v1, s);
        s = fma(c[i + 2], v2, s);
        s = fma(c[i + 3], v3, s);
    }
    for (; i < nv; i++) s = fma(c[i], V[(int64_t)i * ld + k], s);
    w[k] = fma(sign, s, w[k]);
}

// y = A x with the scaled rows (ELL)
__global__ void k_ell_matvec(BandView B, const double *__restrict__ x, double *__restrict__ y) {
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= (int64_t)B.NB * B.nb) return;
    double s = 0.0;
    for (int k = 0; k < B.ell; k++) {
        const int c = B.ell_cols[row * B.ell + k];
        if (c >= 0) s = fma(B.ell_vals[row * B.ell + k], x[c], s);
    }
    y[row] = s;
}

__global__ void k_scale(double *__restrict__ dst, const double *__restrict__ src, double f,
                        int64_t n) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = src[k] * f;
}

int kalloc(erebus_state *s, BandSystem &sys, int m) {
    if (sys.kbasis && sys.kdim >= m) return EREBUS_OK;
    if (sys.kbasis) cudaFree(sys.kbasis);
    if (sys.kwork) cudaFree(sys.kwork);
    if (sys.khost) cudaFreeHost(sys.khost);
    sys.kbasis = nullptr;
    sys.kwork = nullptr;
    sys.khost = nullptr;
    const int64_t np = (int64_t)sys.NB * sys.nb;
    cudaError_t e = cudaMalloc(&sys.kbasis, (size_t)(2 * m + 1) * np * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMalloc(&sys.kwork, (size_t)(KB * (m + 2) + 4 * (m + 2)) * sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&sys.khost, (size_t)(2 * m + 2) * sizeof(double));
    if (e != cudaSuccess) {
        s->last_error = std::string("krylov basis: ") + cudaGetErrorString(e);
        return EREBUS_ENOMEM;
    }
    sys.kdim = m;
    return EREBUS_OK;
}

// Cost of one factorisation of `sys` in Krylov iterations, from the plan:
// the factorisation as FP64 tile flops at 15 TFLOP/s plus 0.25 ms per tree
// level, an iteration as the factor bytes one triangular solve reads at
// 3 TB/s plus 25 us per level plus ~30 FP64 vector passes at 5 TB/s
// (rates of the multifrontal kernels measured on a B200 at 141x141 and
// 401x401: 11 and 36 iterations against 14 and 32 from the model).
double refactor_cost(const erebus_state *s, const BandSystem &sys) {
    ErebusFactorStats fs = {};
    mf_stats(s, sys, &fs);
    const double np = (double)sys.NB * sys.nb;
    const double tf = fs.flops / 15e12 + fs.levels * 0.25e-3;
    const double ti = fs.solve_bytes / 3e12 + fs.levels * 25e-6 + np * 8.0 * 30.0 / 5e12;
    return tf / ti;
}

// Factor the current matrix in FP64 (and, for the Stokes-Darcy system when
// precond_fp32 is set, make the FP32 copy its triangular solves read; the
// scalar systems' solves are short, and their FP64 factors save the extra
// iterations an FP32 copy costs).
int refactor(erebus_state *s, BandSystem &sys) {
    timer_end(s, sys.ph_solve);
    timer_begin(s, sys.ph_factor);
    int rc = mf_factor(s, sys, false);
    if (!rc && s->opt.precond_fp32 && sys.dofs > 1) rc = mf_convert_fp32(s, sys);
    timer_end(s, sys.ph_factor);
    timer_begin(s, sys.ph_solve);
    return rc;
}

}  // namespace

int krylov_solve(erebus_state *s, BandSystem &sys, double rtol, ErebusSolveStats *st) {
    const int m = s->opt.krylov_restart;
    const int thr = s->opt.refactor_iterations;
    int rc = kalloc(s, sys, m);
    if (rc) return rc;
    const int64_t np = (int64_t)sys.NB * sys.nb;
    double *V = sys.kbasis;                        // V_0 .. V_m
    double *Z = sys.kbasis + (int64_t)(m + 1) * np;   // Z_0 .. Z_{m-1}
    double *part = sys.kwork;                      // KB * (m + 2)
    double *hd = part + (int64_t)KB * (m + 2);      // h column (m + 2)
    double *h2 = hd + (m + 2);                     // second Gram-Schmidt pass
    double *yd = h2 + (m + 2);                     // update coefficients
    double *nd = yd + (m + 2);                     // |w|^2
    BandView B = band_view(sys);
    const int nb = nblocks(np);

    if (thr == 0 && sys.refactor_cost == 0.0) sys.refactor_cost = refactor_cost(s, sys);
    // iterations at which the next solve would cost the cycle's average
    const int even = thr > 0 ? thr
                             : std::max(4, (int)std::ceil((sys.refactor_cost + sys.cyc_iters) /
                                                          std::max(1, sys.cyc_solves)));
    timer_begin(s, sys.ph_solve);
    int at_factor = 0;   // iterations of this solve before its factorisation
    const bool stale = thr > 0 ? sys.last_iterations > thr
                               : sys.cyc_solves > 0 &&
                                     (double)sys.last_iterations * sys.cyc_solves >=
                                         sys.refactor_cost + sys.cyc_iters;
    if (!sys.has_factor || (!sys.factored && stale)) {
        rc = refactor(s, sys);
        if (rc) return rc;
        sys.cyc_solves = 0;
        sys.cyc_iters = 0;
    }
    if (!sys.have_x) cudaMemsetAsync(sys.x, 0, np * 8, s->stream);

    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1);
    // page-locked, so the copies of the Hessenberg column and of the update
    // coefficients are asynchronous (one host wait per iteration)
    double *hh = sys.khost, *y = sys.khost + (m + 2);
    double *r = sys.r;                             // residual work vector
    int total = 0;
    double rel = INFINITY, prev_cycle = INFINITY, bnorm = 0.0;
    bool stalled = false;
    double *part2 = s->norm_part;
    for (int cycle = 0;; cycle++) {
        // true residual r = b - A x, and its norm with |b|
        EREBUS_LAUNCH(s, k_band_residual, nb, kThreads, 0, B, sys.x, r);
        EREBUS_LAUNCH(s, k_norms2_part, NORM_BLOCKS, NORM_THREADS, 0, r, sys.rhs, np, part2);
        EREBUS_LAUNCH(s, k_norms2_sum, 1, NORM_THREADS, 0, part2, NORM_BLOCKS,
                      &s->dsc->norms[0]);
        rc = check_cuda(s, cudaMemcpyAsync(&s->hsc->norms[0], &s->dsc->norms[0], 16,
                                           cudaMemcpyDeviceToHost, s->stream), "krylov norms");
        if (!rc) rc = mf_check_error(s, sys, "krylov");
        if (rc) return rc;
        const double rr = s->hsc->norms[0], bb = s->hsc->norms[1];
        bnorm = bb > 0.0 ? sqrt(bb) : 1.0;
        rel = sqrt(rr) / bnorm;
        if (rel <= rtol || rr == 0.0) break;
        if (!(rel < INFINITY)) {
            s->last_error = std::string(sys.name) + " krylov solve: non-finite residual";
            return EREBUS_ENONFINITE;
        }
        if (cycle > 0 && rel > 0.5 * prev_cycle) {   // a whole cycle did not halve it
            if (!sys.factored) {                      // lagged factors: refresh them
                rc = refactor(s, sys);
                if (rc) return rc;
                sys.cyc_solves = 0;
                sys.cyc_iters = 0;
                at_factor = total;
                prev_cycle = INFINITY;
                continue;
            }
            stalled = true;
            break;
        }
        // within a factor 2 of the residual at which this system's solves last
        // stalled above the target: accept (every kFloorUses-th solve runs to
        // the stall again, so the floor is measured afresh)
        if (total > 0 && sys.floor_rel > 0.0 && rel <= 2.0 * sys.floor_rel &&
            sys.floor_uses < kFloorUses) {
            sys.floor_uses++;
            break;
        }
        if (total >= 3 * even && !sys.factored) {     // lagged factors no longer pay
            rc = refactor(s, sys);
            if (rc) return rc;
            sys.cyc_solves = 0;
            sys.cyc_iters = 0;
            at_factor = total;
        }
        if (total >= 40 * std::max(even, 8)) break;
        prev_cycle = rel;
        const double beta = sqrt(rr);
        EREBUS_LAUNCH(s, k_scale, nb, kThreads, 0, V, r, 1.0 / beta, np);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        for (; j < m; j++) {
            double *Vj = V + (int64_t)j * np, *Zj = Z + (int64_t)j * np;
            double *W = V + (int64_t)(j + 1) * np;
            rc = check_cuda(s, cudaMemcpyAsync(Zj, Vj, np * 8, cudaMemcpyDeviceToDevice,
                                               s->stream), "krylov copy");
            if (!rc) rc = mf_solve(s, sys, Zj);
            if (rc) return rc;
            EREBUS_LAUNCH(s, k_ell_matvec, nb, kThreads, 0, B, Zj, W);
            // classical Gram-Schmidt, twice
            EREBUS_LAUNCH(s, k_mdot_part, KB, KT, 0, V, np, j + 1, W, np, part);
            EREBUS_LAUNCH(s, k_mdot_sum, j + 1, KT, 0, part, hd, (double *)nullptr);
            EREBUS_LAUNCH(s, k_maxpy, nb, kThreads, 0, W, V, np, j + 1, hd, -1.0, np);
            EREBUS_LAUNCH(s, k_mdot_part, KB, KT, 0, V, np, j + 1, W, np, part);
            EREBUS_LAUNCH(s, k_mdot_sum, j + 1, KT, 0, part, h2, hd);
            EREBUS_LAUNCH(s, k_maxpy, nb, kThreads, 0, W, V, np, j + 1, h2, -1.0, np);
            EREBUS_LAUNCH(s, k_mdot_part, KB, KT, 0, W, np, 1, W, np, part);
            EREBUS_LAUNCH(s, k_mdot_sum, 1, KT, 0, part, nd, (double *)nullptr);
            rc = check_cuda(s, cudaMemcpyAsync(hh, hd, (j + 1) * 8,
                                               cudaMemcpyDeviceToHost, s->stream), "krylov h");
            if (!rc) rc = check_cuda(s, cudaMemcpyAsync(&hh[j + 1], nd, 8,
                                                        cudaMemcpyDeviceToHost, s->stream),
                                     "krylov h");
            if (!rc) rc = stream_sync(s, "krylov h");
            if (rc) return rc;
            total++;
            const double wn = sqrt(hh[j + 1]);
            // Givens rotations of the new Hessenberg column
            for (int i = 0; i < j; i++) {
                const double a = hh[i], b = hh[i + 1];
                hh[i] = cs[i] * a + sn[i] * b;
                hh[i + 1] = -sn[i] * a + cs[i] * b;
            }
            const double a = hh[j], d = std::hypot(a, wn);
            cs[j] = d > 0.0 ? a / d : 1.0;
            sn[j] = d > 0.0 ? wn / d : 0.0;
            hh[j] = d;
            for (int i = 0; i <= j; i++) H[(size_t)i * m + j] = hh[i];
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            const double est = fabs(g[j + 1]) / bnorm;
            if (!(wn > 0.0) || !(est < INFINITY)) { j++; break; }
            EREBUS_LAUNCH(s, k_scale, nb, kThreads, 0, W, W, 1.0 / wn, np);
            if (est <= 0.5 * rtol) { j++; break; }
        }
        if (j > m) j = m;
        // y = R^{-1} g (upper triangular, j x j), x += Z y
        for (int i = j - 1; i >= 0; i--) {
            double t = g[i];
            for (int c = i + 1; c < j; c++) t -= H[(size_t)i * m + c] * y[c];
            y[i] = t / H[(size_t)i * m + i];
        }
        rc = check_cuda(s, cudaMemcpyAsync(yd, y, j * 8, cudaMemcpyHostToDevice,
                                           s->stream), "krylov y");
        if (rc) return rc;
        EREBUS_LAUNCH(s, k_maxpy, nb, kThreads, 0, sys.x, Z, np, j, yd, 1.0, np);
        // the host vector y is read by the copy above before it is reused
        rc = stream_sync(s, "krylov update");
        if (rc) return rc;
    }
    timer_end(s, sys.ph_solve);
    sys.last_iterations = total;
    sys.krylov_iterations += total;
    sys.cyc_solves++;
    sys.cyc_iters += total - at_factor;
    sys.have_x = rel < 1e-6;
    sys.warm_ok = false;
    if (rel <= rtol) {
        sys.floor_rel = 0.0;
    } else if (stalled) {
        sys.floor_rel = rel;
        sys.floor_uses = 0;
    }
    if (st) {
        st->iterations = total;
        st->converged = rel <= rtol;
        st->rel_residual = rel;
    }
    if (!(rel <= rtol) && !(rel < 1e-6)) {
        char msg[160];
        snprintf(msg, sizeof msg,
                 "%s krylov solve did not reach tolerance: relative residual %.3e after %d "
                 "iterations", sys.name, rel, total);
        s->last_error = msg;
        return EREBUS_ENOCONV;
    }
    return EREBUS_OK;
}

void krylov_free(BandSystem &sys) {
    if (sys.kbasis) cudaFree(sys.kbasis);
    if (sys.kwork) cudaFree(sys.kwork);
    if (sys.khost) cudaFreeHost(sys.khost);
    sys.kbasis = nullptr;
    sys.kwork = nullptr;
    sys.khost = nullptr;
    sys.kdim = 0;
}

}  // namespace erebus
