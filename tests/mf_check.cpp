// CPU check of the multifrontal analysis (erebus.jl_b200/csrc/mf_plan.h).
//
// Test infrastructure: built by tests/test_mf_plan.py with g++ into a
// temporary directory.  It runs the same block algorithm as the device
// solver (tile LU without pivoting with inverted diagonal tiles, extend-add
// of the children's Schur complements, forward and backward sweeps over the
// fronts) in plain loops on the host, so that the analysis (tree, unknown
// lists, extend-add maps, entry targets) is checked without a GPU.
#include <cmath>
#include <cstring>
#include <set>
#include <utility>
#include <vector>

#include "../erebus.jl_b200/csrc/mf_plan.h"
#include "../erebus.jl_b200/csrc/mf_tasks.h"

using namespace erebus;

namespace {
const int T = MF_TILE;

double *tile(std::vector<double> &S, const MfFront &F, int I, int J) {
    return &S[F.off + ((long long)J * F.Mt + I) * T * T];
}
// C (+)= sgn * A * B for 64 x 64 column-major tiles
void gemm(double *C, const double *A, const double *B, double sgn) {
    for (int c = 0; c < T; c++)
        for (int k = 0; k < T; k++) {
            double b = sgn * B[c * T + k];
            for (int r = 0; r < T; r++) C[c * T + r] += A[k * T + r] * b;
        }
}
bool invert(double *A) {   // Gauss-Jordan, no pivoting, in place
    for (int k = 0; k < T; k++) {
        double p = A[k * T + k];
        if (!(std::fabs(p) > 0.0)) return false;
        double ip = 1.0 / p;
        for (int c = 0; c < T; c++)
            if (c != k)
                for (int r = 0; r < T; r++)
                    if (r != k) A[c * T + r] -= A[k * T + r] * ip * A[c * T + k];
        for (int r = 0; r < T; r++)
            if (r != k) A[k * T + r] = -A[k * T + r] * ip;
        for (int c = 0; c < T; c++)
            if (c != k) A[c * T + k] *= ip;
        A[k * T + k] = ip;
    }
    return true;
}
// The pivot-block inversion of the device solver's cooperative levels
// (k_mf_invert, mfront.cu), step by step with the same task numbering:
// tiles below the diagonal become Y = I - L^{-1}, above it
// Z_KJ = Y'_KJ D_J^{-1} with Y' = I - (I + D^{-1} N)^{-1}.
void invert_pivots(std::vector<double> &S, const MfFront &F) {
    const int Kt = F.Kt;
    if (Kt < 2) return;
    std::vector<double> tmp(T * T);
    auto t = [&](int I, int J) { return tile(S, F, I, J); };
    auto mul = [&](double *C, const double *A, const double *B) {
        std::fill(tmp.begin(), tmp.end(), 0.0);
        gemm(tmp.data(), A, B, 1.0);
        std::memcpy(C, tmp.data(), sizeof(double) * T * T);
    };
    for (int s = 0; s < Kt; s++) {
        const int cnt = (s == 0 || s == Kt - 1) ? Kt * (Kt - 1) / 2 : 2 * s * (Kt - 1 - s);
        for (int u = 0; u < cnt; u++) {
            if (s == 0 || s == Kt - 1) {
                int J = 1;
                while ((J + 1) * J / 2 <= u) J++;
                const int K = u - J * (J - 1) / 2;
                if (s == 0) mul(t(K, J), t(K, K), t(K, J));
                else mul(t(K, J), t(K, J), t(J, J));
            } else {
                const int e = Kt - 1 - s;
                if (u < s * e) gemm(t(s + 1 + u % e, u / e), t(s + 1 + u % e, s), t(s, u / e), -1.0);
                else {
                    const int v = u - s * e, K = v % s, J = s + 1 + v / s;
                    gemm(t(K, J), t(K, s), t(s, J), -1.0);
                }
            }
        }
    }
}
int solve_inverted(const MfPlan &P, std::vector<double> &S, const double *b, double *x) {
    std::vector<double> w(b, b + P.n), fv(P.vec, 0.0), fy(P.vec, 0.0);
    for (size_t f = 0; f < P.fronts.size(); f++) {
        const MfFront &F = P.fronts[f];
        double *v = &fv[F.vec_off], *y = &fy[F.vec_off];
        const int *var = &P.vars[F.var_off];
        const int *m = &P.eamap[F.map_off];
        for (int a = 0; a < F.M; a++) {
            double s = (a < F.Kp && var[a] >= 0) ? w[var[a]] : 0.0;
            for (int q = 0; q < 2; q++) {
                int c = q == 0 ? F.c0 : F.c1;
                if (c >= 0 && m[2 * a + q] >= 0) s += fv[P.fronts[c].vec_off + P.fronts[c].Kp + m[2 * a + q]];
            }
            v[a] = s;
        }
        for (int I = 0; I < F.Kt; I++) {          // y_I = v_I - sum_K Y_IK v_K
            for (int r = 0; r < T; r++) y[I * T + r] = v[I * T + r];
            for (int K = 0; K < I; K++) {
                const double *Y = tile(S, F, I, K);
                for (int c = 0; c < T; c++)
                    for (int r = 0; r < T; r++) y[I * T + r] -= Y[c * T + r] * v[K * T + c];
            }
        }
        for (int I = F.Kt; I < F.Mt; I++) {       // update rows, 8-tile chunks when longer
            const int nc = F.Kt <= 8 ? 1 : (F.Kt + 7) / 8;
            double acc[T] = {0.0};
            for (int ch = 0; ch < nc; ch++) {
                double p[T] = {0.0};
                for (int K = ch * 8; K < (nc == 1 ? F.Kt : std::min(F.Kt, ch * 8 + 8)); K++) {
                    const double *L = tile(S, F, I, K);
                    for (int c = 0; c < T; c++)
                        for (int r = 0; r < T; r++) p[r] += L[c * T + r] * y[K * T + c];
                }
                for (int r = 0; r < T; r++) acc[r] += p[r];
            }
            for (int r = 0; r < T; r++) v[I * T + r] -= acc[r];
        }
    }
    for (size_t f = P.fronts.size(); f-- > 0;) {
        const MfFront &F = P.fronts[f];
        double *v = &fv[F.vec_off], *y = &fy[F.vec_off];
        const int *var = &P.vars[F.var_off];
        for (int a = F.Kp; a < F.M; a++) v[a] = var[a] >= 0 ? w[var[a]] : 0.0;
        std::vector<double> t(F.Kp);
        for (int K = 0; K < F.Kt; K++) {          // t_K = y_K - ring partials, 16 tiles each
            for (int r = 0; r < T; r++) t[K * T + r] = y[K * T + r];
            for (int j0 = F.Kt; j0 < F.Mt; j0 += 16) {
                double p[T] = {0.0};
                for (int J = j0; J < std::min(F.Mt, j0 + 16); J++) {
                    const double *U = tile(S, F, K, J);
                    for (int c = 0; c < T; c++)
                        for (int r = 0; r < T; r++) p[r] += U[c * T + r] * v[J * T + c];
                }
                for (int r = 0; r < T; r++) t[K * T + r] -= p[r];
            }
        }
        for (int K = 0; K < F.Kt; K++) {          // x_K = D_K^{-1} t_K - sum_J Z_KJ t_J,
            const int m = F.Kt - K;                // 8-tile chunks when longer
            const int nc = m <= 8 ? 1 : (m + 7) / 8;
            for (int r = 0; r < T; r++) v[K * T + r] = 0.0;
            for (int ch = 0; ch < nc; ch++) {
                const int j1 = nc == 1 ? F.Kt : std::min(F.Kt, K + ch * 8 + 8);
                for (int r = 0; r < T; r++) {
                    double s = 0.0;
                    for (int J = K + ch * 8; J < j1; J++) {
                        const double *Z = tile(S, F, K, J);
                        const double sg = J == K ? 1.0 : -1.0;
                        for (int c = 0; c < T; c++) s += sg * Z[c * T + r] * t[J * T + c];
                    }
                    v[K * T + r] += s;
                }
            }
        }
        for (int a = 0; a < F.k; a++) w[var[a]] = v[a];
    }
    std::memcpy(x, w.data(), sizeof(double) * P.n);
    return 0;
}
}  // namespace

extern "C" {

// Analysis statistics: fronts, levels, storage doubles, max Kt, max Mt.
int mf_check_stats(int d, int ny, int nx, int leaf, long long *out) {
    MfPlan P;
    if (!mf_analyse(P, d, ny, nx, leaf)) return 1;
    out[0] = (long long)P.fronts.size();
    out[1] = (long long)P.level_begin.size() - 1;
    out[2] = P.storage;
    out[3] = P.max_kt;
    out[4] = P.max_mt;
    return 0;
}

// Solves the ELL system (rows x ell, rows >= n; rows >= n are ignored) for
// right-hand side b (n values) into x.  Returns 0, or 1 analysis failed,
// 2 entry outside the fronts, 3 zero pivot.
// With `inverted`, every front's pivot block is inverted after its
// factorisation and the sweeps take the device's inverted form: y_P = v_P -
// Y v_P, ring products in partial sums of 16 tiles, x_K = D_K^{-1} t_K -
// sum_{J>K} Z_KJ t_J; update rows and pivot rows of more than 8 tiles sum
// 8-tile chunk partials in chunk order.
int mf_check_solve(int d, int ny, int nx, int leaf, const int *cols, const double *vals,
                   long long rows, int ell, const double *b, double *x, int inverted) {
    MfPlan P;
    if (!mf_analyse(P, d, ny, nx, leaf)) return 1;
    std::vector<long long> target;
    if (!mf_targets(P, cols, rows, ell, target)) return 2;
    std::vector<double> S(P.storage, 0.0);
    for (long long e = 0; e < rows * ell; e++)
        if (target[e] >= 0) S[target[e]] += vals[e];
    for (const MfFront &F : P.fronts)
        for (int a = F.k; a < F.Kp; a++) S[mf_elem(F, a, a)] = 1.0;
    std::vector<double> tmp(T * T);
    for (size_t f = 0; f < P.fronts.size(); f++) {
        const MfFront &F = P.fronts[f];
        for (int s = 0; s < 2; s++) {
            int c = s == 0 ? F.c0 : F.c1;
            if (c < 0) continue;
            const MfFront &C = P.fronts[c];
            const int *m = &P.eamap[F.map_off];
            for (int bb = 0; bb < F.M; bb++) {
                int jb = m[2 * bb + s];
                if (jb < 0) continue;
                for (int a = 0; a < F.M; a++) {
                    int ia = m[2 * a + s];
                    if (ia >= 0) S[mf_elem(F, a, bb)] += S[mf_elem(C, C.Kp + ia, C.Kp + jb)];
                }
            }
        }
        for (int K = 0; K < F.Kt; K++) {
            if (!invert(tile(S, F, K, K))) return 3;
            for (int I = K + 1; I < F.Mt; I++) {
                std::fill(tmp.begin(), tmp.end(), 0.0);
                gemm(tmp.data(), tile(S, F, I, K), tile(S, F, K, K), 1.0);
                std::memcpy(tile(S, F, I, K), tmp.data(), sizeof(double) * T * T);
            }
            for (int J = K + 1; J < F.Mt; J++)
                for (int I = K + 1; I < F.Mt; I++)
                    if (I < F.Kt || J < F.Kt)
                        gemm(tile(S, F, I, J), tile(S, F, I, K), tile(S, F, K, J), -1.0);
        }
        for (int J = F.Kt; J < F.Mt; J++)
            for (int I = F.Kt; I < F.Mt; I++)
                for (int K = 0; K < F.Kt; K++)
                    gemm(tile(S, F, I, J), tile(S, F, I, K), tile(S, F, K, J), -1.0);
    }
    if (inverted) {
        for (const MfFront &F : P.fronts) invert_pivots(S, F);
        return solve_inverted(P, S, b, x);
    }
    // forward sweep
    std::vector<double> w(b, b + P.n), fv(P.vec, 0.0);
    for (size_t f = 0; f < P.fronts.size(); f++) {
        const MfFront &F = P.fronts[f];
        double *v = &fv[F.vec_off];
        const int *var = &P.vars[F.var_off];
        const int *m = &P.eamap[F.map_off];
        for (int a = 0; a < F.M; a++) {
            double s = (a < F.Kp && var[a] >= 0) ? w[var[a]] : 0.0;
            for (int q = 0; q < 2; q++) {
                int c = q == 0 ? F.c0 : F.c1;
                if (c >= 0 && m[2 * a + q] >= 0) s += fv[P.fronts[c].vec_off + P.fronts[c].Kp + m[2 * a + q]];
            }
            v[a] = s;
        }
        for (int K = 0; K < F.Kt; K++)
            for (int I = K + 1; I < F.Mt; I++) {
                const double *L = tile(S, F, I, K);
                for (int c = 0; c < T; c++)
                    for (int r = 0; r < T; r++) v[I * T + r] -= L[c * T + r] * v[K * T + c];
            }
    }
    // backward sweep
    for (size_t f = P.fronts.size(); f-- > 0;) {
        const MfFront &F = P.fronts[f];
        double *v = &fv[F.vec_off];
        const int *var = &P.vars[F.var_off];
        for (int a = F.Kp; a < F.M; a++) v[a] = var[a] >= 0 ? w[var[a]] : 0.0;
        for (int K = F.Kt - 1; K >= 0; K--) {
            double t[T];
            for (int r = 0; r < T; r++) t[r] = v[K * T + r];
            for (int J = K + 1; J < F.Mt; J++) {
                const double *U = tile(S, F, K, J);
                for (int c = 0; c < T; c++)
                    for (int r = 0; r < T; r++) t[r] -= U[c * T + r] * v[J * T + c];
            }
            const double *Di = tile(S, F, K, K);
            for (int r = 0; r < T; r++) {
                double s = 0.0;
                for (int c = 0; c < T; c++) s += Di[c * T + r] * t[c];
                v[K * T + r] = s;
            }
        }
        for (int a = 0; a < F.k; a++) w[var[a]] = v[a];
    }
    std::memcpy(x, w.data(), sizeof(double) * P.n);
    return 0;
}

// Checks the cooperative solve's task maps (mf_tasks.h, the decoders the
// device solver runs) for every (Kt, Mt) with Kt <= kt_max and Kt <= Mt <=
// Kt + mt_extra (Mt >= 1), and for every front of the plans of the 41 x 41,
// 141 x 141 and 401 x 401 grids: each phase's tasks cover the phase's tiles
// exactly once, and every partial-sum slot (B1 ring partials, F1 chunks,
// chunked F2 and B2 rows) is used once and lies inside the front's storage.
// Returns the number of failures.
int mf_check_tasks(int kt_max, int mt_extra) {
    int fails = 0;
    auto check = [&](int Kt, int Mt) {
        MfFront f{};
        f.Kt = Kt;
        f.Mt = Mt;
        f.poff = 640;
        const long long end = f.poff + 64 * mf_part_slots(Kt, Mt);
        std::set<long long> used;
        auto slot = [&](long long o) {
            if (o < f.poff || o + 64 > end || !used.insert(o).second) fails++;
        };
        std::set<std::pair<int, int>> cov;
        auto tile = [&](int I, int J) {
            if (!cov.insert({I, J}).second) fails++;
        };
        // B1: ring tiles of the pivot rows
        for (int u = 0; u < mf_b1_tasks(Kt, Mt); u++) {
            int K, ch, j0, n;
            mf_b1_task(Kt, Mt, u, K, ch, j0, n);
            if (K < 0 || K >= Kt || n < 1 || j0 < Kt || j0 + n > Mt) fails++;
            for (int j = 0; j < n; j++) tile(K, j0 + j);
            slot(mf_ring_part(f, K, ch));
        }
        if ((long long)cov.size() != (long long)Kt * (Mt - Kt)) fails++;
        // F1: tiles (I, K), K < I < Kt
        cov.clear();
        for (int u = 0; u < mf_f1_tasks(Kt); u++) {
            int I, ch, k0, n;
            mf_f1_task(Kt, u, I, ch, k0, n);
            if (I < 0 || I >= Kt || ch >= mf_f1_chunks(I) || n < 0 || k0 + n > I) fails++;
            for (int i = 0; i < n; i++) tile(I, k0 + i);
            if (ch >= 1) slot(mf_f1_part(f, I, ch));
        }
        if ((long long)cov.size() != (long long)Kt * (Kt - 1) / 2) fails++;
        // F2 and B2, one task per row and chunked
        for (int chunked = 0; chunked < 2; chunked++) {
            std::set<long long> used0 = used;
            const int nrc = chunked ? mf_row_chunks(Kt) : 1;
            cov.clear();
            for (int u = 0; u < mf_f2_tasks(Kt, Mt, nrc); u++) {
                int I, ch, k0, n;
                mf_f2_task(Kt, nrc, u, I, ch, k0, n);
                if (I < Kt || I >= Mt || (n < 1 && Kt > 0) || k0 + n > Kt) fails++;
                for (int i = 0; i < n; i++) tile(I, k0 + i);
                if (nrc > 1) slot(mf_row_part(f, I, ch));
            }
            if ((long long)cov.size() != (long long)(Mt - Kt) * Kt) fails++;
            cov.clear();
            for (int u = 0; u < mf_b2_count(Kt, chunked); u++) {
                int K, ch, r, i0, n;
                mf_b2_task(Kt, chunked, u, K, ch, r, i0, n);
                if (K < 0 || K >= Kt || ch >= r || n < 1 || K + i0 + n > Kt) fails++;
                if (r > 1 && r > mf_row_chunks(Kt)) fails++;
                for (int i = 0; i < n; i++) tile(K, K + i0 + i);
                if (r > 1) slot(mf_row_part(f, K, ch));
            }
            if ((long long)cov.size() != (long long)Kt * (Kt + 1) / 2) fails++;
            used = used0;   // the two forms are alternatives
        }
    };
    for (int Kt = 0; Kt <= kt_max; Kt++)
        for (int Mt = Kt > 1 ? Kt : 1; Mt <= Kt + mt_extra; Mt++) check(Kt, Mt);
    const int grids[3] = {41, 141, 401};
    for (int g : grids)
        for (int d : {6, 1}) {
            MfPlan P;
            if (!mf_analyse(P, d, g, g, d == 6 ? 32 : 64)) {
                fails++;
                continue;
            }
            for (const MfFront &F : P.fronts) check(F.Kt, F.Mt);
        }
    return fails;
}
}
