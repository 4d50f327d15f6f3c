// solver.cuh -- linear systems: device assembly and the block-banded LU.
#pragma once
#include "state.cuh"

namespace erebus {

enum { SYS_HYDRO = 0, SYS_THERMAL = 1, SYS_GRAVITY = 2 };

// Device pointers to the grid fields, with the field names of the reference
// (the host struct's layout is reused for device pointers).
typedef ErebusGridHost GridPtrs;
static_assert(sizeof(ErebusGridHost) == G_COUNT * sizeof(void *), "grid struct layout");

inline GridPtrs grid_ptrs(erebus_state *s) {
    GridPtrs g;
    void **dst = reinterpret_cast<void **>(&g);
    for (int k = 0; k < G_COUNT; k++) dst[k] = s->grid[k];
    return g;
}

// Kernel-side view of a BandSystem.
struct BandView {
    int64_t n;
    int nb, NB, Bb, ell;
    double *tiles, *rhs, *rscale, *x;
    int *ell_cols;
    double *ell_vals;
};

// Address of element (r, c) (|r - c| <= half bandwidth) in tile storage:
// tile (R, C) of row R is slot C - R + Bb; tiles are column-major nb x nb.
__device__ __forceinline__ double *band_at(const BandView &B, int64_t r, int64_t c) {
    int64_t R = r / B.nb, C = c / B.nb;
    int64_t t = R * (2 * B.Bb + 1) + (C - R + B.Bb);
    return B.tiles + t * (int64_t)B.nb * B.nb + (c % B.nb) * B.nb + (r % B.nb);
}
__device__ __forceinline__ double *tile_ptr(const BandView &B, int R, int C) {
    int64_t t = (int64_t)R * (2 * B.Bb + 1) + (C - R + B.Bb);
    return B.tiles + t * (int64_t)B.nb * B.nb;
}

BandSystem &band_of(erebus_state *s, int kind);
BandView band_view(BandSystem &sys);
int band_alloc(erebus_state *s, BandSystem &sys, int64_t n, int b, int nb, int ell);
int band_free(BandSystem &sys);
int band_zero(erebus_state *s, BandSystem &sys);
int band_factor(erebus_state *s, BandSystem &sys);
// Solves A x = rhs (scaled system) into sys.x with iterative refinement
// until ||rhs - A x|| <= rtol * ||rhs|| (at most `max_ir` corrections).
int band_solve_refined(erebus_state *s, BandSystem &sys, double rtol, int max_ir,
                       ErebusSolveStats *st);
// y = A x with the assembled (unscaled) entries
int band_apply_unscaled(erebus_state *s, BandSystem &sys, const double *x, double *y);
int assemble_system(erebus_state *s, int kind);
// Hands the ELL rows just written into `sys` to its direct solver (the
// factors are recomputed at the next solve).
int commit_assembly(erebus_state *s, BandSystem &sys);
// Nested-dissection multifrontal LU (mfront.cu): factor the assembled ELL
// matrix of `sys`, solve in place, release the factor storage.
int mf_factor(erebus_state *s, BandSystem &sys, bool fp32);
bool mf_is_fp32(const BandSystem &sys);
int mf_solve(erebus_state *s, BandSystem &sys, double *w);
void mf_release(BandSystem &sys);
void mf_clear_counts(erebus_state *s, BandSystem &sys);
void mf_stats(const erebus_state *s, const BandSystem &sys, ErebusFactorStats *o);
void band_stats(const BandSystem &sys, ErebusFactorStats *o);
// Residual and norm kernels of the refinement loop (bandlu.cu), shared with
// the Krylov solves (krylov.cu).
constexpr int NORM_BLOCKS = 296, NORM_THREADS = 256;   // norm_part holds 2 x 1024
__global__ void k_band_residual(BandView B, const double *x, double *r);
__global__ void k_norms2_part(const double *a, const double *b, int64_t n, double *part);
__global__ void k_norms2_sum(const double *part, int nparts, double *out);
// Reads the device error flag of the LU kernels (synchronises the stream).
int mf_check_error(erebus_state *s, BandSystem &sys, const char *what);
// An FP32 copy of the current FP64 multifrontal factors; later triangular
// solves read the copy (until the next factorisation).
int mf_convert_fp32(erebus_state *s, BandSystem &sys);
// Mixed-precision Krylov mode (krylov.cu): flexible GMRES in FP64 with the
// multifrontal LU of an earlier matrix as preconditioner.
constexpr int KRYLOV_MAX_RESTART = 64;
int krylov_solve(erebus_state *s, BandSystem &sys, double rtol, ErebusSolveStats *st);
void krylov_free(BandSystem &sys);
// true when `sys` is factored by the multifrontal LU (else the band LU)
bool use_multifrontal(const erebus_state *s);
int export_system(erebus_state *s, int kind, int64_t *nnz, int64_t *rows, int64_t *cols,
                  double *vals, double *rhs);

}  // namespace erebus
