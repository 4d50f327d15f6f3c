// state.cuh -- device-resident state of one planetesimal.
#pragma once
#include <string>
#include <vector>
#include "common.cuh"

namespace erebus {

// Marker fields, in the order of ErebusMarkersHost.  `tm` is stored as int8
// on the device (values 1..3) and as int64 on the host.
enum MarkerField {
    M_xm, M_ym, M_tm, M_tkm, M_sxxm, M_sxym, M_etavpm, M_phim, M_phinewm,
    M_pfm0, M_XWsolidm, M_XWsolidm0, M_rhototalm, M_rhocptotalm,
    M_etatotalm, M_hrtotalm, M_ktotalm, M_tkm_rhocptotalm,
    M_etafluidcur_inv_kphim, M_inv_gggtotalm, M_fricttotalm, M_cohestotalm,
    M_tenstotalm, M_rhofluidcur, M_alphasolidcur, M_alphafluidcur,
    M_etasolidm_m, M_COUNT
};

// Grid fields, in the order of ErebusGridHost.
enum GridField {
    G_ETA, G_ETA0, G_GGG, G_EXY, G_SXY, G_SXY0, G_wyx, G_COH, G_TEN, G_FRI,
    G_YNY, G_ETA5, G_ETA00, G_YNY5, G_YNY00, G_YNY_inv_ETA, G_DSXY, G_DSY,
    G_RHOX, G_RHOFX, G_KX, G_PHIX, G_vx, G_vxf, G_RX, G_qxD, G_gx,
    G_RHOY, G_RHOFY, G_KY, G_PHIY, G_vy, G_vyf, G_RY, G_qyD, G_gy,
    G_RHO, G_RHOCP, G_ALPHA, G_ALPHAF, G_HR, G_HA, G_HS, G_ETAP, G_GGGP,
    G_EXX, G_SXX, G_SXX0, G_tk1, G_tk2, G_DT, G_DT0,
    G_vxp, G_vyp, G_vxpf, G_vypf, G_pr, G_pf, G_ps, G_pr0, G_pf0, G_ps0,
    G_ETAPHI, G_BETAPHI, G_PHI, G_APHI, G_FI, G_DMP, G_DHP, G_XWS,
    G_EII, G_SII, G_DSXX, G_tk0, G_COUNT
};
constexpr int G_FIRST_P = G_RHOX;   // fields from here on are (Ny1,Nx1)

// Scatter sums, in the order of ErebusSumsHost.
enum SumField {
    S_ETA0SUM, S_ETASUM, S_GGGSUM, S_SXYSUM, S_COHSUM, S_TENSUM, S_FRISUM,
    S_WTSUM, S_RHOXSUM, S_RHOFXSUM, S_KXSUM, S_PHIXSUM, S_RXSUM, S_WTXSUM,
    S_RHOYSUM, S_RHOFYSUM, S_KYSUM, S_PHIYSUM, S_RYSUM, S_WTYSUM, S_RHOSUM,
    S_RHOCPSUM, S_ALPHASUM, S_ALPHAFSUM, S_HRSUM, S_GGGPSUM, S_SXXSUM,
    S_TKSUM, S_PHISUM, S_DMPSUM, S_DHPSUM, S_XWSSUM, S_WTPSUM, S_COUNT
};
constexpr int S_FIRST_P = S_RHOXSUM;

// Small device-side scalars read back by the host driver.
struct DevScalars {
    double dt;
    double maxabs[8];          // reduction slots (bits of |x| as uint64)
    double sum_ddd;            // plastic yielding error sum of squares
    double norms[2];           // residual / right-hand side sums of squares
    double norms0[2];          // the same at the start of a solve (first correction made
                               // before they are read)
    int    ynpl;
    int    repl_count;         // markers to add in replenishment
    int    err;                // device-side error flag
    int    _pad;
};
enum MaxSlot { X_APHI = 0, X_VX, X_VY, X_VXF, X_VYF, X_DT, X_PFERR, X_DMP };

// Cell-sorted marker index of one node set: the markers of cell c are
// idx[start[c] .. start[c+1]) in ascending marker number.
struct CellSort {
    int ncells;
    int *count, *start, *cursor, *idx, *tmp;
};

// Block-banded matrix (no pivoting LU) of one linear system.
struct MfDevice;   // multifrontal factor storage and plan (mfront.cu)

struct BandSystem {
    int64_t n = 0;             // unknowns
    int dofs = 1;              // unknowns per P node
    const char *name = "";     // for error messages
    int b = 0;                 // half bandwidth (max |row-col|)
    int nb = 0;                // tile size
    int NB = 0;                // tile rows/cols
    int Bb = 0;                // tile half bandwidth
    double *tiles = nullptr;   // NB * (2Bb+1) tiles of nb*nb, column-major (band LU only)
    MfDevice *mf = nullptr;    // multifrontal LU (default direct solver)
    double *rscale = nullptr;  // row scale (1/sum|row|)
    double *rhs = nullptr;     // scaled right-hand side
    double *x = nullptr;       // solution
    double *r = nullptr;       // residual / correction work
    double *d = nullptr;       // correction
    double *ell_vals = nullptr;  // scaled entries per row (ELL, width `ell`)
    int *ell_cols = nullptr;
    int ell = 0;
    double *ell_prev = nullptr;    // entries the current factors came from
    int *changed = nullptr;        // set when the assembled matrix differs
    unsigned int *bar = nullptr;   // grid barrier words
    int *err = nullptr;            // device error flag of the LU kernels
    bool factored = false;
    bool have_x = false;           // x holds a converged solution
    bool warm_ok = false;          // the last solve's starting point already met the target
    double floor_rel = 0.0;        // residual at which refinement last stalled above its
                                   // target (0: none seen since it last reached the target)
    int floor_uses = 0;            // solves accepted at that floor since it was measured
    int factorizations = 0;        // number of factorisations so far
    int fp64_refactorizations = 0; // FP64 factorisations after stalled FP32 refinement
    int ph_factor = -1, ph_solve = -1;   // timer phases of this system
    int ph_precond = -1;                 // timer phase of its triangular solves
    // Krylov mode (krylov.cu)
    bool has_factor = false;       // factors exist (possibly of an earlier matrix)
    int krylov_iterations = 0;     // FGMRES iterations so far
    int last_iterations = 0;       // iterations of this system's previous solve
    double refactor_cost = 0.0;    // modelled factorisation cost in Krylov iterations (0: not yet)
    int cyc_solves = 0;            // solves since the last factorisation
    int cyc_iters = 0;             // their iterations
    int kdim = 0;                  // restart length the basis below was allocated for
    double *kbasis = nullptr;      // V (kdim + 1 vectors) then Z (kdim vectors), np each
    double *kwork = nullptr;       // dot partials, h, y (device)
    double *khost = nullptr;       // Hessenberg column and update coefficients (page-locked)
};

}  // namespace erebus

struct erebus_state {
    ErebusParams p;
    ErebusSolverOptions opt;
    erebus::Geo g;
    int64_t capacity = 0;
    int64_t marknum = 0;
    double dt = 0.0, timesum = 0.0;
    cudaStream_t stream = nullptr;
    int device = 0;
    int64_t launches = 0;
    int64_t host_syncs = 0;                    // host waits on the state's streams
    // the Stokes-Darcy post-processing sequence as a CUDA graph (stencils.cu),
    // for the solution vector it was captured with
    cudaGraphExec_t post_graph = nullptr;
    const double *post_graph_S = nullptr;
    int64_t post_graph_launches = 0;
    std::string last_error;

    // device memory
    void *mem_markers = nullptr;
    double *m[erebus::M_COUNT] = {};   // m[M_tm] is unused (tm8 holds tm)
    int8_t *tm8 = nullptr;
    double *grid[erebus::G_COUNT] = {};   // YNY* are uint8 stored in the slots
    double *sums[erebus::S_COUNT] = {};
    std::vector<void *> allocations;

    erebus::CellSort sort[4];
    double *r_dM = nullptr, *r_dH = nullptr;   // per-marker reaction outputs
    int8_t *r_flag = nullptr;
    double *tmp_node = nullptr;                // node-sized scratch
    double *wcache = nullptr;                  // markers' weights on the 4 node sets
    double *norm_part = nullptr;               // partial sums of the residual norms
    // asynchronous snapshot (erebus_snapshot_begin / _wait)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t snap_ready = nullptr, snap_done = nullptr;
    char *snap_dev = nullptr;                  // device staging copy of the state
    int8_t *snap_tm = nullptr;                 // pinned host copy of the types
    size_t snap_cap = 0;
    bool snap_pending = false;
    int64_t snap_marknum = 0;
    double snap_dt = 0.0, snap_timesum = 0.0;
    int64_t *snap_tm_dst = nullptr;
    int64_t *tm64 = nullptr;                   // int64 marker types (erebus_step_host)
    // erebus_share_solver_stream: cooperative launches go to a per-device
    // stream shared by all states that opted in
    bool shared_coop = false;
    cudaEvent_t ev_to_coop = nullptr, ev_from_coop = nullptr;
    double *partials = nullptr;                // reduction partials
    // replenishment scratch (per marker-grid anchor)
    unsigned long long *a_mdis = nullptr;
    int *a_mnum = nullptr, *a_src = nullptr, *a_rank = nullptr, *a_flag = nullptr;
    int *a_part = nullptr;   // per-tile sums of the anchor-flag scan

    erebus::DevScalars *dsc = nullptr;    // device scalars
    erebus::DevScalars *hsc = nullptr;    // pinned host mirror

    erebus::BandSystem hydro, thermal, gravity;
    erebus::BandSystem heat_adjoint;    // transposed heat system (adjoint.cu)
    double *adj_mem = nullptr;          // adjoint tape and work arrays
    size_t adj_cap = 0;
    bool sorted_valid = false;
    double last_maxDT = 0.0;     // max|DT| of the last heat solve

    // phase timing with CUDA events on `stream` (enabled on request)
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
    cudaEvent_t ev_open[32] = {};
    double phase_ms[32] = {};
    int64_t phase_count[32] = {};
};

namespace erebus {
// Launch bookkeeping and error capture.
int check_cuda(erebus_state *s, cudaError_t e, const char *what);
// Waits for the state's stream (counted in erebus_state::host_syncs).
int stream_sync(erebus_state *s, const char *what);
#define EREBUS_LAUNCH(s, kernel, grid, block, smem, ...)                      \
    do {                                                                      \
        kernel<<<(grid), (block), (smem), (s)->stream>>>(__VA_ARGS__);        \
        (s)->launches++;                                                      \
    } while (0)

// Phases timed by the event timer (erebus_phase_times).
enum Phase {
    PH_MARKERS_TO_NODES = 0, PH_GRAVITY, PH_REACTION, PH_HYDRO_ASSEMBLE,
    PH_HYDRO_FACTOR, PH_HYDRO_SOLVE, PH_HYDRO_POST, PH_THERMAL_ASSEMBLE,
    PH_THERMAL_FACTOR, PH_THERMAL_SOLVE, PH_NODES_TO_MARKERS, PH_RK4,
    PH_BACKTRACE, PH_REPLENISH, PH_SCATTER_MERGE, PH_HYDRO_PRECOND, PH_COUNT
};
void timer_begin(erebus_state *s, int phase);
void timer_end(erebus_state *s, int phase);
void timer_collect(erebus_state *s);   // after a stream sync

// entry points of the kernel files (all enqueue on s->stream)
int markers_to_nodes(erebus_state *s, double timesum);
int thermochemical_reaction(erebus_state *s, double dt, int timestep, int titer);
int nodes_to_markers(erebus_state *s, double dt, int timestep);
int advect(erebus_state *s, double dt);
int replenish(erebus_state *s, int timestep, int64_t *marknum);
int build_cell_sort(erebus_state *s);
// P-node sums of w * vals[m] over the markers in marker order (the scatter of
// marker_to_p_nodes!, E:1814-1863), and of the weights, without normalising.
int scatter_p_values(erebus_state *s, const double *vals, double *sum, double *wt);
// Launches a grid-synchronised (cooperative) kernel for state s: on s->stream,
// or, when the state shares the solver stream, on the per-device stream that
// all such states share, ordered after s->stream's work and before its next.
int coop_launch(erebus_state *s, const void *fn, int blocks, int threads, void **args,
                size_t smem, const char *what);
}  // namespace erebus
