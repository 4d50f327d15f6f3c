// api.cu -- the extern "C" boundary of liberebus_b200.so (include/erebus_b200.h)
// and the host-side timestep driver.
//
// The timestep follows simulation_loop (src/Erebus.jl:6370-7235): every phase
// is enqueued on the state's stream; the host waits only where the
// reference makes a decision (plastic and thermochemical convergence, the
// dt updates, the new marker count).
#include <algorithm>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include "stencils.cuh"

using namespace erebus;

namespace erebus {
int check_cuda(erebus_state *s, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return EREBUS_OK;
    if (s) s->last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? EREBUS_ENOMEM : EREBUS_ECUDA;
}

int stream_sync(erebus_state *s, const char *what) {
    s->host_syncs++;
    return check_cuda(s, cudaStreamSynchronize(s->stream), what);
}

static cudaEvent_t timer_event(erebus_state *s) {
    if (!s->ev_pool.empty()) {
        cudaEvent_t e = s->ev_pool.back();
        s->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void timer_begin(erebus_state *s, int phase) {
    if (!s->timing || phase < 0 || phase >= 32) return;
    cudaEvent_t e = timer_event(s);
    cudaEventRecord(e, s->stream);
    s->ev_open[phase] = e;
}

void timer_end(erebus_state *s, int phase) {
    if (!s->timing || phase < 0 || phase >= 32 || !s->ev_open[phase]) return;
    cudaEvent_t e = timer_event(s);
    cudaEventRecord(e, s->stream);
    s->ev_pending.push_back({phase, {s->ev_open[phase], e}});
    s->ev_open[phase] = nullptr;
}

void timer_collect(erebus_state *s) {
    for (auto &p : s->ev_pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess) {
            s->phase_ms[p.first] += ms;
            s->phase_count[p.first] += 1;
        }
        s->ev_pool.push_back(p.second.first);
        s->ev_pool.push_back(p.second.second);
    }
    s->ev_pending.clear();
}

// One stream per device for the cooperative launches of states that share it.
static std::mutex g_coop_mutex;
static cudaStream_t g_coop_stream[64];

int coop_launch(erebus_state *s, const void *fn, int blocks, int threads, void **args,
                size_t smem, const char *what) {
    if (!s->shared_coop)
        return check_cuda(s, cudaLaunchCooperativeKernel(fn, blocks, threads, args, smem,
                                                         s->stream), what);
    std::lock_guard<std::mutex> lock(g_coop_mutex);
    if (s->device < 0 || s->device >= 64) return EREBUS_EINVAL;
    cudaStream_t &cs = g_coop_stream[s->device];
    if (!cs && cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
        cs = nullptr;
        return check_cuda(s, cudaErrorUnknown, "shared solver stream");
    }
    // the four calls run under the lock, so launches of different states
    // follow one another on the shared stream without interleaving
    int rc = check_cuda(s, cudaEventRecord(s->ev_to_coop, s->stream), what);
    if (!rc) rc = check_cuda(s, cudaStreamWaitEvent(cs, s->ev_to_coop, 0), what);
    if (!rc) rc = check_cuda(s, cudaLaunchCooperativeKernel(fn, blocks, threads, args, smem, cs),
                             what);
    if (!rc) rc = check_cuda(s, cudaEventRecord(s->ev_from_coop, cs), what);
    if (!rc) rc = check_cuda(s, cudaStreamWaitEvent(s->stream, s->ev_from_coop, 0), what);
    return rc;
}
}  // namespace erebus

#define TRY(x)                   \
    do {                         \
        int _rc = (x);           \
        if (_rc) return _rc;     \
    } while (0)

static bool is_basic_field(int f) { return f < G_FIRST_P; }
static bool is_bool_field(int f) { return f == G_YNY || f == G_YNY5 || f == G_YNY00; }
static bool is_basic_sum(int f) { return f < S_FIRST_P; }

static void set3(double *a, double x, double y, double z) {
    a[0] = x;
    a[1] = y;
    a[2] = z;
}

extern "C" {

// src/constants.jl (C:1-447)
int erebus_default_params(ErebusParams *p, int32_t Nx, int32_t Ny) {
    if (!p) return EREBUS_EINVAL;
    std::memset(p, 0, sizeof(*p));
    p->Nx = Nx;
    p->Ny = Ny;
    p->Nxmc = p->Nymc = 4;
    p->xsize = p->ysize = 14000.0;
    p->rplanet = 5000.0;
    p->rcrust = 4800.0;
    p->psurface = 1.0e3;
    set3(p->rhosolidm, 3300.0, 3300.0, 1.0);
    set3(p->rhofluidm, 1000.0, 1000.0, 1.0);
    set3(p->etasolidm, 1e19, 1e19, 1e16);
    set3(p->etasolidmm, 1e19, 1e19, 1e16);
    set3(p->etafluidm, 1e12, 1e12, 1e-3);
    set3(p->etafluidmm, 1e-3, 1e-3, 1e-3);
    set3(p->rhocpsolidm, 3.3e6, 3.3e6, 3.0e6);
    set3(p->rhocpfluidm, 1.0e6, 1.0e6, 3.0e6);
    set3(p->alphasolidm, 3.0e-5, 3.0e-5, 0.0);
    set3(p->alphafluidm, 5.0e-5, 5.0e-5, 0.0);
    set3(p->ksolidm, 3.0, 3.0, 3000.0);
    set3(p->kfluidm, 50.0, 50.0, 3000.0);
    set3(p->start_hrsolidm, 0.0, 0.0, 0.0);
    set3(p->start_hrfluidm, 0.0, 0.0, 0.0);
    set3(p->gggsolidm, 1e10, 1e10, 1e10);
    set3(p->frictsolidm, 0.6, 0.6, 0.0);
    set3(p->cohessolidm, 1e8, 1e8, 1e8);
    set3(p->tenssolidm, 6e7, 6e7, 6e7);
    set3(p->kphim0, 1e-13, 1e-13, 1e-17);
    set3(p->tkm0, 170.0, 170.0, 170.0);
    set3(p->XWsolidm_init, 0.5, 0.5, NAN);
    p->marker_property_mode = 9;
    p->reaction_rate_coeff_mode = 1;
    p->etaphikoef = 1.0;
    p->hr_al = 1;
    p->hr_fe = 0;
    p->t_half_al = 717000.0 * 31540000.0;
    p->ratio_al = 5.0e-5;
    p->E_al = 5.0470e-13;
    p->f_al = 1.9e23;
    p->t_half_fe = 2620000.0 * 31540000.0;
    p->ratio_fe = 1.0e-6;
    p->E_fe = 4.34e-13;
    p->f_fe = 1.957e24;
    p->tmsolidphase = 1416.0;
    p->tmfluidphase = 273.0;
    p->Lf = 333.55e3;
    p->phim0 = 0.2;
    p->phimin = 1.0e-4;
    p->phimax = 1.0 - p->phimin;
    p->RG = 8.314;
    p->MH2O = 0.018;
    p->MD = 0.120;
    p->rhoDs = 3300.0;
    p->rhoWs = 2600.0;
    p->rhoH2Of = 1000.0;
    p->rhoH2Ofi = 917.0;
    p->dHWD = 40000.0;
    p->dSWD = 60.0;
    p->pfcoeff = 0.5;
    p->pferrmax = 1.0e5;
    p->reaction_active = 1;
    p->dtreaction = 1.0e10;
    p->log_completion_rate = std::log(0.01);
    p->A_I = 1.0e-11;
    p->b_I = 2.5e-4;
    p->c_I = 543.0;
    p->Sxo_B = 2.0e-11;
    p->Tscl_B = 10.0;
    p->To_B = 293.0;
    p->Sxo_T = 2.0e-11;
    p->To_T = 293.0;
    p->Ea_T = 63.8e3;
    p->bcleft = p->bcright = p->bctop = p->bcbottom = -1.0;
    p->bcfleft = p->bcfright = p->bcftop = p->bcfbottom = -1.0;
    p->strainrate = 0.0;
    p->G = 6.672e-11;
    p->Kcont = 1.0e20;
    p->dt_longest = 1.0e11;
    p->dtcoefdn = 0.5;
    p->dtcoefup = 1.2;
    p->dtstep = 200;
    p->nplast = 100000;
    p->dxymax = 0.05;
    p->DTmax = 20.0;
    p->dsubgridt = p->dsubgrids = 0.0;
    const double yearlength = 365.25 * 24 * 3600;
    p->start_time = 2.25e6 * yearlength;
    p->endtime = 15.0e6 * yearlength;
    p->etamin = 1e12;
    p->etamax = 1e23;
    p->titermax = 10000;
    p->random_markers = 1;
    p->yerrmax = 1e2;
    p->etawt = 0.0;
    p->dphimax = 100.01;
    p->seed = 42;
    p->per_marker_eta = 0;
    return EREBUS_OK;
}

int erebus_default_solver_options(ErebusSolverOptions *o) {
    if (!o) return EREBUS_EINVAL;
    o->hydro_rtol = 1e-13;
    o->thermal_rtol = 1e-13;
    o->gravity_rtol = 1e-13;
    o->max_refinements = 8;   // refinement stops earlier once a step stops paying
    o->reuse_factors = 1;
    o->direct_solver = EREBUS_SOLVER_MULTIFRONTAL;
    o->factor_fp32 = 0;
    o->krylov = 0;
    o->precond_fp32 = 0;
    o->krylov_restart = 30;
    o->refactor_iterations = 0;
    o->mf_leaf_vector = 0;
    o->mf_leaf_scalar = 0;
    o->mf_local_factor_ops = 0;
    o->mf_local_solve_tiles = 0;
    o->mf_block_substitution = 0;
    return EREBUS_OK;
}

int erebus_check_params(const ErebusParams *p) {
    if (!p) return EREBUS_EINVAL;
    if (p->Nx < 4 || p->Ny < 4 || p->Nx != p->Ny) return EREBUS_EINVAL;
    if (!(p->xsize > 0) || p->xsize != p->ysize) return EREBUS_EINVAL;
    if (p->Nxmc < 1 || p->Nymc < 1) return EREBUS_EINVAL;
    if (p->marker_property_mode != 1 && p->marker_property_mode != 9) return EREBUS_EINVAL;
    int rm = p->reaction_rate_coeff_mode;
    if (rm != 1 && rm != 2 && rm != 3 && rm != 9) return EREBUS_EINVAL;
    if (p->dtstep < 1 || p->titermax < 1 || p->nplast < 1) return EREBUS_EINVAL;
    if (!(p->dsubgridt >= 0.0) || !(p->dsubgrids >= 0.0)) return EREBUS_EINVAL;
    return EREBUS_OK;
}

const char *erebus_last_error(const erebus_state *s) {
    return s ? s->last_error.c_str() : "null state";
}

int erebus_destroy(erebus_state *s) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->post_graph) cudaGraphExecDestroy(s->post_graph);
    for (void *p : s->allocations) cudaFree(p);
    band_free(s->hydro);
    band_free(s->thermal);
    band_free(s->gravity);
    band_free(s->heat_adjoint);
    if (s->adj_mem) cudaFree(s->adj_mem);
    if (s->hsc) cudaFreeHost(s->hsc);
    if (s->copy_stream) {
        s->host_syncs++;
        cudaStreamSynchronize(s->copy_stream);
        cudaStreamDestroy(s->copy_stream);
        cudaEventDestroy(s->snap_ready);
        cudaEventDestroy(s->snap_done);
    }
    if (s->snap_dev) cudaFree(s->snap_dev);
    if (s->snap_tm) cudaFreeHost(s->snap_tm);
    if (s->tm64) cudaFree(s->tm64);
    if (s->ev_to_coop) cudaEventDestroy(s->ev_to_coop);
    if (s->ev_from_coop) cudaEventDestroy(s->ev_from_coop);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return EREBUS_OK;
}

int erebus_share_solver_stream(erebus_state *s, int32_t on) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    if (on && !s->ev_to_coop) {
        if (cudaEventCreateWithFlags(&s->ev_to_coop, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->ev_from_coop, cudaEventDisableTiming) != cudaSuccess) {
            s->last_error = "share_solver_stream: event creation failed";
            return EREBUS_ECUDA;
        }
    }
    s->shared_coop = on != 0;
    return EREBUS_OK;
}

int erebus_grid_layout(const ErebusParams *p, int64_t *offsets, int64_t *total_bytes) {
    if (!p || !offsets || p->Nx < 2 || p->Ny < 2) return EREBUS_EINVAL;
    int64_t nb = (int64_t)p->Nx * p->Ny, np = (int64_t)(p->Nx + 1) * (p->Ny + 1), o = 0;
    for (int f = 0; f < G_COUNT; f++) {
        int64_t n = is_basic_field(f) ? nb : np;
        int64_t b = is_bool_field(f) ? n : n * 8;
        offsets[f] = o;
        o += (b + 255) / 256 * 256;
    }
    if (total_bytes) *total_bytes = o;
    return EREBUS_OK;
}

int erebus_create(const ErebusParams *p, int64_t marker_capacity, erebus_state **out) {
    if (!p || !out || marker_capacity < 1 || marker_capacity > (int64_t)1 << 30)
        return EREBUS_EINVAL;
    *out = nullptr;
    int rc = erebus_check_params(p);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return EREBUS_ENODEVICE;
    erebus_state *s = new erebus_state();
    s->p = *p;
    erebus_default_solver_options(&s->opt);
    s->g = make_geo(*p);
    s->capacity = marker_capacity;
    s->dt = p->dt_longest;
    s->timesum = p->start_time;
    cudaGetDevice(&s->device);
    auto fail = [&](int code, const char *what) {
        s->last_error = std::string("erebus_create: ") + what;
        erebus_destroy(s);
        return code;
    };
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(EREBUS_ECUDA, "stream");
    auto alloc = [&](size_t bytes) -> void * {
        void *ptr = nullptr;
        if (cudaMalloc(&ptr, bytes) != cudaSuccess) return nullptr;
        cudaMemset(ptr, 0, bytes);
        s->allocations.push_back(ptr);
        return ptr;
    };
    const Geo &g = s->g;
    size_t cap = (size_t)marker_capacity;
    size_t np = (size_t)g.Nx1 * g.Ny1, nbn = (size_t)g.Nx * g.Ny;
    for (int f = 0; f < M_COUNT; f++) {
        if (f == M_tm) continue;
        s->m[f] = (double *)alloc(cap * 8);
        if (!s->m[f]) return fail(EREBUS_ENOMEM, "markers");
    }
    s->tm8 = (int8_t *)alloc(cap);
    if (!s->tm8) return fail(EREBUS_ENOMEM, "markers");
    s->wcache = (double *)alloc(cap * 16 * sizeof(double));
    if (!s->wcache) return fail(EREBUS_ENOMEM, "marker weights");
    {   // one slab in the layout of erebus_grid_layout
        int64_t off[G_COUNT], total = 0;
        erebus_grid_layout(p, off, &total);
        char *slab = (char *)alloc((size_t)total);
        if (!slab) return fail(EREBUS_ENOMEM, "grid");
        for (int f = 0; f < G_COUNT; f++) s->grid[f] = (double *)(slab + off[f]);
    }
    (void)nbn;
    for (int f = 0; f < S_COUNT; f++) {
        s->sums[f] = (double *)alloc((is_basic_sum(f) ? nbn : np) * 8);
        if (!s->sums[f]) return fail(EREBUS_ENOMEM, "sums");
    }
    for (int gr = 0; gr < 4; gr++) {
        GridSpec sp = grid_spec(g, gr);
        CellSort &cs = s->sort[gr];
        cs.ncells = sp.rows * sp.cols;
        cs.count = (int *)alloc((cs.ncells + 1) * 4);
        cs.cursor = (int *)alloc((cs.ncells + 1) * 4);
        cs.start = (int *)alloc((cs.ncells + 1) * 4);
        cs.idx = (int *)alloc(cap * 4);
        cs.tmp = (int *)alloc(cap * 4);
        if (!cs.count || !cs.cursor || !cs.start || !cs.idx || !cs.tmp)
            return fail(EREBUS_ENOMEM, "sort");
    }
    s->r_dM = (double *)alloc(cap * 8);
    s->r_dH = (double *)alloc(cap * 8);
    s->r_flag = (int8_t *)alloc(cap);
    s->tmp_node = (double *)alloc(2 * np * 8);
    s->norm_part = (double *)alloc(2 * 1024 * 8);
    size_t na = (size_t)g.Nxm * g.Nym;
    s->a_mdis = (unsigned long long *)alloc(na * 8);
    s->a_mnum = (int *)alloc(na * 4);
    s->a_src = (int *)alloc(na * 4);
    s->a_rank = (int *)alloc(na * 4);
    s->a_flag = (int *)alloc(na * 4);
    s->a_part = (int *)alloc((na / 1024 + 2) * 4);
    s->dsc = (DevScalars *)alloc(sizeof(DevScalars));
    if (!s->r_dM || !s->r_dH || !s->r_flag || !s->tmp_node || !s->norm_part || !s->a_mdis || !s->a_mnum ||
        !s->a_src || !s->a_rank || !s->a_flag || !s->a_part || !s->dsc)
        return fail(EREBUS_ENOMEM, "scratch");
    if (cudaMallocHost(&s->hsc, sizeof(DevScalars)) != cudaSuccess)
        return fail(EREBUS_ENOMEM, "pinned scalars");
    std::memset(s->hsc, 0, sizeof(DevScalars));
    if (band_alloc(s, s->hydro, 6 * (int64_t)np, 6 * g.Ny1 + 2, 64, 12))
        return fail(EREBUS_ENOMEM, "hydro system");
    s->hydro.dofs = 6;
    s->hydro.name = "Stokes-Darcy";
    s->thermal.name = "heat";
    s->gravity.name = "gravity";
    if (band_alloc(s, s->thermal, (int64_t)np, g.Ny1, 64, 5))
        return fail(EREBUS_ENOMEM, "thermal system");
    if (band_alloc(s, s->gravity, (int64_t)np, g.Ny1, 64, 5))
        return fail(EREBUS_ENOMEM, "gravity system");
    s->hydro.ph_factor = PH_HYDRO_FACTOR;
    s->hydro.ph_solve = PH_HYDRO_SOLVE;
    s->hydro.ph_precond = PH_HYDRO_PRECOND;
    s->thermal.ph_factor = PH_THERMAL_FACTOR;
    s->thermal.ph_solve = PH_THERMAL_SOLVE;
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(EREBUS_ECUDA, "init");
    *out = s;
    return EREBUS_OK;
}

int erebus_factor_stats(erebus_state *s, int32_t system, ErebusFactorStats *out) {
    if (!s || !out || system < 0 || system > 2) return EREBUS_EINVAL;
    BandSystem &sys = band_of(s, system);
    std::memset(out, 0, sizeof(*out));
    out->direct_solver = s->opt.direct_solver;
    if (use_multifrontal(s)) mf_stats(s, sys, out);
    else band_stats(sys, out);
    out->unknowns = sys.n;
    out->factorizations = sys.factorizations;
    out->fp64_refactorizations = sys.fp64_refactorizations;
    out->krylov_iterations = sys.krylov_iterations;
    return EREBUS_OK;
}

int erebus_set_solver_options(erebus_state *s, const ErebusSolverOptions *o) {
    if (!s || !o) return EREBUS_EINVAL;
    if (o->direct_solver != EREBUS_SOLVER_MULTIFRONTAL && o->direct_solver != EREBUS_SOLVER_BAND)
        return EREBUS_EINVAL;
    if (o->mf_leaf_vector < 0 || o->mf_leaf_scalar < 0 || o->mf_local_factor_ops < 0 ||
        o->mf_local_solve_tiles < 0 ||
        (o->mf_block_substitution != 0 && o->mf_block_substitution != 1))
        return EREBUS_EINVAL;
    if (o->krylov && (o->direct_solver != EREBUS_SOLVER_MULTIFRONTAL || o->factor_fp32 ||
                      o->krylov_restart < 1 || o->krylov_restart > KRYLOV_MAX_RESTART ||
                      o->refactor_iterations < 0))
        return EREBUS_EINVAL;
    if (o->mf_leaf_vector != s->opt.mf_leaf_vector ||
        o->mf_leaf_scalar != s->opt.mf_leaf_scalar ||
        o->mf_local_factor_ops != s->opt.mf_local_factor_ops ||
        o->mf_local_solve_tiles != s->opt.mf_local_solve_tiles ||
        o->mf_block_substitution != s->opt.mf_block_substitution) {   // analysed again
        for (BandSystem *b : {&s->hydro, &s->thermal, &s->gravity}) {
            mf_release(*b);
            b->factored = false;
        }
    }
    if (o->direct_solver != s->opt.direct_solver ||
        (o->factor_fp32 != 0) != (s->opt.factor_fp32 != 0) ||
        (o->krylov != 0) != (s->opt.krylov != 0) ||
        (o->precond_fp32 != 0) != (s->opt.precond_fp32 != 0)) {   // stale factors
        for (BandSystem *b : {&s->hydro, &s->thermal, &s->gravity}) {
            b->factored = false;
            b->has_factor = false;
        }
    }
    s->opt = *o;
    return EREBUS_OK;
}

// ---- host <-> device --------------------------------------------------------
int erebus_upload_markers(erebus_state *s, const ErebusMarkersHost *m, int64_t marknum) {
    if (!s || !m || marknum < 0 || marknum > s->capacity) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    const void *const *src = reinterpret_cast<const void *const *>(m);
    for (int f = 0; f < M_COUNT; f++) {
        if (f == M_tm) continue;
        if (!src[f]) {
            if (f == M_etasolidm_m && !s->p.per_marker_eta) continue;
            return EREBUS_EINVAL;
        }
        TRY(check_cuda(s, cudaMemcpyAsync(s->m[f], src[f], marknum * 8,
                                          cudaMemcpyHostToDevice, s->stream), "upload"));
    }
    std::vector<int8_t> t(marknum);
    for (int64_t k = 0; k < marknum; k++) {
        int64_t v = m->tm[k];
        if (v < 1 || v > 3) return EREBUS_EINVAL;
        t[k] = (int8_t)v;
    }
    TRY(check_cuda(s, cudaMemcpyAsync(s->tm8, t.data(), marknum, cudaMemcpyHostToDevice,
                                      s->stream), "upload tm"));
    TRY(stream_sync(s, "upload"));
    s->marknum = marknum;
    s->sorted_valid = false;
    return EREBUS_OK;
}

int erebus_download_markers(erebus_state *s, ErebusMarkersHost *m, int64_t *marknum) {
    if (!s || !m) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    int64_t n = s->marknum;
    void **dst = reinterpret_cast<void **>(m);
    for (int f = 0; f < M_COUNT; f++) {
        if (f == M_tm || !dst[f]) continue;
        TRY(check_cuda(s, cudaMemcpyAsync(dst[f], s->m[f], n * 8, cudaMemcpyDeviceToHost,
                                          s->stream), "download"));
    }
    std::vector<int8_t> t(n);
    TRY(check_cuda(s, cudaMemcpyAsync(t.data(), s->tm8, n, cudaMemcpyDeviceToHost, s->stream),
                   "download tm"));
    TRY(stream_sync(s, "download"));
    if (m->tm)
        for (int64_t k = 0; k < n; k++) m->tm[k] = t[k];
    if (marknum) *marknum = n;
    return EREBUS_OK;
}

static size_t field_bytes(erebus_state *s, int f) {
    size_t n = is_basic_field(f) ? (size_t)s->g.Nx * s->g.Ny : (size_t)s->g.Nx1 * s->g.Ny1;
    return is_bool_field(f) ? n : n * 8;
}

int erebus_upload_grid(erebus_state *s, const ErebusGridHost *gh) {
    if (!s || !gh) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    const void *const *src = reinterpret_cast<const void *const *>(gh);
    for (int f = 0; f < G_COUNT; f++) {
        if (!src[f]) return EREBUS_EINVAL;
        TRY(check_cuda(s, cudaMemcpyAsync(s->grid[f], src[f], field_bytes(s, f),
                                          cudaMemcpyHostToDevice, s->stream), "upload grid"));
    }
    return stream_sync(s, "upload grid");
}

int erebus_download_grid(erebus_state *s, ErebusGridHost *gh) {
    if (!s || !gh) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    void **dst = reinterpret_cast<void **>(gh);
    for (int f = 0; f < G_COUNT; f++) {
        if (!dst[f]) continue;
        TRY(check_cuda(s, cudaMemcpyAsync(dst[f], s->grid[f], field_bytes(s, f),
                                          cudaMemcpyDeviceToHost, s->stream), "download grid"));
    }
    return stream_sync(s, "download grid");
}

int erebus_download_sums(erebus_state *s, ErebusSumsHost *sh) {
    if (!s || !sh) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    void **dst = reinterpret_cast<void **>(sh);
    for (int f = 0; f < S_COUNT; f++) {
        if (!dst[f]) continue;
        size_t n = is_basic_sum(f) ? (size_t)s->g.Nx * s->g.Ny : (size_t)s->g.Nx1 * s->g.Ny1;
        TRY(check_cuda(s, cudaMemcpyAsync(dst[f], s->sums[f], n * 8, cudaMemcpyDeviceToHost,
                                          s->stream), "download sums"));
    }
    return stream_sync(s, "download sums");
}

// save_state (E:5718-5960) every savematstep timesteps (E:7106): the state is
// staged in device memory on the library's stream (so the following steps may
// overwrite it at once) and drained to the caller's host buffers on a second
// stream while the simulation goes on.
int erebus_snapshot_begin(erebus_state *s, const ErebusGridHost *gh,
                          const ErebusMarkersHost *mh) {
    if (!s || !gh || !mh || s->snap_pending) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    const void *const *gd = reinterpret_cast<const void *const *>(gh);
    for (int f = 0; f < G_COUNT; f++)
        if (!gd[f]) return EREBUS_EINVAL;
    const int64_t n = s->marknum;
    size_t need = 0;
    for (int f = 0; f < G_COUNT; f++) need += (field_bytes(s, f) + 255) / 256 * 256;
    const size_t mbytes = ((size_t)s->capacity * 8 + 255) / 256 * 256;
    need += (size_t)M_COUNT * mbytes;
    if (!s->copy_stream) {
        if (cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->snap_ready, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->snap_done, cudaEventDisableTiming) != cudaSuccess) {
            s->last_error = "snapshot: stream or event creation failed";
            return EREBUS_ECUDA;
        }
    }
    if (s->snap_cap < need) {
        if (s->snap_dev) cudaFree(s->snap_dev);
        if (s->snap_tm) cudaFreeHost(s->snap_tm);
        s->snap_dev = nullptr;
        s->snap_tm = nullptr;
        s->snap_cap = 0;
        if (cudaMalloc(&s->snap_dev, need) != cudaSuccess ||
            cudaMallocHost(&s->snap_tm, (size_t)s->capacity) != cudaSuccess) {
            s->last_error = "snapshot: staging allocation failed";
            return EREBUS_ENOMEM;
        }
        s->snap_cap = need;
    }
    // stage on the library's stream
    char *p = s->snap_dev;
    std::vector<char *> gst(G_COUNT), mst(M_COUNT);
    for (int f = 0; f < G_COUNT; f++) {
        gst[f] = p;
        TRY(check_cuda(s, cudaMemcpyAsync(p, s->grid[f], field_bytes(s, f),
                                          cudaMemcpyDeviceToDevice, s->stream), "snapshot"));
        p += (field_bytes(s, f) + 255) / 256 * 256;
    }
    void *const *mdst = reinterpret_cast<void *const *>(mh);
    for (int f = 0; f < M_COUNT; f++) {
        mst[f] = p;
        const void *src = f == M_tm ? (const void *)s->tm8 : (const void *)s->m[f];
        size_t b = f == M_tm ? (size_t)n : (size_t)n * 8;
        if (b && mdst[f]) TRY(check_cuda(s, cudaMemcpyAsync(p, src, b, cudaMemcpyDeviceToDevice,
                                                 s->stream), "snapshot"));
        p += mbytes;
    }
    TRY(check_cuda(s, cudaEventRecord(s->snap_ready, s->stream), "snapshot"));
    // drain on the copy stream
    TRY(check_cuda(s, cudaStreamWaitEvent(s->copy_stream, s->snap_ready, 0), "snapshot"));
    void *const *gdst = reinterpret_cast<void *const *>(gh);
    for (int f = 0; f < G_COUNT; f++)
        TRY(check_cuda(s, cudaMemcpyAsync(gdst[f], gst[f], field_bytes(s, f),
                                          cudaMemcpyDeviceToHost, s->copy_stream), "snapshot"));
    for (int f = 0; f < M_COUNT; f++) {
        if (f == M_tm) {
            if (n && mh->tm) TRY(check_cuda(s, cudaMemcpyAsync(s->snap_tm, mst[f], (size_t)n,
                                                     cudaMemcpyDeviceToHost, s->copy_stream),
                                  "snapshot"));
            continue;
        }
        if (!mdst[f] || !n) continue;
        TRY(check_cuda(s, cudaMemcpyAsync(mdst[f], mst[f], (size_t)n * 8,
                                          cudaMemcpyDeviceToHost, s->copy_stream), "snapshot"));
    }
    TRY(check_cuda(s, cudaEventRecord(s->snap_done, s->copy_stream), "snapshot"));
    s->snap_tm_dst = mh->tm;
    s->snap_marknum = n;
    s->snap_dt = s->dt;
    s->snap_timesum = s->timesum;
    s->snap_pending = true;
    return EREBUS_OK;
}

int erebus_snapshot_wait(erebus_state *s, int64_t *marknum, double *dt, double *timesum) {
    if (!s || !s->snap_pending) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    s->snap_pending = false;
    TRY(check_cuda(s, cudaEventSynchronize(s->snap_done), "snapshot wait"));
    if (s->snap_tm_dst)
        for (int64_t k = 0; k < s->snap_marknum; k++) s->snap_tm_dst[k] = s->snap_tm[k];
    if (marknum) *marknum = s->snap_marknum;
    if (dt) *dt = s->snap_dt;
    if (timesum) *timesum = s->snap_timesum;
    return EREBUS_OK;
}

int erebus_set_time(erebus_state *s, double dt, double timesum) {
    if (!s) return EREBUS_EINVAL;
    s->dt = dt;
    s->timesum = timesum;
    return EREBUS_OK;
}

int erebus_get_time(const erebus_state *s, double *dt, double *timesum) {
    if (!s) return EREBUS_EINVAL;
    if (dt) *dt = s->dt;
    if (timesum) *timesum = s->timesum;
    return EREBUS_OK;
}

int erebus_kernel_launches(const erebus_state *s, int64_t *count) {
    if (!s || !count) return EREBUS_EINVAL;
    *count = s->launches;
    return EREBUS_OK;
}

int erebus_host_syncs(const erebus_state *s, int64_t *count) {
    if (!s || !count) return EREBUS_EINVAL;
    *count = s->host_syncs;
    return EREBUS_OK;
}

int erebus_get_stream(const erebus_state *s, void **stream) {
    if (!s || !stream) return EREBUS_EINVAL;
    *stream = (void *)s->stream;
    return EREBUS_OK;
}

int erebus_enable_phase_timing(erebus_state *s, int32_t on) {
    if (!s) return EREBUS_EINVAL;
    cudaStreamSynchronize(s->stream);
    timer_collect(s);
    s->timing = on != 0;
    for (int k = 0; k < 32; k++) {
        s->phase_ms[k] = 0.0;
        s->phase_count[k] = 0;
    }
    return EREBUS_OK;
}

int erebus_phase_times(erebus_state *s, double *ms, int64_t *counts, int32_t n) {
    if (!s || !ms || !counts || n < 1) return EREBUS_EINVAL;
    cudaStreamSynchronize(s->stream);
    timer_collect(s);
    for (int k = 0; k < n && k < 32; k++) {
        ms[k] = s->phase_ms[k];
        counts[k] = s->phase_count[k];
    }
    return EREBUS_OK;
}

}  // extern "C"

// ---- phases -----------------------------------------------------------------
static int set_dev_dt(erebus_state *s, double dt) {
    s->hsc->dt = dt;
    return check_cuda(s, cudaMemcpyAsync(&s->dsc->dt, &s->hsc->dt, sizeof(double),
                                         cudaMemcpyHostToDevice, s->stream), "dt");
}

static int read_scalars(erebus_state *s) {
    TRY(check_cuda(s, cudaMemcpyAsync(s->hsc, s->dsc, sizeof(DevScalars),
                                      cudaMemcpyDeviceToHost, s->stream), "scalars"));
    return stream_sync(s, "scalars");
}

static double slot(const erebus_state *s, int k) { return s->hsc->maxabs[k]; }

// One solve of an assembled system: direct LU plus FP64 refinement (the
// plain path), or the mixed-precision Krylov mode.
static int solve_system(erebus_state *s, BandSystem &sys, double rtol, ErebusSolveStats *st) {
    if (s->opt.krylov) return krylov_solve(s, sys, rtol, st);
    return band_solve_refined(s, sys, rtol, s->opt.max_refinements, st);
}

extern "C" {

int erebus_markers_to_nodes(erebus_state *s, double timesum) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(markers_to_nodes(s, timesum));
    return stream_sync(s, "markers_to_nodes");
}

int erebus_gravity(erebus_state *s, ErebusSolveStats *st) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(assemble_system(s, SYS_GRAVITY));
    TRY(solve_system(s, s->gravity, s->opt.gravity_rtol, st));
    size_t np = (size_t)s->g.Nx1 * s->g.Ny1;
    TRY(check_cuda(s, cudaMemcpyAsync(s->grid[G_FI], s->gravity.x, np * 8,
                                      cudaMemcpyDeviceToDevice, s->stream), "FI"));
    TRY(gravity_post(s));
    return stream_sync(s, "gravity");
}

int erebus_thermochemical_reaction(erebus_state *s, double dt, int32_t timestep,
                                   int32_t titer) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(thermochemical_reaction(s, dt, timestep, titer));
    return stream_sync(s, "reaction");
}

int erebus_hydromech_pass(erebus_state *s, double *dt, int32_t iplast, int32_t *converged,
                          ErebusSolveStats *st) {
    if (!s || !dt) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(set_dev_dt(s, *dt));
    timer_begin(s, PH_HYDRO_ASSEMBLE);
    TRY(bulk_viscosity(s));
    TRY(assemble_system(s, SYS_HYDRO));
    timer_end(s, PH_HYDRO_ASSEMBLE);
    TRY(solve_system(s, s->hydro, s->opt.hydro_rtol, st));
    timer_begin(s, PH_HYDRO_POST);
    TRY(hydro_post(s, s->hydro.x));
    timer_end(s, PH_HYDRO_POST);
    TRY(read_scalars(s));
    double d = s->hsc->dt;
    int ynpl = s->hsc->ynpl;
    double yerr = ynpl > 0 ? std::sqrt(s->hsc->sum_ddd / ynpl) : 0.0;
    int conv = ynpl == 0 || yerr < s->p.yerrmax || iplast == s->p.nplast;
    if (!conv) {
        int rollback = iplast % s->p.dtstep == 0;
        if (rollback) d *= s->p.dtcoefdn;
        TRY(finalize_plastic(s, rollback));
        TRY(set_dev_dt(s, d));
    }
    *dt = d;
    if (converged) *converged = conv;
    return stream_sync(s, "hydromech_pass");
}

int erebus_thermal_solve(erebus_state *s, double dt, int32_t timestep, double *maxDT,
                         ErebusSolveStats *st) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(heating(s));
    if (timestep == 1) {
        size_t np = (size_t)s->g.Nx1 * s->g.Ny1 * 8;
        cudaMemcpyAsync(s->grid[G_pr0], s->grid[G_pr], np, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(s->grid[G_pf0], s->grid[G_pf], np, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(s->grid[G_ps0], s->grid[G_ps], np, cudaMemcpyDeviceToDevice, s->stream);
    }
    TRY(adiabatic(s));
    TRY(set_dev_dt(s, dt));
    timer_begin(s, PH_THERMAL_ASSEMBLE);
    TRY(assemble_system(s, SYS_THERMAL));
    timer_end(s, PH_THERMAL_ASSEMBLE);
    TRY(solve_system(s, s->thermal, s->opt.thermal_rtol, st));
    TRY(thermal_post(s, s->thermal.x));
    TRY(read_scalars(s));
    s->last_maxDT = slot(s, X_DT);
    if (maxDT) *maxDT = s->last_maxDT;
    return EREBUS_OK;
}

int erebus_nodes_to_markers(erebus_state *s, double dt, int32_t timestep) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(nodes_to_markers(s, dt, timestep));
    return stream_sync(s, "nodes_to_markers");
}

int erebus_advect_rk4(erebus_state *s, double dt) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(velocities_rotation(s));
    TRY(advect(s, dt));
    return stream_sync(s, "advect");
}

int erebus_replenish(erebus_state *s, int32_t timestep, int64_t *marknum) {
    if (!s) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    return replenish(s, timestep, marknum);
}

// One timestep (E:6370-7235).  `after_m2n` (may be NULL) is called once the
// markers->nodes phase is enqueued.
typedef int (*StepHook)(erebus_state *s, void *ctx);
static int step_impl(erebus_state *s, int32_t timestep, ErebusStepStats *st,
                     StepHook after_m2n, void *ctx) {
    const ErebusParams &p = s->p;
    ErebusStepStats stats = {};
    double worst = 0.0;
    int hydro_f0 = s->hydro.factorizations, th_f0 = s->thermal.factorizations;
    timer_begin(s, PH_MARKERS_TO_NODES);
    TRY(markers_to_nodes(s, s->timesum));
    timer_end(s, PH_MARKERS_TO_NODES);
    if (after_m2n) TRY(after_m2n(s, ctx));
    ErebusSolveStats gs = {};
    timer_begin(s, PH_GRAVITY);
    TRY(erebus_gravity(s, &gs));
    timer_end(s, PH_GRAVITY);
    stats.gravity_solves = gs.iterations;
    worst = gs.rel_residual;
    double dt = std::fmin(s->dt * p.dtcoefup, p.dt_longest);   // E:6619
    size_t npb = (size_t)s->g.Nx1 * s->g.Ny1 * 8, nbb = (size_t)s->g.Nx * s->g.Ny;
    for (int titer = 1; titer <= p.titermax; titer++) {
        stats.titer = titer;
        timer_begin(s, PH_REACTION);
        if (p.reaction_active) TRY(thermochemical_reaction(s, dt, timestep, titer));
        timer_end(s, PH_REACTION);
        // E:6658-6669
        cudaMemcpyAsync(s->grid[G_ETA00], s->grid[G_ETA], nbb * 8, cudaMemcpyDeviceToDevice,
                        s->stream);
        cudaMemcpyAsync(s->grid[G_YNY00], s->grid[G_YNY], nbb, cudaMemcpyDeviceToDevice,
                        s->stream);
        if (timestep == 1) cudaMemsetAsync(s->grid[G_BETAPHI], 0, npb, s->stream);
        cudaMemcpyAsync(s->grid[G_pr0], s->grid[G_pr], npb, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(s->grid[G_pf0], s->grid[G_pf], npb, cudaMemcpyDeviceToDevice, s->stream);
        for (int iplast = 1; iplast <= p.titermax; iplast++) {
            stats.iplast_total++;
            int conv = 0;
            ErebusSolveStats hs = {};
            TRY(erebus_hydromech_pass(s, &dt, iplast, &conv, &hs));
            stats.hydro_solves += hs.iterations;
            worst = std::fmax(worst, hs.rel_residual);
            if (conv) break;
        }
        ErebusSolveStats ts = {};
        double maxDT = 0.0;
        TRY(erebus_thermal_solve(s, dt, timestep, &maxDT, &ts));
        stats.thermal_solves += ts.iterations;
        worst = std::fmax(worst, ts.rel_residual);
        if (titer == 1 && maxDT > p.DTmax) dt *= p.DTmax * (1.0 / maxDT);   // E:4187-4197
        double pferr = slot(s, X_PFERR), dmpmax = slot(s, X_DMP);        // E:4216-4223
        if (pferr < p.pferrmax && (titer > 2 || dmpmax <= 0.0)) break;
    }
    timer_begin(s, PH_NODES_TO_MARKERS);
    TRY(nodes_to_markers(s, dt, timestep));
    TRY(velocities_rotation(s));
    timer_end(s, PH_NODES_TO_MARKERS);
    TRY(advect(s, dt));
    int64_t n = 0;
    timer_begin(s, PH_REPLENISH);
    TRY(replenish(s, timestep, &n));
    timer_end(s, PH_REPLENISH);
    s->dt = dt;
    s->timesum += dt;
    stats.marknum = s->marknum;
    stats.dt = dt;
    stats.timesum = s->timesum;
    stats.worst_rel_residual = worst;
    stats.factorizations = (s->hydro.factorizations - hydro_f0) * 1000 + (s->thermal.factorizations - th_f0);
    if (st) *st = stats;
    return EREBUS_OK;
}

int erebus_step(erebus_state *s, int32_t timestep, ErebusStepStats *st) {
    if (!s || timestep < 1) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    return step_impl(s, timestep, st, nullptr, nullptr);
}

// ---- one timestep on host arrays --------------------------------------------
// Marker fields the timestep does not change for the markers it starts with
// (replenishment only appends): the material constants, and the derived
// properties once compute_marker_properties! (E:700-750) has run.  They are
// copied back while the rest of the timestep runs.
static const int kEarlyFields[] = {
    M_rhototalm, M_rhocptotalm, M_etatotalm, M_hrtotalm, M_ktotalm, M_tkm_rhocptotalm,
    M_etafluidcur_inv_kphim, M_inv_gggtotalm, M_fricttotalm, M_cohestotalm, M_tenstotalm,
    M_rhofluidcur, M_alphasolidcur, M_alphafluidcur, M_etasolidm_m};

static bool is_early(int f) {
    for (int e : kEarlyFields)
        if (e == f) return true;
    return false;
}

__global__ void k_tm_narrow(const int64_t *tm, int8_t *tm8, int64_t n, int *err) {
    int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    int64_t t = tm[m];
    if (t < 1 || t > 3) {
        atomicExch(err, 1);
        t = 3;
    }
    tm8[m] = (int8_t)t;
}
__global__ void k_tm_widen(const int8_t *tm8, int64_t *tm, int64_t b, int64_t e) {
    int64_t m = b + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m < e) tm[m] = tm8[m];
}

// Copies the grid between the device slab and host arrays: one copy when the
// host arrays sit at the offsets of erebus_grid_layout from the first one,
// else one per field.
static int copy_grid(erebus_state *s, double *dev, const void *const *host,
                     cudaMemcpyKind kind) {
    int64_t off[G_COUNT], total = 0;
    erebus_grid_layout(&s->p, off, &total);
    const char *h0 = (const char *)host[0];
    bool slab = true;
    for (int f = 0; f < G_COUNT && slab; f++) slab = (const char *)host[f] == h0 + off[f];
    if (slab) {
        void *d = kind == cudaMemcpyHostToDevice ? (void *)dev : (void *)h0;
        const void *src = kind == cudaMemcpyHostToDevice ? (const void *)h0 : (const void *)dev;
        return check_cuda(s, cudaMemcpyAsync(d, src, (size_t)total, kind, s->stream), "grid copy");
    }
    for (int f = 0; f < G_COUNT; f++) {
        char *d = (char *)dev + off[f];
        int rc = kind == cudaMemcpyHostToDevice
                     ? check_cuda(s, cudaMemcpyAsync(d, host[f], field_bytes(s, f), kind,
                                                     s->stream), "grid copy")
                     : check_cuda(s, cudaMemcpyAsync((void *)host[f], d, field_bytes(s, f), kind,
                                                     s->stream), "grid copy");
        if (rc) return rc;
    }
    return EREBUS_OK;
}

struct HostStepCtx {
    ErebusMarkersHost *out;
    int64_t n;
};

static int early_copies(erebus_state *s, void *vctx) {
    HostStepCtx &c = *static_cast<HostStepCtx *>(vctx);
    void *const *dst = reinterpret_cast<void *const *>(c.out);
    TRY(check_cuda(s, cudaEventRecord(s->snap_ready, s->stream), "step_host"));
    TRY(check_cuda(s, cudaStreamWaitEvent(s->copy_stream, s->snap_ready, 0), "step_host"));
    if (c.n == 0) return EREBUS_OK;
    for (int f : kEarlyFields)
        if (dst[f])
            TRY(check_cuda(s, cudaMemcpyAsync(dst[f], s->m[f], c.n * 8, cudaMemcpyDeviceToHost,
                                              s->copy_stream), "step_host"));
    // tm of these markers is what was uploaded
    return check_cuda(s, cudaMemcpyAsync(c.out->tm, s->tm64, c.n * 8, cudaMemcpyDeviceToHost,
                                         s->copy_stream), "step_host");
}

int erebus_step_host(erebus_state *s, int32_t timestep, const ErebusMarkersHost *in,
                     int64_t marknum, const ErebusGridHost *gin, ErebusMarkersHost *out,
                     int64_t *marknum_out, ErebusGridHost *gout, ErebusStepStats *st) {
    if (!s || timestep < 1 || !in || !gin || !out || !gout || marknum < 0 ||
        marknum > s->capacity)
        return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    const void *const *src = reinterpret_cast<const void *const *>(in);
    void *const *dst = reinterpret_cast<void *const *>(out);
    const void *const *gsrc = reinterpret_cast<const void *const *>(gin);
    void *const *gdst = reinterpret_cast<void *const *>(gout);
    for (int f = 0; f < M_COUNT; f++) {
        bool optional = f == M_etasolidm_m && !s->p.per_marker_eta;
        if ((!src[f] || !dst[f]) && !optional) return EREBUS_EINVAL;
    }
    for (int f = 0; f < G_COUNT; f++)
        if (!gsrc[f] || !gdst[f]) return EREBUS_EINVAL;
    if (!s->copy_stream) {
        if (cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->snap_ready, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->snap_done, cudaEventDisableTiming) != cudaSuccess) {
            s->last_error = "step_host: stream or event creation failed";
            return EREBUS_ECUDA;
        }
    }
    if (s->snap_pending) return EREBUS_EINVAL;   // the copy stream is busy
    if (!s->tm64 && cudaMalloc(&s->tm64, (size_t)s->capacity * 8) != cudaSuccess) {
        s->tm64 = nullptr;
        s->last_error = "step_host: scratch allocation failed";
        return EREBUS_ENOMEM;
    }
    // host -> device: markers (tm widened to int64 on the host side, narrowed
    // and checked on the device) and the grid
    for (int f = 0; f < M_COUNT; f++) {
        if (f == M_tm || !src[f] || marknum == 0) continue;
        TRY(check_cuda(s, cudaMemcpyAsync(s->m[f], src[f], marknum * 8,
                                          cudaMemcpyHostToDevice, s->stream), "step_host"));
    }
    if (marknum > 0)
        TRY(check_cuda(s, cudaMemcpyAsync(s->tm64, in->tm, marknum * 8, cudaMemcpyHostToDevice,
                                          s->stream), "step_host"));
    TRY(copy_grid(s, s->grid[0], gsrc, cudaMemcpyHostToDevice));
    TRY(check_cuda(s, cudaMemsetAsync(&s->dsc->err, 0, sizeof(int), s->stream), "step_host"));
    if (marknum > 0)
        EREBUS_LAUNCH(s, k_tm_narrow, nblocks(marknum), kThreads, 0, s->tm64, s->tm8, marknum,
                      &s->dsc->err);
    int bad = 0;
    TRY(check_cuda(s, cudaMemcpyAsync(&bad, &s->dsc->err, sizeof(int), cudaMemcpyDeviceToHost,
                                      s->stream), "step_host"));
    TRY(stream_sync(s, "step_host"));
    if (bad) {
        s->last_error = "step_host: marker type outside 1..3";
        return EREBUS_EINVAL;
    }
    s->marknum = marknum;
    s->sorted_valid = false;
    // the timestep, with the early copies on the copy stream
    HostStepCtx ctx = {out, marknum};
    ErebusStepStats stats = {};
    int rc = step_impl(s, timestep, &stats, early_copies, &ctx);
    if (rc) {
        s->host_syncs++;
        cudaStreamSynchronize(s->copy_stream);
        return rc;
    }
    // device -> host: the rest
    const int64_t n2 = s->marknum;
    for (int f = 0; f < M_COUNT; f++) {
        if (f == M_tm || !dst[f]) continue;
        int64_t b = is_early(f) ? marknum : 0;
        if (n2 > b)
            TRY(check_cuda(s, cudaMemcpyAsync((double *)dst[f] + b, s->m[f] + b, (n2 - b) * 8,
                                              cudaMemcpyDeviceToHost, s->stream), "step_host"));
    }
    if (n2 > marknum) {
        EREBUS_LAUNCH(s, k_tm_widen, nblocks(n2 - marknum), kThreads, 0, s->tm8, s->tm64,
                      marknum, n2);
        TRY(check_cuda(s, cudaMemcpyAsync(out->tm + marknum, s->tm64 + marknum,
                                          (n2 - marknum) * 8, cudaMemcpyDeviceToHost, s->stream),
                       "step_host"));
    }
    TRY(copy_grid(s, s->grid[0], (const void *const *)gdst, cudaMemcpyDeviceToHost));
    s->host_syncs++;
    TRY(check_cuda(s, cudaStreamSynchronize(s->copy_stream), "step_host"));
    TRY(stream_sync(s, "step_host"));
    if (marknum_out) *marknum_out = n2;
    if (st) *st = stats;
    return EREBUS_OK;
}

int erebus_export_hydromech(erebus_state *s, double dt, int64_t *nnz_out, int64_t *rows,
                            int64_t *cols, double *vals, double *R) {
    if (!s || !nnz_out) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(set_dev_dt(s, dt));
    TRY(bulk_viscosity(s));   // as the next plastic pass (E:6678)
    return export_system(s, SYS_HYDRO, nnz_out, rows, cols, vals, R);
}

int erebus_apply_hydromech(erebus_state *s, double dt, const double *x, double *y) {
    if (!s || !x || !y) return EREBUS_EINVAL;
    cudaSetDevice(s->device);
    TRY(set_dev_dt(s, dt));
    TRY(bulk_viscosity(s));
    BandSystem &sys = s->hydro;
    BandView B = band_view(sys);
    // assemble into the ELL arrays without touching the factors
    int64_t n = sys.n;
    double *dx = nullptr, *dy = nullptr;
    TRY(check_cuda(s, cudaMallocAsync(&dx, n * 8, s->stream), "apply alloc"));
    TRY(check_cuda(s, cudaMallocAsync(&dy, n * 8, s->stream), "apply alloc"));
    cudaMemcpyAsync(dx, x, n * 8, cudaMemcpyHostToDevice, s->stream);
    TRY(assemble_system(s, SYS_HYDRO));
    (void)B;
    TRY(band_apply_unscaled(s, sys, dx, dy));
    cudaMemcpyAsync(y, dy, n * 8, cudaMemcpyDeviceToHost, s->stream);
    int rc = stream_sync(s, "apply");
    cudaFreeAsync(dx, s->stream);
    cudaFreeAsync(dy, s->stream);
    return rc;
}

}  // extern "C"
