/*
 * erebus_b200.h -- C ABI of the B200-native marker-in-cell timestep library
 * (liberebus_b200.so).
 *
 * The library replaces the per-timestep hot path of Erebus.jl (src/Erebus.jl,
 * `simulation_loop` E:6370-7235) with device-resident state and hand-written
 * sm_100a kernels.  Every entry point returns an int status (0 = OK, see
 * EREBUS_E*); nothing throws and nothing aborts.  Host arrays stay owned by
 * the caller; the library owns all device memory.  A state is not thread-safe.
 *
 * Array layouts are those of the reference: node arrays are column-major
 * (Julia `Matrix{Float64}`), element (i,j) (1-based) at linear index
 * (j-1)*rows + (i-1).  Basic-node arrays are (Ny, Nx); Vx, Vy and P arrays are
 * all (Ny1, Nx1) with Ny1 = Ny+1, Nx1 = Nx+1 (src/Erebus.jl:173-277).  Bool
 * arrays (YNY*) are one byte per element, as Julia's Array{Bool}.  Marker
 * arrays are structure-of-arrays vectors of length >= marknum; the material
 * type `tm` is Julia `Int` (int64).  Only square grids are supported
 * (Nx == Ny, xsize == ysize), as in the reference, whose axis vectors are
 * sized with the other dimension (src/constants.jl:47, :119).
 */
#ifndef EREBUS_B200_H
#define EREBUS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define EREBUS_OK               0
#define EREBUS_EINVAL           1   /* bad argument / parameter set */
#define EREBUS_ECUDA            2   /* CUDA runtime error */
#define EREBUS_ENOMEM           3   /* device allocation failed */
#define EREBUS_ECAPACITY        4   /* marker capacity exceeded (replenish) */
#define EREBUS_ENOCONV          5   /* a linear solve did not reach tolerance */
#define EREBUS_ENONFINITE       6   /* NaN/Inf found where finite data is required */
#define EREBUS_ENODEVICE        7   /* no CUDA device */

/*
 * Runtime parameter set: replaces the compile-time constants of
 * src/constants.jl (C:1-447).  Material tables are indexed by marker type
 * minus one (1 = mantle, 2 = crust, 3 = sticky air).  erebus_default_params()
 * fills the values of src/constants.jl except for the grid, which callers set.
 */
typedef struct ErebusParams {
    /* grid and geometry (C:6-33, C:104-106) */
    int32_t Nx, Ny;            /* basic grid resolution; Nx1 = Nx+1 */
    int32_t Nxmc, Nymc;        /* markers per cell in x and y */
    double  xsize, ysize;      /* model size [m] */
    double  rplanet, rcrust;   /* planet and crust radius [m] */
    double  psurface;          /* surface pressure [Pa] */
    /* material tables (C:146-186) */
    double rhosolidm[3], rhofluidm[3], etasolidm[3], etasolidmm[3];
    double etafluidm[3], etafluidmm[3], rhocpsolidm[3], rhocpfluidm[3];
    double alphasolidm[3], alphafluidm[3], ksolidm[3], kfluidm[3];
    double start_hrsolidm[3], start_hrfluidm[3], gggsolidm[3];
    double frictsolidm[3], cohessolidm[3], tenssolidm[3];
    double kphim0[3], tkm0[3], XWsolidm_init[3];
    int32_t marker_property_mode;   /* 1: T-dependent laws, 9: constants (C:188) */
    int32_t reaction_rate_coeff_mode;   /* 1, 2, 3 or 9 (C:271) */
    double etaphikoef;               /* compaction viscosity coefficient (C:190) */
    /* radiogenic heating (C:2-4, C:195-214) */
    int32_t hr_al, hr_fe;
    double t_half_al, ratio_al, E_al, f_al;
    double t_half_fe, ratio_fe, E_fe, f_fe;
    /* melting and porosity (C:216-229) */
    double tmsolidphase, tmfluidphase, Lf;
    double phim0, phimin, phimax;
    /* thermodynamics of the dehydration reaction (C:230-281) */
    double RG, MH2O, MD, rhoDs, rhoWs, rhoH2Of, rhoH2Ofi;
    double dHWD, dSWD;
    double pfcoeff, pferrmax;
    int32_t reaction_active, _pad0;
    double dtreaction, log_completion_rate;
    double A_I, b_I, c_I, Sxo_B, Tscl_B, To_B, Sxo_T, To_T, Ea_T;
    /* boundary conditions (C:283-310) */
    double bcleft, bcright, bctop, bcbottom;
    double bcfleft, bcfright, bcftop, bcfbottom;
    double strainrate;         /* vxleft..vybottom derive from it (C:303-310) */
    /* physics (C:137-143) */
    double G, Kcont;
    /* time stepping (C:311-366) */
    double dt_longest, dtcoefdn, dtcoefup;
    int32_t dtstep, nplast;
    double dxymax, DTmax, dsubgridt, dsubgrids;
    double start_time, endtime, etamin, etamax;
    int32_t titermax, random_markers;
    double yerrmax, etawt, dphimax;
    uint64_t seed;
    /* Extension with no reference counterpart: when non-zero, the solid
       viscosity of rock markers comes from the per-marker array
       `etasolidm_m` instead of the table `etasolidm[tm]` (workloads with a
       log-uniform viscosity per marker).  0 = reference behaviour. */
    int32_t per_marker_eta, _pad1;
} ErebusParams;

/*
 * Host views of the marker SoA (src/Erebus.jl:426-552).  All pointers are
 * caller-owned arrays of length >= the marker count in use.
 */
typedef struct ErebusMarkersHost {
    double  *xm, *ym;
    int64_t *tm;
    double  *tkm, *sxxm, *sxym, *etavpm, *phim, *phinewm, *pfm0;
    double  *XWsolidm, *XWsolidm0;
    double  *rhototalm, *rhocptotalm, *etatotalm, *hrtotalm, *ktotalm;
    double  *tkm_rhocptotalm, *etafluidcur_inv_kphim, *inv_gggtotalm;
    double  *fricttotalm, *cohestotalm, *tenstotalm, *rhofluidcur;
    double  *alphasolidcur, *alphafluidcur;
    double  *etasolidm_m;      /* extension; NULL unless per_marker_eta */
} ErebusMarkersHost;

/*
 * Host views of the staggered-grid state (src/Erebus.jl:147-415).  Basic
 * arrays are (Ny,Nx); all others (Ny1,Nx1).  YNY, YNY5, YNY00 are bytes.
 */
typedef struct ErebusGridHost {
    /* basic nodes */
    double *ETA, *ETA0, *GGG, *EXY, *SXY, *SXY0, *wyx, *COH, *TEN, *FRI;
    uint8_t *YNY;
    double *ETA5, *ETA00;
    uint8_t *YNY5, *YNY00;
    double *YNY_inv_ETA, *DSXY, *DSY;
    /* Vx nodes */
    double *RHOX, *RHOFX, *KX, *PHIX, *vx, *vxf, *RX, *qxD, *gx;
    /* Vy nodes */
    double *RHOY, *RHOFY, *KY, *PHIY, *vy, *vyf, *RY, *qyD, *gy;
    /* P nodes */
    double *RHO, *RHOCP, *ALPHA, *ALPHAF, *HR, *HA, *HS, *ETAP, *GGGP;
    double *EXX, *SXX, *SXX0, *tk1, *tk2, *DT, *DT0;
    double *vxp, *vyp, *vxpf, *vypf, *pr, *pf, *ps, *pr0, *pf0, *ps0;
    double *ETAPHI, *BETAPHI, *PHI, *APHI, *FI, *DMP, *DHP, *XWS;
    double *EII, *SII, *DSXX, *tk0;
} ErebusGridHost;

/*
 * Weighted sums of the marker->node scatter (src/Erebus.jl:851-923): the
 * SUM arrays the reference keeps between phases.  Exported for parity tests.
 * Basic (Ny,Nx): ETA0SUM..WTSUM; Vx/Vy/P (Ny1,Nx1): the rest.
 */
typedef struct ErebusSumsHost {
    double *ETA0SUM, *ETASUM, *GGGSUM, *SXYSUM, *COHSUM, *TENSUM, *FRISUM, *WTSUM;
    double *RHOXSUM, *RHOFXSUM, *KXSUM, *PHIXSUM, *RXSUM, *WTXSUM;
    double *RHOYSUM, *RHOFYSUM, *KYSUM, *PHIYSUM, *RYSUM, *WTYSUM;
    double *RHOSUM, *RHOCPSUM, *ALPHASUM, *ALPHAFSUM, *HRSUM, *GGGPSUM;
    double *SXXSUM, *TKSUM, *PHISUM, *DMPSUM, *DHPSUM, *XWSSUM, *WTPSUM;
} ErebusSumsHost;

/* Per linear solve statistics. */
typedef struct ErebusSolveStats {
    int32_t iterations;        /* Krylov iterations (0 for a direct solve) */
    int32_t converged;         /* 1 when the tolerance was met */
    double  rel_residual;      /* ||b - A x|| / ||b|| at exit (scaled system) */
} ErebusSolveStats;

/* Per timestep statistics (what the reference logs, E:7217-7225). */
typedef struct ErebusStepStats {
    int32_t titer;             /* thermochemical iterations taken */
    int32_t iplast_total;      /* plastic iterations summed over titer */
    int32_t hydro_solves;      /* Stokes-Darcy triangular solves (refinement steps) summed */
    int32_t thermal_solves;    /* heat-equation triangular solves summed */
    int32_t gravity_solves;    /* gravity triangular solves */
    int32_t factorizations;    /* LU factorisations (1000 * Stokes-Darcy + heat) */
    int64_t marknum;           /* markers in use after replenishment */
    double  dt;                /* timestep taken [s] */
    double  timesum;           /* model time after the step [s] */
    double  maxT;              /* max(tk2) [K] */
    double  worst_rel_residual;/* worst final relative residual of any solve */
} ErebusStepStats;

/* Solver controls.  The reference solves each system with a sparse direct
   LU (UMFPACK); here the direct solver is a no-pivot LU of the row-scaled
   system, followed by iterative refinement to the relative residual below.
   Defaults come from erebus_default_solver_options. */
#define EREBUS_SOLVER_MULTIFRONTAL 0   /* nested-dissection multifrontal LU */
#define EREBUS_SOLVER_BAND         1   /* block-banded LU in the reference's unknown order */
typedef struct ErebusSolverOptions {
    double  hydro_rtol;        /* Stokes-Darcy relative residual target */
    double  thermal_rtol;      /* heat equation relative residual target */
    double  gravity_rtol;      /* Poisson relative residual target */
    int32_t max_refinements;   /* refinement corrections per solve */
    int32_t reuse_factors;     /* 1: keep the LU factors while the scaled
                                  matrix is bitwise unchanged */
    int32_t direct_solver;     /* EREBUS_SOLVER_MULTIFRONTAL or EREBUS_SOLVER_BAND */
    int32_t factor_fp32;       /* 1: the multifrontal factors are computed and
                                  stored in FP32 (tensor-core products with three
                                  TF32 terms), residuals and refinement stay FP64 */
    /* Mixed-precision Krylov mode (no reference counterpart; multifrontal
       solver only).  With krylov = 1 each solve is a flexible GMRES in FP64
       (residuals, matrix products, orthogonalisation, the solution update)
       preconditioned by the multifrontal LU factors.  The factors are kept
       as the preconditioner after the matrix changes and computed again (in
       FP64) when they stop paying.  With refactor_iterations = 0 (default)
       that is when the previous solve's iterations times the solves since
       the last factorisation reach the factorisation's cost (modelled from
       the plan, in iterations) plus those solves' iterations, i.e. when a
       solve costs as much as the average solve since the factorisation,
       the factorisation included; with refactor_iterations = n > 0, when
       the previous solve needed more than n iterations.  A solve that
       reaches three times that break-even count without converging
       refactors on the spot.  With precond_fp32 = 1 the
       Stokes-Darcy preconditioner is applied from an FP32 copy of those FP64
       factors (half the bytes per triangular solve); the heat and gravity
       systems, whose solves are short, keep applying FP64 factors.  The
       residual targets above apply unchanged. */
    int32_t krylov;            /* 1: FGMRES with lagged LU preconditioner */
    int32_t precond_fp32;      /* 1: apply the preconditioner from FP32 factors */
    int32_t krylov_restart;    /* FGMRES restart length (1..64) */
    int32_t refactor_iterations; /* 0: cost rule above; n > 0: after a solve that took more than n */
    /* Multifrontal analysis (no reference counterpart), 0 = the built-in
       default; erebus_b200.autotune picks them per grid size by timing.
       Changing them takes effect at the next analysis (a new state, or a
       direct_solver / precision change). */
    int32_t mf_leaf_vector;       /* nested-dissection leaf size, nodes, Stokes-Darcy (32) */
    int32_t mf_leaf_scalar;       /* the same for the heat and gravity systems (64) */
    int32_t mf_local_factor_ops;  /* a level factors one front per CTA when a CTA's
                                     share is at most this many tile operations (8) */
    int32_t mf_local_solve_tiles; /* ... and solves so when at most this many tiles (64) */
    /* Levels solved cooperatively (by all CTAs): 0 (default) inverts their
       fronts' pivot blocks after the factorisation, so each triangular
       sweep of a level is two rounds of independent row-block products;
       1 keeps the block substitution, a chain of dependent pivot blocks per
       front. */
    int32_t mf_block_substitution;
} ErebusSolverOptions;

/* Size and work of one system's direct solver (diagnostics; no reference
   counterpart).  flops counts the FP64 multiply-adds of the 64 x 64 tile
   algorithm (2 flops each, padding included); solve_bytes is the factor
   storage one forward plus backward solve reads. */
#define EREBUS_SYSTEM_HYDRO   0
#define EREBUS_SYSTEM_THERMAL 1
#define EREBUS_SYSTEM_GRAVITY 2
typedef struct ErebusFactorStats {
    int32_t direct_solver;     /* EREBUS_SOLVER_* in use */
    int32_t fronts;            /* multifrontal fronts (0 for the band LU) */
    int32_t levels;            /* tree levels (band LU: tile rows) */
    int32_t factorizations;    /* factorisations so far */
    int32_t fp64_refactorizations; /* mixed precision: matrices factored again in
                                      FP64 because refinement with the FP32
                                      factors stalled */
    int32_t krylov_iterations; /* FGMRES iterations so far (krylov mode) */
    int64_t unknowns;
    int64_t storage_bytes;     /* factor storage */
    double  flops;             /* per factorisation */
    double  solve_bytes;       /* per solve */
} ErebusFactorStats;

/* Statistics of one erebus_adjoint_heat call. */
typedef struct ErebusAdjointStats {
    int32_t steps;             /* timesteps run forward and reversed */
    int32_t checkpoints;       /* marker-temperature checkpoints stored */
    int32_t adjoint_solves;    /* triangular solves of the transposed heat systems */
    int32_t factorizations;    /* factorisations of the transposed heat systems */
    int64_t markers;           /* entries written to dJ_dphim */
    double  J;                 /* objective after the last timestep [K] */
    double  body_nodes;        /* basic nodes inside the body (J's average) */
} ErebusAdjointStats;

typedef struct erebus_state erebus_state;

/* ---- parameters --------------------------------------------------------- */
/* Fills *p with the values of src/constants.jl (C:1-447) for the given
   grid; derived quantities (dx, axes, marker grid) follow from the fields. */
int erebus_default_params(ErebusParams *p, int32_t Nx, int32_t Ny);
int erebus_default_solver_options(ErebusSolverOptions *o);
/* Checks a parameter set (square grid, sizes, table values). */
int erebus_check_params(const ErebusParams *p);

/* ---- lifecycle (replaces the setup_* allocators E:55-592, E:851, E:2976) */
int erebus_create(const ErebusParams *p, int64_t marker_capacity,
                  erebus_state **out);
/* Byte offsets of the grid arrays (ErebusGridHost order) in one block of
   *total_bytes: each array follows the previous one at the next multiple of
   256 bytes.  The device keeps its grid in this layout; host grid arrays
   placed at these offsets from the first one are copied in one transfer by
   erebus_step_host (else one transfer per array). */
int erebus_grid_layout(const ErebusParams *p, int64_t *offsets, int64_t *total_bytes);
int erebus_destroy(erebus_state *s);
int erebus_set_solver_options(erebus_state *s, const ErebusSolverOptions *o);
/* For states advanced concurrently from several host threads (an ensemble of
   planetesimals): with on != 0 the state's grid-synchronised solver kernels
   (factorisations and triangular solves: cooperative launches whose CTAs
   wait for one another) are queued on one stream per device shared by all
   states that opted in, so that two of them are never in flight together;
   the state's other kernels stay on its own stream and overlap with other
   states' work.  on = 0 restores the default (the state's own stream).  No
   reference counterpart. */
int erebus_share_solver_stream(erebus_state *s, int32_t on);
/* Sizes and work of the direct solver of `system` (EREBUS_SYSTEM_*). */
int erebus_factor_stats(erebus_state *s, int32_t system, ErebusFactorStats *out);
/* Last CUDA/solver error text for a state (NUL-terminated, owned by state). */
const char *erebus_last_error(const erebus_state *s);

/* ---- host <-> device ---------------------------------------------------- */
int erebus_upload_markers(erebus_state *s, const ErebusMarkersHost *m,
                          int64_t marknum);
int erebus_download_markers(erebus_state *s, ErebusMarkersHost *m,
                            int64_t *marknum);
int erebus_upload_grid(erebus_state *s, const ErebusGridHost *g);
int erebus_download_grid(erebus_state *s, ErebusGridHost *g);
int erebus_download_sums(erebus_state *s, ErebusSumsHost *sums);
/* Asynchronous snapshot of the state for save_state (src/Erebus.jl:5718-5960,
   written every savematstep timesteps, src/Erebus.jl:7106).  _begin stages
   every grid field and the marker arrays whose pointer is non-NULL in device
   memory, in stream order after the work already issued, and drains them to
   the given host buffers on a second stream; it returns at once, and steps
   may follow while the copies run.  Every grid pointer must be non-NULL.
   Host buffers must stay valid until _wait, and must be page-locked for the
   copies to overlap the steps (pageable buffers make _begin wait for them).
   _wait blocks until the copies have landed, widens tm to int64 and returns
   marknum, dt and timesum as they were at _begin.  EREBUS_EINVAL: _begin
   while a snapshot is pending, or _wait with none pending. */
int erebus_snapshot_begin(erebus_state *s, const ErebusGridHost *g,
                          const ErebusMarkersHost *m);
int erebus_snapshot_wait(erebus_state *s, int64_t *marknum, double *dt,
                         double *timesum);
/* dt / timesum / timestep counters of the device-side driver. */
int erebus_set_time(erebus_state *s, double dt, double timesum);
int erebus_get_time(const erebus_state *s, double *dt, double *timesum);

/* ---- per-phase drop-ins (same semantics as the Julia functions) --------- */
/* E:6376-6604: reset_interpolated_properties!, calculate_radioactive_heating,
   compute_marker_properties! + marker_to_{basic,vx,vy,p}_nodes! over all
   markers, compute_{basic,vx,vy,p}_node_properties!,
   apply_insulating_boundary_conditions!(tk1). */
int erebus_markers_to_nodes(erebus_state *s, double timesum);
/* E:6610-6614: assemble_gravitational_lse!, LP\RP,
   process_gravitational_solution! */
int erebus_gravity(erebus_state *s, ErebusSolveStats *st);
/* E:2558-2694: perform_thermochemical_reaction! */
int erebus_thermochemical_reaction(erebus_state *s, double dt, int32_t timestep,
                                   int32_t titer);
/* E:6678-6869: one plastic pass: recompute_bulk_viscosity!,
   assemble_hydromechanical_lse! + solve, process_hydromechanical_solution!,
   compute_Aphi!, compute_fluid_velocities!, compute_displacement_timestep,
   compute_stress_strainrate!, compute_Aphi!, symmetrize_p_node_observables!,
   compute_nodal_adjustment! and (when not converged)
   finalize_plastic_iteration_pass!.  *dt is updated; *converged receives the
   value compute_nodal_adjustment! returns. */
int erebus_hydromech_pass(erebus_state *s, double *dt, int32_t iplast,
                          int32_t *converged, ErebusSolveStats *st);
/* E:6887-6927: compute_shear_heating!, (timestep==1 pressure copy),
   compute_adiabatic_heating!, assemble_thermal_lse! + solve, DT = tk2-tk1.
   Returns max|DT| in *maxDT. */
int erebus_thermal_solve(erebus_state *s, double dt, int32_t timestep,
                         double *maxDT, ErebusSolveStats *st);
/* E:6945-7019: DT0 copy, update_marker_viscosity!, update_marker_stress!,
   update_marker_temperature!, XWsolidm0/phim copies, update_marker_porosity!,
   update_p_nodes_melt_composition! */
int erebus_nodes_to_markers(erebus_state *s, double dt, int32_t timestep);
/* E:7026-7059: compute_velocities!, compute_rotation_rate!,
   move_markers_rk4!, backtrace_pressures_rk4! */
int erebus_advect_rk4(erebus_state *s, double dt);
/* E:7065: replenish_markers!; *marknum receives the new count.
   EREBUS_ECAPACITY when the marker capacity would be exceeded. */
int erebus_replenish(erebus_state *s, int32_t timestep, int64_t *marknum);
/* E:6370-7235: one whole timestep (all of the above in reference order,
   with the thermochemical and plastic iteration loops).  Updates the
   state's dt and timesum. */
int erebus_step(erebus_state *s, int32_t timestep, ErebusStepStats *st);
/* The same timestep on host arrays: uploads `in` (marknum markers) and `gin`,
   runs the timestep and copies the markers (*marknum_out after
   replenishment) and the grid into `out` and `gout`, which may be the same
   arrays as `in` and `gin`.  The marker fields the timestep does not change
   for the markers it starts with (material constants, and the derived
   properties once compute_marker_properties! has run) are copied back on a
   second stream while the solves run, so with page-locked host arrays part
   of the copy-out overlaps the timestep.  `out` arrays need room for the
   state's capacity.  EREBUS_EINVAL for a NULL array (etasolidm_m may be NULL
   unless per_marker_eta), a marker type outside 1..3 (nothing runs), or a
   snapshot in flight. */
int erebus_step_host(erebus_state *s, int32_t timestep, const ErebusMarkersHost *in,
                     int64_t marknum, const ErebusGridHost *gin, ErebusMarkersHost *out,
                     int64_t *marknum_out, ErebusGridHost *gout, ErebusStepStats *st);

/* ---- adjoint of the heat path (no reference counterpart) ----------------
   Runs n_steps timesteps forward from the current state (erebus_step with
   timesteps first_timestep, first_timestep+1, ...), evaluates
       J = mean over the basic nodes inside the body (distance from the centre
           < rplanet) of the 4-P-node average of tk2 after the last step
   and returns dJ/d(phim[m]) for the markers present at the call and
   dJ/d(ratio_al), by reverse-mode differentiation: transposed heat solves
   (assembled from the tape of each step's RHOCP, KX, KY, dt), the transposed
   node normalisations and marker scatters (gathers), the transposed
   temperature gather (a marker-order scatter) and the derivatives of the
   marker laws (E:700-750, E:1116-1357, E:2272-2358).  Marker temperatures are
   checkpointed every `checkpoint_every` steps and recomputed in between from
   the per-step node temperatures.

   Scope: states at mechanical rest -- self-gravity G = 0, no boundary
   strain rate, reactions off, no subgrid diffusion, zero marker stresses --
   in which velocities, porosity change and marker motion vanish, so the heat
   path is the whole first-order dependence of J on phim and ratio_al.  Other
   states return EREBUS_EINVAL before running; a forward run in which a
   time-step limiter acts, a second thermochemical iteration is taken, a
   marker moves or the marker count changes returns EREBUS_EINVAL after it
   (the state has then advanced).  dJ_dphim (marknum entries) and
   dJ_dratio_al may be NULL. */
int erebus_adjoint_heat(erebus_state *s, int32_t first_timestep, int32_t n_steps,
                        int32_t checkpoint_every, double *J, double *dJ_dphim,
                        double *dJ_dratio_al, ErebusAdjointStats *st);

/* ---- debugging / parity ----------------------------------------------- */
/* Runs recompute_bulk_viscosity! (E:3634), then assembles the Stokes-Darcy
   system of E:3089-3572 from the current device state (with the given dt),
   i.e. the system the next plastic pass solves, and copies it out as COO
   triplets (0-based,
   the reference's unknown order, entries of a row in the order of its
   updateindex! calls).  nnz_out receives the entry count; pass
   rows/cols/vals = NULL to query it.  R (may be NULL) receives the
   right-hand side (6*Ny1*Nx1). */
int erebus_export_hydromech(erebus_state *s, double dt, int64_t *nnz_out,
                            int64_t *rows, int64_t *cols, double *vals,
                            double *R);
/* Applies the device Stokes-Darcy operator y = L x (matrix-free, same
   coefficients as the assembled matrix). */
int erebus_apply_hydromech(erebus_state *s, double dt, const double *x,
                           double *y);
/* Number of kernel launches issued by this state since creation. */
int erebus_kernel_launches(const erebus_state *s, int64_t *count);
/* Number of times the host waited for this state's streams since creation
   (a timestep waits where the reference makes a decision: convergence of a
   solve or of the plastic and thermochemical iterations, the dt updates,
   the new marker count).  No reference counterpart. */
int erebus_host_syncs(const erebus_state *s, int64_t *count);
/* The CUDA stream (cudaStream_t) all work of this state is enqueued on,
   for callers that time it with their own events.  No reference
   counterpart. */
int erebus_get_stream(const erebus_state *s, void **stream);
/* Per-phase device time measured with CUDA events on the state's stream
   (no reference counterpart).  Phases, in order: markers->nodes, gravity,
   reaction, Stokes-Darcy assembly, factorisation, triangular solves and
   refinement, post-solve stencils, heat assembly, factorisation, solves,
   nodes->markers, RK4 advection, pressure back-trace, replenishment,
   scatter merge kernels, and the Stokes-Darcy triangular-solve launches
   alone (inside the solve phase).  Enabling resets the accumulators. */
int erebus_enable_phase_timing(erebus_state *s, int32_t on);
int erebus_phase_times(erebus_state *s, double *ms, int64_t *counts, int32_t n);

/* ---- allocation-free marker -> node pass ------------------------------- */
/* Device-pointer views: the same layouts as the host structs above, with
   every pointer a device address (tm is int64 on the device too). */
typedef ErebusMarkersHost ErebusMarkersDevice;
typedef ErebusGridHost ErebusGridDevice;

/* Largest problem the allocation-free pass accepts. */
#define EREBUS_NOALLOC_MAX_MARKERS 131072
#define EREBUS_NOALLOC_MAX_NODES 16384   /* (Ny+1)*(Nx+1), e.g. up to 127x127 */

/* No counterpart in the reference (an addition of this library).
   Same computation as erebus_markers_to_nodes, for callers that cannot let
   a library allocate device memory: a host framework that owns every
   device buffer through its own pool (a Julia GPU-array pool, for
   instance) or an application held to a fixed device-memory budget.  For
   them a hidden cudaMalloc would escape their accounting, can fail once
   their pool holds the device, and synchronises the whole device.
   The caller passes device pointers for all inputs and outputs: m (the
   marker SoA; the seven derived marker properties are written back into
   it) and g (the node fields of compute_{basic,vx,vy,p}_node_properties!
   and tk1; other pointers of g may be NULL).  Scratch (the cell sort and
   the weighted sums) is a file-scope device array of about 6.4 MB that
   every GPU which loads the library keeps until the process exits.  The
   call allocates nothing.  Every call looks up that array's device
   address with the calling device current (the address is not cached,
   since it can change if the device's context is reset); the first call on
   a device also loads the library's device code there, so that first call
   should come before any stream capture.
   marknum above EREBUS_NOALLOC_MAX_MARKERS or a grid with more than
   EREBUS_NOALLOC_MAX_NODES nodes returns EREBUS_ECAPACITY without
   launching anything; a marker type outside 1..3 returns EREBUS_EINVAL.
   All calls share the scratch array: calls that overlap on the GPU (two
   streams, two host threads) race and give wrong results.  `stream` is a
   cudaStream_t (NULL = legacy default stream); the call returns after the
   stream has drained. */
int erebus_markers_to_nodes_noalloc(const ErebusParams *p,
                                    const ErebusMarkersDevice *m,
                                    int64_t marknum,
                                    const ErebusGridDevice *g,
                                    double timesum, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* EREBUS_B200_H */
