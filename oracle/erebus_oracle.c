/*
 * erebus_oracle.c -- CPU oracle for the Erebus.jl timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle against which the
 * CUDA library is compared, and the timed CPU baseline of bench.py.  Nothing
 * in the product (the erebus.jl_b200 package, its CUDA library) links, loads
 * or calls it.
 *
 * It is a plain-C FP64 restatement of the functions of src/Erebus.jl that
 * one timestep runs (simulation_loop, E:6370-7235), in the reference's loop
 * order and with its arithmetic order (no fast-math, no FMA contraction), so
 * that IEEE Inf/NaN behaviour and quirks are reproduced.  Each function
 * cites the reference lines it follows.  Julia is not available here, so
 * parity of this restatement is pinned against re-expressions of the
 * reference's own unit tests (test/runtests.jl), not against outputs of the
 * reference run here.  The linear solves are done by the Python driver
 * (oracle/oracle.py) with SuperLU on the CSC systems assembled here.
 *
 * Index convention: i, j are 1-based as in the reference; AT(A,rows,i,j)
 * addresses the column-major element (i,j).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "../include/erebus_b200.h"

void oracle_thermodynamic_xfer(const ErebusParams *p, const ErebusSumsHost *s,
                               ErebusGridHost *G);
void oracle_melt_composition(const ErebusParams *p, const ErebusMarkersHost *M,
                             int64_t marknum, ErebusGridHost *G, ErebusSumsHost *s);

#define AT(A, rows, i, j) (A)[((int64_t)(j) - 1) * (rows) + ((i) - 1)]

/* ------------------------------------------------------------------------ */
/* grid geometry derived from the parameter set (src/constants.jl:25-124)   */
/* ------------------------------------------------------------------------ */
typedef struct {
    int Nx, Ny, Nx1, Ny1, Nxm, Nym;
    double dx, dy, dxm, dym, xcenter, ycenter;
    double VDs, VWs, VH2Of, VH2Ofi, dVWD, tau_al, tau_fe;
    double vxleft, vxright, vytop, vybottom;
} Geo;

static Geo geo(const ErebusParams *p) {
    Geo g;
    g.Nx = p->Nx; g.Ny = p->Ny; g.Nx1 = p->Nx + 1; g.Ny1 = p->Ny + 1;
    g.dx = p->xsize / (p->Nx - 1);
    g.dy = p->ysize / (p->Ny - 1);
    g.Nxm = (p->Nx - 1) * p->Nxmc;
    g.Nym = (p->Ny - 1) * p->Nymc;
    g.dxm = p->xsize / g.Nxm;
    g.dym = p->ysize / g.Nym;
    g.xcenter = p->xsize / 2;
    g.ycenter = p->ysize / 2;
    g.VDs = p->MD / p->rhoDs;                       /* C:247 */
    g.VWs = (p->MD + p->MH2O) / p->rhoWs;           /* C:249 */
    g.VH2Of = p->MH2O / p->rhoH2Of;                 /* C:251 */
    g.VH2Ofi = p->MH2O / p->rhoH2Ofi;               /* C:253 */
    g.dVWD = g.VDs + g.VH2Of - g.VWs;               /* C:259 */
    g.tau_al = p->t_half_al / log(2.0);             /* C:198 */
    g.tau_fe = p->t_half_fe / log(2.0);             /* C:208 */
    g.vxleft = p->strainrate * p->xsize / 2;        /* C:303 */
    g.vxright = -p->strainrate * p->xsize / 2;
    g.vytop = -p->strainrate * p->ysize / 2;
    g.vybottom = p->strainrate * p->ysize / 2;
    return g;
}

/* axis origins: basic (0,0), Vx (0,-dy/2), Vy (-dx/2,0), P (-dx/2,-dy/2)
   (C:40-65); axis[k] = origin + (k-1)*step (all configured steps are exact). */
static inline double ax(double origin, double step, int k) {
    return origin + (double)(k - 1) * step;
}

/* Julia max/min semantics for floats: NaN propagates. */
static inline double jmax(double a, double b) {
    if (a != a || b != b) return NAN;
    return a > b ? a : b;
}
static inline double jmin(double a, double b) {
    if (a != a || b != b) return NAN;
    return a < b ? a : b;
}

/* truncation toward zero as unsafe_trunc(Int, v) (NaN and overflow are
   undefined in the reference; they are mapped to a very negative index and
   clamped). */
static inline int64_t jtrunc(double v) {
    if (!(v > -4.0e18 && v < 4.0e18)) return INT64_MIN / 2;
    return (int64_t)v;
}

/* fix (E:1456-1470) */
static inline void fix(double x, double y, double x0, double y0, double dx,
                       double dy, int jmin_, int jmax_, int imin_, int imax_,
                       int *iout, int *jout) {
    int64_t j = jtrunc((x - x0) * (1.0 / dx)) + 1;
    int64_t i = jtrunc((y - y0) * (1.0 / dy)) + 1;
    if (j < jmin_) j = jmin_;
    else if (j > jmax_) j = jmax_;
    if (i < imin_) i = imin_;
    else if (i > imax_) i = imax_;
    *iout = (int)i;
    *jout = (int)j;
}

/* fix_distances (E:1424-1431) */
static inline void fix_distances(double x, double y, double x0, double y0,
                                 double dx, double dy, int jmin_, int jmax_,
                                 int imin_, int imax_, int *i, int *j,
                                 double *dxmj, double *dymi) {
    fix(x, y, x0, y0, dx, dy, jmin_, jmax_, imin_, imax_, i, j);
    *dxmj = x - ax(x0, dx, *j);
    *dymi = y - ax(y0, dy, *i);
}

/* fix_weights (E:1388-1397): weights of nodes (i,j),(i+1,j),(i,j+1),(i+1,j+1) */
static inline void fix_weights(double x, double y, double x0, double y0,
                               double dx, double dy, int jmin_, int jmax_,
                               int imin_, int imax_, int *i, int *j,
                               double w[4]) {
    double dxmj, dymi;
    fix_distances(x, y, x0, y0, dx, dy, jmin_, jmax_, imin_, imax_, i, j,
                  &dxmj, &dymi);
    w[0] = (1.0 - dymi / dy) * (1.0 - dxmj / dx);
    w[1] = (dymi / dy) * (1.0 - dxmj / dx);
    w[2] = (1.0 - dymi / dy) * (dxmj / dx);
    w[3] = (dymi / dy) * (dxmj / dx);
}

/* per-grid weights with the reference clamp ranges (C:66-101) */
enum { GB = 0, GVX = 1, GVY = 2, GP = 3 };
static inline void grid_weights(const Geo *g, int grid, double x, double y,
                                int *i, int *j, double w[4]) {
    switch (grid) {
    case GB:
        fix_weights(x, y, 0.0, 0.0, g->dx, g->dy, 1, g->Nx - 1, 1, g->Ny - 1,
                    i, j, w);
        break;
    case GVX:
        fix_weights(x, y, 0.0, -g->dy / 2, g->dx, g->dy, 1, g->Nx - 1, 1,
                    g->Ny, i, j, w);
        break;
    case GVY:
        fix_weights(x, y, -g->dx / 2, 0.0, g->dx, g->dy, 1, g->Nx, 1,
                    g->Ny - 1, i, j, w);
        break;
    default:
        fix_weights(x, y, -g->dx / 2, -g->dy / 2, g->dx, g->dy, 1, g->Nx, 1,
                    g->Ny, i, j, w);
        break;
    }
}

/* interpolate_add_to_grid! (E:1517-1525) */
static inline void add_to_grid(double *A, int rows, int i, int j,
                               const double w[4], double v) {
    AT(A, rows, i, j) += v * w[0];
    AT(A, rows, i + 1, j) += v * w[1];
    AT(A, rows, i, j + 1) += v * w[2];
    AT(A, rows, i + 1, j + 1) += v * w[3];
}

/* dot4(grid_vector(i,j,A), w) (E:1137, E:1157) */
static inline double gather4(const double *A, int rows, int i, int j,
                             const double w[4]) {
    return AT(A, rows, i, j) * w[0] + AT(A, rows, i + 1, j) * w[1] +
           AT(A, rows, i, j + 1) * w[2] + AT(A, rows, i + 1, j + 1) * w[3];
}

/* grid_average (E:1176-1180) */
static inline double grid_average(const double *A, int rows, int i, int j) {
    return 0.25 * (AT(A, rows, i, j) + AT(A, rows, i + 1, j) +
                   AT(A, rows, i, j + 1) + AT(A, rows, i + 1, j + 1));
}

/* ------------------------------------------------------------------------ */
/* pointwise material laws                                                  */
/* ------------------------------------------------------------------------ */
static inline double total(double s, double f, double phi) {   /* E:1116 */
    return s * (1.0 - phi) + f * phi;
}
static inline double ktotal(double ks, double kf, double phi) { /* E:1226 */
    double a = ks * (3.0 * phi - 2.0) + kf * (1.0 - 3.0 * phi);
    return sqrt(ks * kf / 2 + (a * a) * (1.0 / 16.0)) -
           0.25 * (ks * (3.0 * phi - 2.0) + kf * (1.0 - 3.0 * phi));
}
/* x^3.0 and x^2.0 of E:1274: Julia evaluates a Float64 power with an
   integral exponent by compensated repeated multiplication (one final
   rounding); x^2 is a single correctly rounded product. */
static inline double cube(double x) {
    double hi = x * x, lo = fma(x, x, -hi);
    double p = hi * x, e = fma(hi, x, -p);
    return p + (e + lo * x);
}
/* eta_f / k(phi), Kozeny-Carman (E:1273-1275) */
static inline double etaf_inv_kphi(const ErebusParams *p, double k0,
                                   double phi, double etaf) {
    double r = (1.0 - phi) * (1.0 / (1.0 - p->phim0));
    return etaf * (1.0 / k0) * cube(p->phim0 * (1.0 / phi)) * (r * r);
}
static inline double Q_radiogenic(double f, double ratio, double E,
                                  double tau, double time) { /* E:1294 */
    return f * ratio * E * exp(-time * (1.0 / tau)) * (1.0 / tau);
}
/* compute_rhocpfluidm (E:2272-2293) */
static inline double rhocpfluid(const ErebusParams *p, double T) {
    if (p->marker_property_mode == 1) {
        double tm = p->tmfluidphase;
        if (T < tm - 5.0) return p->rhoH2Ofi * (7.67 * T);
        if (T < tm) return p->rhoH2Ofi * (7.67 * T + 0.1 * p->Lf);
        if (T < tm + 5.0) return p->rhoH2Of * (4200.0 + 0.1 * p->Lf);
        if (T < 410.0) return p->rhoH2Of * 4200.0;
        return p->rhoH2Of *
               (-4.67e4 + 333 * T - 0.731 * (T * T) + 5.4e-4 * (T * T * T));
    }
    return p->rhocpfluidm[0];
}
/* compute_ksolidm (E:2311-2322) */
static inline double ksolid(const ErebusParams *p, double T) {
    if (p->marker_property_mode == 1) return 0.73 + 1293.0 / (T + 77.0);
    return p->ksolidm[0];
}
/* compute_kfluidm (E:2341-2358) */
static inline double kfluid(const ErebusParams *p, double T) {
    if (p->marker_property_mode == 1) {
        if (T < p->tmfluidphase) return 0.465 + 488.0 / T;
        if (T < 410) return -0.581 + 6.34e-3 * T - 7.93e-6 * (T * T);
        return -0.142 + 4.12e-3 * T - 5.01e-6 * (T * T);
    }
    return p->kfluidm[0];
}
/* compute_dtreaction (E:2382-2397) */
static inline double dtreaction_of(const ErebusParams *p, double T,
                                   double phi) {
    switch (p->reaction_rate_coeff_mode) {
    case 1: {
        double d = T - p->c_I;
        return -p->log_completion_rate / (p->A_I * phi) * exp(p->b_I * (d * d));
    }
    case 2:
        return -p->log_completion_rate / (p->Sxo_B * phi) *
               pow(2.0, (p->To_B - T) / p->Tscl_B);
    case 3:
        return -p->log_completion_rate / (p->Sxo_B * phi) *
               exp(p->Ea_T / p->RG * (1.0 / T - 1.0 / p->To_T));
    default:
        return p->dtreaction;
    }
}
/* etatotal_rocks (E:1312-1318) with the per-marker viscosity extension */
static inline double etatotal_rocks(const ErebusParams *p, double tk, int t,
                                    double eta_marker) {
    double es = tk > p->tmsolidphase ? p->etasolidmm[t - 1]
                                     : (p->per_marker_eta ? eta_marker
                                                          : p->etasolidm[t - 1]);
    double ef = tk > p->tmfluidphase ? p->etafluidmm[t - 1]
                                     : p->etafluidm[t - 1];
    return jmax(jmax(p->etamin, es), ef);
}

/* ------------------------------------------------------------------------ */
/* marker -> node scatter (E:6376-6604)                                     */
/* ------------------------------------------------------------------------ */
#define NSUMP(s) (s)

/* reset_interpolated_properties! (E:968-1035) */
static void reset_sums(const Geo *g, ErebusSumsHost *s) {
    size_t nb = (size_t)g->Nx * g->Ny, np = (size_t)g->Nx1 * g->Ny1;
    double *b[] = {s->ETA0SUM, s->ETASUM, s->GGGSUM, s->SXYSUM, s->COHSUM,
                   s->TENSUM, s->FRISUM, s->WTSUM};
    double *q[] = {s->RHOXSUM, s->RHOFXSUM, s->KXSUM, s->PHIXSUM, s->RXSUM,
                   s->WTXSUM, s->RHOYSUM, s->RHOFYSUM, s->KYSUM, s->PHIYSUM,
                   s->RYSUM, s->WTYSUM, s->RHOSUM, s->RHOCPSUM, s->ALPHASUM,
                   s->ALPHAFSUM, s->HRSUM, s->GGGPSUM, s->SXXSUM, s->TKSUM,
                   s->PHISUM, s->WTPSUM};
    for (size_t k = 0; k < sizeof b / sizeof *b; k++) memset(b[k], 0, nb * 8);
    for (size_t k = 0; k < sizeof q / sizeof *q; k++) memset(q[k], 0, np * 8);
}

/* compute_marker_properties! (E:700-750) */
static void marker_properties(const ErebusParams *p, const Geo *g,
                              ErebusMarkersHost *M, int64_t m,
                              const double hrs[3], const double hrf[3]) {
    int t = (int)M->tm[m];
    double etafluidcur;
    double tk = M->tkm[m], phi = M->phim[m];
    if (t < 3) {
        double XW = M->XWsolidm0[m];
        double XD = 1.0 - XW;
        double rhos = (p->MD + p->MH2O * XW) / (g->VDs * XD + g->VWs * XW);
        double rhof = tk > p->tmfluidphase ? p->rhoH2Of : p->rhoH2Ofi;
        M->rhototalm[m] = total(rhos, rhof, phi);
        M->rhocptotalm[m] = total(p->rhocpsolidm[t - 1], rhocpfluid(p, tk), phi);
        double es = tk > p->tmsolidphase
                        ? p->etasolidmm[t - 1]
                        : (p->per_marker_eta ? M->etasolidm_m[m]
                                             : p->etasolidm[t - 1]);
        etafluidcur = tk > p->tmfluidphase ? p->etafluidmm[t - 1]
                                           : p->etafluidm[t - 1];
        M->etatotalm[m] = jmax(jmax(p->etamin, es), etafluidcur);
        M->hrtotalm[m] = total(hrs[t - 1], hrf[t - 1], phi);
        M->ktotalm[m] = ktotal(ksolid(p, tk), kfluid(p, tk), phi);
    } else {
        etafluidcur = p->etafluidm[t - 1];
    }
    M->tkm_rhocptotalm[m] = tk * M->rhocptotalm[m];
    M->etafluidcur_inv_kphim[m] =
        etaf_inv_kphi(p, p->kphim0[t - 1], phi, etafluidcur);
}

/* calculate_radioactive_heating (E:1336-1357) */
static void radioactive_heating(const ErebusParams *p, const Geo *g,
                                double timesum, double hrs[3], double hrf[3]) {
    hrs[0] = hrs[1] = hrs[2] = 0.0;
    hrf[0] = hrf[1] = hrf[2] = 0.0;
    if (p->hr_al) {
        double Q = Q_radiogenic(p->f_al, p->ratio_al, p->E_al, g->tau_al,
                                timesum);
        hrs[0] = Q * p->rhosolidm[0];
        hrs[1] = Q * p->rhosolidm[1];
    }
    if (p->hr_fe) {
        double Q = Q_radiogenic(p->f_fe, p->ratio_fe, p->E_fe, g->tau_fe,
                                timesum);
        hrf[0] = Q * p->rhofluidm[0];
    }
}

/* marker_to_{basic,vx,vy,p}_nodes! (E:1605-1863) for marker m */
static void scatter_marker(const Geo *g, const ErebusMarkersHost *M,
                           int64_t m, ErebusSumsHost *s) {
    int i, j, Ny = g->Ny, Ny1 = g->Ny1;
    double w[4], x = M->xm[m], y = M->ym[m];
    grid_weights(g, GB, x, y, &i, &j, w);
    add_to_grid(s->ETA0SUM, Ny, i, j, w, M->etatotalm[m]);
    add_to_grid(s->ETASUM, Ny, i, j, w, M->etavpm[m]);
    add_to_grid(s->GGGSUM, Ny, i, j, w, M->inv_gggtotalm[m]);
    add_to_grid(s->SXYSUM, Ny, i, j, w, M->sxym[m]);
    add_to_grid(s->COHSUM, Ny, i, j, w, M->cohestotalm[m]);
    add_to_grid(s->TENSUM, Ny, i, j, w, M->tenstotalm[m]);
    add_to_grid(s->FRISUM, Ny, i, j, w, M->fricttotalm[m]);
    add_to_grid(s->WTSUM, Ny, i, j, w, 1.0);
    grid_weights(g, GVX, x, y, &i, &j, w);
    add_to_grid(s->RHOXSUM, Ny1, i, j, w, M->rhototalm[m]);
    add_to_grid(s->RHOFXSUM, Ny1, i, j, w, M->rhofluidcur[m]);
    add_to_grid(s->KXSUM, Ny1, i, j, w, M->ktotalm[m]);
    add_to_grid(s->PHIXSUM, Ny1, i, j, w, M->phim[m]);
    add_to_grid(s->RXSUM, Ny1, i, j, w, M->etafluidcur_inv_kphim[m]);
    add_to_grid(s->WTXSUM, Ny1, i, j, w, 1.0);
    grid_weights(g, GVY, x, y, &i, &j, w);
    add_to_grid(s->RHOYSUM, Ny1, i, j, w, M->rhototalm[m]);
    add_to_grid(s->RHOFYSUM, Ny1, i, j, w, M->rhofluidcur[m]);
    add_to_grid(s->KYSUM, Ny1, i, j, w, M->ktotalm[m]);
    add_to_grid(s->PHIYSUM, Ny1, i, j, w, M->phim[m]);
    add_to_grid(s->RYSUM, Ny1, i, j, w, M->etafluidcur_inv_kphim[m]);
    add_to_grid(s->WTYSUM, Ny1, i, j, w, 1.0);
    grid_weights(g, GP, x, y, &i, &j, w);
    add_to_grid(s->GGGPSUM, Ny1, i, j, w, M->inv_gggtotalm[m]);
    add_to_grid(s->SXXSUM, Ny1, i, j, w, M->sxxm[m]);
    add_to_grid(s->RHOSUM, Ny1, i, j, w, M->rhototalm[m]);
    add_to_grid(s->RHOCPSUM, Ny1, i, j, w, M->rhocptotalm[m]);
    add_to_grid(s->ALPHASUM, Ny1, i, j, w, M->alphasolidcur[m]);
    add_to_grid(s->ALPHAFSUM, Ny1, i, j, w, M->alphafluidcur[m]);
    add_to_grid(s->HRSUM, Ny1, i, j, w, M->hrtotalm[m]);
    add_to_grid(s->PHISUM, Ny1, i, j, w, M->phim[m]);
    add_to_grid(s->TKSUM, Ny1, i, j, w, M->tkm_rhocptotalm[m]);
    add_to_grid(s->WTPSUM, Ny1, i, j, w, 1.0);
}

/* compute_{basic,vx,vy,p}_node_properties! (E:1970-2189) */
static void node_properties(const Geo *g, const ErebusSumsHost *s,
                            ErebusGridHost *G) {
    int Ny = g->Ny, Ny1 = g->Ny1;
    for (int j = 1; j <= g->Nx; j++)
        for (int i = 1; i <= Ny; i++) {
            double wt = AT(s->WTSUM, Ny, i, j);
            if (wt > 0.0) {
                AT(G->ETA0, Ny, i, j) = AT(s->ETA0SUM, Ny, i, j) * (1.0 / wt);
                AT(G->ETA, Ny, i, j) = AT(s->ETASUM, Ny, i, j) * (1.0 / wt);
                if (AT(G->ETA, Ny, i, j) < AT(G->ETA0, Ny, i, j))
                    AT(G->YNY, Ny, i, j) = 1;
                AT(G->GGG, Ny, i, j) = (1.0 / AT(s->GGGSUM, Ny, i, j)) * wt;
                AT(G->SXY0, Ny, i, j) = AT(s->SXYSUM, Ny, i, j) * (1.0 / wt);
                AT(G->COH, Ny, i, j) = AT(s->COHSUM, Ny, i, j) * (1.0 / wt);
                AT(G->TEN, Ny, i, j) = AT(s->TENSUM, Ny, i, j) * (1.0 / wt);
                AT(G->FRI, Ny, i, j) = AT(s->FRISUM, Ny, i, j) * (1.0 / wt);
            }
        }
    for (int j = 1; j <= g->Nx1; j++)
        for (int i = 1; i <= Ny1; i++) {
            double wt = AT(s->WTXSUM, Ny1, i, j);
            if (wt > 0.0) {
                AT(G->RHOX, Ny1, i, j) = AT(s->RHOXSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->RHOFX, Ny1, i, j) = AT(s->RHOFXSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->KX, Ny1, i, j) = AT(s->KXSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->PHIX, Ny1, i, j) = AT(s->PHIXSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->RX, Ny1, i, j) = AT(s->RXSUM, Ny1, i, j) * (1.0 / wt);
            }
        }
    for (int j = 1; j <= g->Nx1; j++)
        for (int i = 1; i <= Ny1; i++) {
            double wt = AT(s->WTYSUM, Ny1, i, j);
            if (wt > 0.0) {
                AT(G->RHOY, Ny1, i, j) = AT(s->RHOYSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->RHOFY, Ny1, i, j) = AT(s->RHOFYSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->KY, Ny1, i, j) = AT(s->KYSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->PHIY, Ny1, i, j) = AT(s->PHIYSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->RY, Ny1, i, j) = AT(s->RYSUM, Ny1, i, j) * (1.0 / wt);
            }
        }
    for (int j = 1; j <= g->Nx1; j++)
        for (int i = 1; i <= Ny1; i++) {
            double wt = AT(s->WTPSUM, Ny1, i, j);
            if (wt > 0.0) {
                AT(G->RHO, Ny1, i, j) = AT(s->RHOSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->RHOCP, Ny1, i, j) = AT(s->RHOCPSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->ALPHA, Ny1, i, j) = AT(s->ALPHASUM, Ny1, i, j) * (1.0 / wt);
                AT(G->ALPHAF, Ny1, i, j) = AT(s->ALPHAFSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->HR, Ny1, i, j) = AT(s->HRSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->GGGP, Ny1, i, j) = (1.0 / AT(s->GGGPSUM, Ny1, i, j)) * wt;
                AT(G->SXX0, Ny1, i, j) = AT(s->SXXSUM, Ny1, i, j) * (1.0 / wt);
                AT(G->tk1, Ny1, i, j) =
                    AT(s->TKSUM, Ny1, i, j) * (1.0 / AT(s->RHOCPSUM, Ny1, i, j));
                AT(G->PHI, Ny1, i, j) = AT(s->PHISUM, Ny1, i, j) * (1.0 / wt);
                AT(G->BETAPHI, Ny1, i, j) =
                    (1.0 / AT(G->GGGP, Ny1, i, j)) * AT(G->PHI, Ny1, i, j);
            }
        }
}

/* apply_insulating_boundary_conditions! (E:2432-2449) on an (Ny1,Nx1) array */
static void insulating_bc(const Geo *g, double *t) {
    int R = g->Ny1, C = g->Nx1;
    if (R > 2 && C > 2) {
        for (int j = 2; j <= C - 1; j++) AT(t, R, 1, j) = AT(t, R, 2, j);
        for (int j = 2; j <= C - 1; j++) AT(t, R, R, j) = AT(t, R, R - 1, j);
        for (int i = 1; i <= R; i++) AT(t, R, i, 1) = AT(t, R, i, 2);
        for (int i = 1; i <= R; i++) AT(t, R, i, C) = AT(t, R, i, C - 1);
    }
}

/* E:6376-6604: one marker->node pass.  Marker loop is serial, as E:6419. */
int oracle_markers_to_nodes(const ErebusParams *p, ErebusMarkersHost *M,
                            int64_t marknum, ErebusGridHost *G,
                            ErebusSumsHost *s, double timesum) {
    Geo g = geo(p);
    double hrs[3], hrf[3];
    reset_sums(&g, s);
    radioactive_heating(p, &g, timesum, hrs, hrf);
    for (int64_t m = 0; m < marknum; m++) {
        marker_properties(p, &g, M, m, hrs, hrf);
        scatter_marker(&g, M, m, s);
    }
    node_properties(&g, s, G);
    insulating_bc(&g, G->tk1);
    return 0;
}

/* compute_relative_enthalpy (E:2502-2504) */
static inline double rel_enthalpy(const ErebusParams *p, double Xs, double XW) {
    return -Xs * XW * p->dHWD / (p->MD + p->MH2O);
}
/* compute_gibbs_free_energy (E:2470-2482) */
static inline double gibbs(const ErebusParams *p, const Geo *g, double T, double pf,
                           double XD, double XW, double dt, double dtr) {
    if (dt < dtr)
        return (p->dHWD - T * p->dSWD + pf * g->dVWD + p->RG * T * log(XD / XW)) *
               (1.0 - dt / dtr);
    return 0.0;
}
/* compute_reaction_constant (E:2521-2524) */
static inline double reaction_constant(const ErebusParams *p, const Geo *g, double T,
                                       double pf, double dG) {
    return exp(-(p->dHWD - T * p->dSWD + g->dVWD * pf - dG) / (p->RG * T));
}

/* ------------------------------------------------------------------------ */
/* thermochemical reaction (E:2558-2694)                                    */
/* ------------------------------------------------------------------------ */
int oracle_thermochemical_reaction(const ErebusParams *p, ErebusMarkersHost *M,
                                   int64_t marknum, ErebusGridHost *G,
                                   ErebusSumsHost *s, double dt, int timestep,
                                   int titer) {
    Geo g = geo(p);
    int Ny1 = g.Ny1;
    size_t np = (size_t)g.Nx1 * g.Ny1;
    memset(s->DMPSUM, 0, np * 8);
    memset(s->DHPSUM, 0, np * 8);
    memset(s->WTPSUM, 0, np * 8);
    for (int64_t m = 0; m < marknum; m++) {
        if (M->tm[m] >= 3) continue;
        int i, j;
        double w[4];
        grid_weights(&g, GP, M->xm[m], M->ym[m], &i, &j, w);
        double tknm = gather4(G->tk2, Ny1, i, j, w);
        double pfnm = jmax(0.0, gather4(G->pf, Ny1, i, j, w));
        if (titer > 2) pfnm = pfnm * (1.0 - p->pfcoeff) + M->pfm0[m] * p->pfcoeff;
        M->pfm0[m] = pfnm;
        double XW0 = M->XWsolidm0[m], phi = M->phim[m];
        double XD0 = 1.0 - XW0;
        double VH2O = tknm > p->tmfluidphase ? g.VH2Of : g.VH2Ofi;
        double Xf0 = phi * (XW0 * g.VWs + XD0 * g.VDs) /
                     ((1.0 - phi) * VH2O + phi * (XW0 * g.VWs + XD0 * g.VDs));
        double Xs0 = 1.0 - Xf0;
        double XH2Ot = (XW0 * Xs0 + Xf0) / (1.0 + XW0 * Xs0);
        double XDt = 1.0 - XH2Ot;
        double rhos0 = (p->MD + p->MH2O * XW0) / (g.VDs * XD0 + g.VWs * XW0);
        double rhof0 = tknm > p->tmfluidphase ? p->rhoH2Of : p->rhoH2Ofi;
        double dtr = dtreaction_of(p, tknm, phi);
        double Ht0 = rel_enthalpy(p, Xs0, XW0);
        double dGWD0 = gibbs(p, &g, tknm, pfnm, XD0, XW0, dt, dtr);
        double KWD = reaction_constant(p, &g, tknm, pfnm, dGWD0);
        double XW1 = 1.0 / (KWD + 1.0);
        double XD1 = 1.0 - XW1;
        double Xs1 = XDt / (1.0 - XDt * XW1);
        double Xf1 = 1.0 - Xs1;
        if (0.0 < Xf1 && Xf1 < 1.0) {
            double phi1 = Xf1 * VH2O / (Xf1 * VH2O + Xs1 * (XW1 * g.VWs + XD1 * g.VDs));
            double rhos1 = (p->MD + p->MH2O * XW1) / (g.VDs * XD1 + g.VWs * XW1);
            double rhof1 = tknm > p->tmfluidphase ? p->rhoH2Of : p->rhoH2Ofi;
            double Ht1 = rel_enthalpy(p, Xs1, XW1);
            double dHt = Ht1 - Ht0;
            double RV = (rhos1 * (1.0 - phi1) + rhof1 * phi1) /
                        (rhos0 * (1.0 - phi) + rhof0 * phi);
            double Gmass = (rhos0 * RV * (1.0 - phi) - rhos1 * (1.0 - phi1)) / dt;
            double dMm = (1.0 - RV) / dt;
            double dHm = Gmass * dHt;
            M->XWsolidm[m] = XW1;
            M->phinewm[m] = phi1;
            if (timestep == 1) {
                M->XWsolidm0[m] = M->XWsolidm[m];
                M->phim[m] = M->phinewm[m];
            }
            add_to_grid(s->DMPSUM, Ny1, i, j, w, dMm);
            add_to_grid(s->DHPSUM, Ny1, i, j, w, dHm);
            add_to_grid(s->WTPSUM, Ny1, i, j, w, 1.0);
        }
    }
    oracle_thermodynamic_xfer(p, s, G);
    return 0;
}

/* compute_thermodynamic_xfer! (E:2208-2222): DMP, DHP at the P nodes from
   the reaction's marker sums, zero where no marker reacted. */
void oracle_thermodynamic_xfer(const ErebusParams *p, const ErebusSumsHost *s,
                               ErebusGridHost *G) {
    Geo g = geo(p);
    size_t np = (size_t)g.Nx1 * g.Ny1;
    for (size_t k = 0; k < np; k++) {
        double wt = s->WTPSUM[k];
        if (wt > 0.0) {
            G->DMP[k] = s->DMPSUM[k] * (1.0 / wt);
            G->DHP[k] = s->DHPSUM[k] * (1.0 / wt);
        } else {
            G->DMP[k] = G->DHP[k] = 0.0;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* gravity (E:2798-2878)                                                    */
/* ------------------------------------------------------------------------ */
/* Emits the COO triplets of LP (0-based) and RP; returns the entry count. */
int64_t oracle_assemble_gravity(const ErebusParams *p, const ErebusGridHost *G,
                                int64_t *rows, int64_t *cols, double *vals,
                                double *RP) {
    Geo g = geo(p);
    int Ny1 = g.Ny1, Nx1 = g.Nx1;
    int64_t n = 0;
#define PUT(r, c, v) do { rows[n] = (r); cols[n] = (c); vals[n] = (v); n++; } while (0)
    memset(RP, 0, sizeof(double) * (size_t)Nx1 * Ny1);
    double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
    for (int j = 1; j <= Nx1; j++)
        for (int i = 1; i <= Ny1; i++) {
            int64_t gk = (int64_t)(j - 1) * Ny1 + i - 1;
            double xpj = ax(-g.dx / 2, g.dx, j), ypi = ax(-g.dy / 2, g.dy, i);
            double dxc = xpj - g.xcenter, dyc = ypi - g.ycenter;
            double dist = sqrt(dxc * dxc + dyc * dyc);
            if (i == 1 || i == Ny1 || j == 1 || j == Nx1 || dist > g.xcenter) {
                PUT(gk, gk, 1.0);
            } else {
                PUT(gk, gk - Ny1, idx2);
                PUT(gk, gk - 1, idy2);
                PUT(gk, gk, -2.0 * (idx2 + idy2));
                PUT(gk, gk + 1, idy2);
                PUT(gk, gk + Ny1, idx2);
                RP[gk] = 4.0 * 2.0 * (1.0 / 3.0) * M_PI * p->G *
                         AT(G->RHO, Ny1, i, j);
            }
        }
#undef PUT
    return n;
}

/* process_gravitational_solution! (E:2865-2878) */
int oracle_process_gravity(const ErebusParams *p, const double *SP,
                           ErebusGridHost *G) {
    Geo g = geo(p);
    int Ny1 = g.Ny1, Nx1 = g.Nx1;
    memcpy(G->FI, SP, sizeof(double) * (size_t)Nx1 * Ny1);
    for (int j = 1; j <= g.Nx; j++)
        for (int i = 1; i <= Ny1; i++)
            AT(G->gx, Ny1, i, j) =
                -(AT(G->FI, Ny1, i, j + 1) - AT(G->FI, Ny1, i, j)) / g.dx;
    for (int j = 1; j <= Nx1; j++)
        for (int i = 1; i <= g.Ny; i++)
            AT(G->gy, Ny1, i, j) =
                -(AT(G->FI, Ny1, i + 1, j) - AT(G->FI, Ny1, i, j)) / g.dy;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Stokes-Darcy (E:3089-3647)                                               */
/* ------------------------------------------------------------------------ */
/* recompute_bulk_viscosity! (E:3634-3647) */
int oracle_bulk_viscosity(const ErebusParams *p, ErebusGridHost *G) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1;
    for (int j = 2; j <= g.Nx; j++)
        for (int i = 2; i <= Ny; i++)
            AT(G->ETAP, Ny1, i, j) =
                4.0 / (1.0 / AT(G->ETA, Ny, i - 1, j - 1) +
                       1.0 / AT(G->ETA, Ny, i, j - 1) +
                       1.0 / AT(G->ETA, Ny, i - 1, j) + 1.0 / AT(G->ETA, Ny, i, j));
    size_t np = (size_t)g.Nx1 * Ny1;
    for (size_t k = 0; k < np; k++)
        G->ETAPHI[k] = p->etaphikoef * G->ETAP[k] * (1.0 / G->PHI[k]);
    return 0;
}

/* assemble_hydromechanical_lse! (E:3089-3572).  COO triplets, 0-based rows
   in the reference's interleaved order k = ((j-1)*Ny1+i-1)*6 + {0..5}. */
int64_t oracle_assemble_hydromech(const ErebusParams *p,
                                  const ErebusGridHost *G, double dt,
                                  int64_t *rows, int64_t *cols, double *vals,
                                  double *R) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1, Nx = g.Nx, Nx1 = g.Nx1;
    double dx = g.dx, dy = g.dy, Kc = p->Kcont;
    int64_t n = 0;
    int64_t S6 = 6 * (int64_t)Ny1;
#define PUT(r, c, v) do { rows[n] = (r); cols[n] = (c); vals[n] = (v); n++; } while (0)
    memset(R, 0, sizeof(double) * (size_t)Nx1 * Ny1 * 6);
    const double *ETA = G->ETA, *GGG = G->GGG, *SXY0 = G->SXY0;
    const double *ETAP = G->ETAP, *GGGP = G->GGGP, *SXX0 = G->SXX0;
    for (int j = 1; j <= Nx1; j++)
        for (int i = 1; i <= Ny1; i++) {
            int64_t kvx = ((int64_t)(j - 1) * Ny1 + i - 1) * 6;
            int64_t kvy = kvx + 1, kpm = kvx + 2, kqx = kvx + 3, kqy = kvx + 4,
                    kpf = kvx + 5;
            /* x-Stokes (E:3128-3262) */
            if (i == 1 || i == Ny1 || j == 1 || j == Nx || j == Nx1) {
                PUT(kvx, kvx, 1.0);
                if (j == 1) R[kvx] = g.vxleft;
                if (j == Nx) R[kvx] = g.vxright;
                if (i == 1 && 1 < j && j < Nx) PUT(kvx, kvx + 6, p->bctop);
                if (i == Ny1 && 1 < j && j < Nx) PUT(kvx, kvx - 6, p->bcbottom);
            } else {
                double e1 = AT(ETA, Ny, i - 1, j), g1 = AT(GGG, Ny, i - 1, j);
                double e2 = AT(ETA, Ny, i, j), g2 = AT(GGG, Ny, i, j);
                double ep1 = AT(ETAP, Ny1, i, j), gp1 = AT(GGGP, Ny1, i, j);
                double ep2 = AT(ETAP, Ny1, i, j + 1), gp2 = AT(GGGP, Ny1, i, j + 1);
                double ETA1 = e1 * g1 * dt / (g1 * dt + e1);
                double ETA2 = e2 * g2 * dt / (g2 * dt + e2);
                double ETAP1 = ep1 * gp1 * dt / (gp1 * dt + ep1);
                double ETAP2 = ep2 * gp2 * dt / (gp2 * dt + ep2);
                double SXY1 = AT(SXY0, Ny, i - 1, j) * e1 / (g1 * dt + e1);
                double SXY2 = AT(SXY0, Ny, i, j) * e2 / (g2 * dt + e2);
                double SXX1 = AT(SXX0, Ny1, i, j) * ep1 / (gp1 * dt + ep1);
                double SXX2 = AT(SXX0, Ny1, i, j + 1) * ep2 / (gp2 * dt + ep2);
                double dRdx = 0.5 * (AT(G->RHOX, Ny1, i, j + 1) - AT(G->RHOX, Ny1, i, j - 1)) * (1.0 / dx);
                double dRdy = 0.5 * (AT(G->RHOX, Ny1, i + 1, j) - AT(G->RHOX, Ny1, i - 1, j)) * (1.0 / dy);
                double gxij = AT(G->gx, Ny1, i, j);
                double idx = 1.0 / dx, idy = 1.0 / dy;
                PUT(kvx, kvx - S6, ETAP1 / (dx * dx));
                PUT(kvx, kvx - 6, ETA1 / (dy * dy));
                PUT(kvx, kvx, -(ETAP1 + ETAP2) * (1.0 / (dx * dx)) -
                                  (ETA1 + ETA2) * (1.0 / (dy * dy)) -
                                  dRdx * gxij * dt);
                PUT(kvx, kvx + 6, ETA2 / (dy * dy));
                PUT(kvx, kvx + S6, ETAP2 / (dx * dx));
                PUT(kvx, kvy, ETAP1 * idx * idy - ETA2 * idx * idy - dRdy * gxij * dt * 0.25);
                PUT(kvx, kvy + S6, -ETAP2 * idx * idy + ETA2 * idx * idy - dRdy * gxij * dt * 0.25);
                PUT(kvx, kvy - 6, -ETAP1 * idx * idy + ETA1 * idx * idy - dRdy * gxij * dt * 0.25);
                PUT(kvx, kvy + S6 - 6, ETAP2 * idx * idy - ETA1 * idx * idy - dRdy * gxij * dt * 0.25);
                PUT(kvx, kpm, Kc * idx);
                PUT(kvx, kpm + S6, -Kc * idx);
                R[kvx] = -AT(G->RHOX, Ny1, i, j) * gxij - (SXY2 - SXY1) * idy -
                         (SXX2 - SXX1) * idx;
            }
            /* y-Stokes (E:3264-3396) */
            if (i == 1 || i == Ny || i == Ny1 || j == 1 || j == Nx1) {
                PUT(kvy, kvy, 1.0);
                if (i == 1) R[kvy] = g.vytop;
                if (i == Ny) R[kvy] = g.vybottom;
                if (j == 1 && 1 < i && i < Ny) PUT(kvy, kvy + S6, p->bcleft);
                if (j == Nx1 && 1 < i && i < Ny) PUT(kvy, kvy - S6, p->bcright);
            } else {
                double e1 = AT(ETA, Ny, i, j - 1), g1 = AT(GGG, Ny, i, j - 1);
                double e2 = AT(ETA, Ny, i, j), g2 = AT(GGG, Ny, i, j);
                double ep1 = AT(ETAP, Ny1, i, j), gp1 = AT(GGGP, Ny1, i, j);
                double ep2 = AT(ETAP, Ny1, i + 1, j), gp2 = AT(GGGP, Ny1, i + 1, j);
                double ETA1 = e1 * g1 * dt / (g1 * dt + e1);
                double ETA2 = e2 * g2 * dt / (g2 * dt + e2);
                double ETAP1 = ep1 * gp1 * dt / (gp1 * dt + ep1);
                double ETAP2 = ep2 * gp2 * dt / (gp2 * dt + ep2);
                double SXY1 = AT(SXY0, Ny, i, j - 1) * e1 / (g1 * dt + e1);
                double SXY2 = AT(SXY0, Ny, i, j) * e2 / (g2 * dt + e2);
                double SYY1 = -AT(SXX0, Ny1, i, j) * ep1 / (gp1 * dt + ep1);
                double SYY2 = -AT(SXX0, Ny1, i + 1, j) * ep2 / (gp2 * dt + ep2);
                double dRdx = 0.5 * (AT(G->RHOY, Ny1, i, j + 1) - AT(G->RHOY, Ny1, i, j - 1)) / dx;
                double dRdy = 0.5 * (AT(G->RHOY, Ny1, i + 1, j) - AT(G->RHOY, Ny1, i - 1, j)) / dy;
                double gyij = AT(G->gy, Ny1, i, j);
                double idx = 1.0 / dx, idy = 1.0 / dy;
                PUT(kvy, kvy - S6, ETA1 / (dx * dx));
                PUT(kvy, kvy - 6, ETAP1 / (dy * dy));
                PUT(kvy, kvy, -(ETAP1 + ETAP2) * (1.0 / (dy * dy)) -
                                  (ETA1 + ETA2) * (1.0 / (dx * dx)) -
                                  dRdy * gyij * dt);
                PUT(kvy, kvy + 6, ETAP2 * (1.0 / (dy * dy)));
                PUT(kvy, kvy + S6, ETA2 * (1.0 / (dx * dx)));
                PUT(kvy, kvx, ETAP1 * idx * idy - ETA2 * idx * idy - dRdx * gyij * dt * 0.25);
                PUT(kvy, kvx + 6, -ETAP2 * idx * idy + ETA2 * idx * idy - dRdx * gyij * dt * 0.25);
                PUT(kvy, kvx - S6, -ETAP1 * idx * idy + ETA1 * idx * idy - dRdx * gyij * dt * 0.25);
                PUT(kvy, kvx + 6 - S6, ETAP2 * idx * idy - ETA1 * idx * idy - dRdx * gyij * dt * 0.25);
                PUT(kvy, kpm, Kc * idy);
                PUT(kvy, kpm + 6, -Kc * idy);
                R[kvy] = -AT(G->RHOY, Ny1, i, j) * gyij - (SXY2 - SXY1) * idx -
                         (SYY2 - SYY1) * idy;
            }
            int ring = (i == 2 && 2 <= j && j <= Nx) || (j == 2 && 2 < i && i < Ny) ||
                       (i == Ny && 2 <= j && j <= Nx) || (j == Nx && 2 < i && i < Ny);
            /* P total continuity (E:3398-3452) */
            if (i == 1 || i == Ny1 || j == 1 || j == Nx1) {
                PUT(kpm, kpm, 1.0);
            } else if (ring) {
                PUT(kpm, kpm, Kc);
                R[kpm] = p->psurface;
            } else {
                double ph = AT(G->PHI, Ny1, i, j), etph = AT(G->ETAPHI, Ny1, i, j);
                double bph = AT(G->BETAPHI, Ny1, i, j);
                PUT(kpm, kvx - S6, -1.0 / dx);
                PUT(kpm, kvx, 1.0 / dx);
                PUT(kpm, kvy - 6, -1.0 / dy);
                PUT(kpm, kvy, 1.0 / dy);
                PUT(kpm, kpm, Kc / (1 - ph) * (1.0 / etph + bph / dt));
                PUT(kpm, kpf, -Kc / (1 - ph) * (1.0 / etph + bph / dt));
                R[kpm] = (AT(G->pr0, Ny1, i, j) - AT(G->pf0, Ny1, i, j)) / (1 - ph) *
                             bph / dt + AT(G->DMP, Ny1, i, j);
            }
            /* qx Darcy (E:3454-3480) */
            if (i == 1 || i == Ny1 || j == 1 || j == Nx || j == Nx1) {
                PUT(kqx, kqx, 1.0);
                if (i == 1 && 1 < j && j < Nx) PUT(kqx, kqx + 6, p->bcftop);
                if (i == Ny1 && 1 < j && j < Nx) PUT(kqx, kqx - 6, p->bcfbottom);
            } else {
                PUT(kqx, kqx, AT(G->RX, Ny1, i, j));
                PUT(kqx, kpf, -Kc * (1.0 / dx));
                PUT(kqx, kpf + S6, Kc * (1.0 / dx));
                R[kqx] = AT(G->RHOFX, Ny1, i, j) * AT(G->gx, Ny1, i, j);
            }
            /* qy Darcy (E:3482-3514) */
            if (i == 1 || i == Ny || i == Ny1 || j == 1 || j == Nx1) {
                PUT(kqy, kqy, 1.0);
                if (j == 1 && 1 < i && i < Ny) PUT(kqy, kqy + S6, p->bcfleft);
                if (j == Nx1 && 1 < i && i < Ny) PUT(kqy, kqy - S6, p->bcfright);
            } else {
                PUT(kqy, kqy, AT(G->RY, Ny1, i, j));
                PUT(kqy, kpf, -Kc * (1.0 / dy));
                PUT(kqy, kpf + 6, Kc * (1.0 / dy));
                R[kqy] = AT(G->RHOFY, Ny1, i, j) * AT(G->gy, Ny1, i, j);
            }
            /* P fluid continuity (E:3516-3565) */
            if (i == 1 || i == Ny1 || j == 1 || j == Nx1) {
                PUT(kpf, kpf, 1.0);
            } else if (ring) {
                PUT(kpf, kpf, Kc);
                R[kpf] = p->psurface;
            } else {
                double ph = AT(G->PHI, Ny1, i, j), etph = AT(G->ETAPHI, Ny1, i, j);
                double bph = AT(G->BETAPHI, Ny1, i, j);
                PUT(kpf, kqx - S6, -(1.0 / dx));
                PUT(kpf, kqx, 1.0 / dx);
                PUT(kpf, kqy - 6, -(1.0 / dy));
                PUT(kpf, kqy, 1.0 / dy);
                PUT(kpf, kpm, -Kc / (1.0 - ph) * (1.0 / etph + bph / dt));
                PUT(kpf, kpf, Kc / (1.0 - ph) * (1.0 / etph + bph / dt));
                R[kpf] = -(AT(G->pr0, Ny1, i, j) - AT(G->pf0, Ny1, i, j)) / (1 - ph) *
                         bph / dt;
            }
        }
#undef PUT
    return n;
}

/* process_hydromechanical_solution! (E:3593-3617) */
int oracle_process_hydromech(const ErebusParams *p, const double *S,
                             ErebusGridHost *G) {
    Geo g = geo(p);
    size_t np = (size_t)g.Nx1 * g.Ny1;
    for (size_t k = 0; k < np; k++) {
        G->vx[k] = S[6 * k + 0];
        G->vy[k] = S[6 * k + 1];
        G->pr[k] = S[6 * k + 2] * p->Kcont;
        G->qxD[k] = S[6 * k + 3];
        G->qyD[k] = S[6 * k + 4];
        G->pf[k] = S[6 * k + 5] * p->Kcont;
    }
    return 0;
}

/* compute_Aphi! (E:3675-3689); returns max|APHI[2:Ny,2:Nx]| */
double oracle_compute_aphi(const ErebusParams *p, ErebusGridHost *G, double dt) {
    Geo g = geo(p);
    int Ny1 = g.Ny1;
    double mx = -INFINITY;
    for (int j = 2; j <= g.Nx; j++)
        for (int i = 2; i <= g.Ny; i++) {
            double pr = AT(G->pr, Ny1, i, j), pf = AT(G->pf, Ny1, i, j);
            double ph = AT(G->PHI, Ny1, i, j);
            double v = ((pr - pf) / AT(G->ETAPHI, Ny1, i, j) +
                        ((pr - AT(G->pr0, Ny1, i, j)) - (pf - AT(G->pf0, Ny1, i, j))) /
                            dt * AT(G->BETAPHI, Ny1, i, j)) /
                       (1 - ph) / ph;
            AT(G->APHI, Ny1, i, j) = v;
            mx = jmax(mx, fabs(v));
        }
    return mx;
}

/* compute_fluid_velocities! (E:3716-3757) */
int oracle_fluid_velocities(const ErebusParams *p, ErebusGridHost *G) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1, Nx = g.Nx, Nx1 = g.Nx1;
    for (int j = 1; j <= Nx; j++)
        for (int i = 2; i <= Ny; i++)
            AT(G->vxf, Ny1, i, j) = AT(G->qxD, Ny1, i, j) / AT(G->PHIX, Ny1, i, j);
    for (int j = 1; j <= Nx1; j++) {
        AT(G->vxf, Ny1, 1, j) = -p->bcftop * AT(G->vxf, Ny1, 2, j);
        AT(G->vxf, Ny1, Ny1, j) = -p->bcfbottom * AT(G->vxf, Ny1, Ny, j);
    }
    for (int j = 2; j <= Nx; j++)
        for (int i = 1; i <= Ny; i++)
            AT(G->vyf, Ny1, i, j) = AT(G->qyD, Ny1, i, j) / AT(G->PHIY, Ny1, i, j);
    for (int i = 1; i <= Ny1; i++) {
        AT(G->vyf, Ny1, i, 1) = -p->bcfleft * AT(G->vyf, Ny1, i, 2);
        AT(G->vyf, Ny1, i, Nx1) = -p->bcfright * AT(G->vyf, Ny1, i, Nx);
    }
    size_t np = (size_t)Nx1 * Ny1;
    for (size_t k = 0; k < np; k++) {
        G->vxf[k] += G->vx[k];
        G->vyf[k] += G->vy[k];
    }
    return 0;
}

static double maxabs(const double *a, size_t n) {
    double m = -INFINITY;
    for (size_t k = 0; k < n; k++) m = jmax(m, fabs(a[k]));
    return m;
}

/* compute_displacement_timestep (E:3777-3803) */
double oracle_displacement_timestep(const ErebusParams *p,
                                    const ErebusGridHost *G, double dt,
                                    double aphimax) {
    Geo g = geo(p);
    size_t np = (size_t)g.Nx1 * g.Ny1;
    double maxvx = maxabs(G->vx, np), maxvy = maxabs(G->vy, np);
    double maxvxf = maxabs(G->vxf, np), maxvyf = maxabs(G->vyf, np);
    double lx = p->dxymax * g.dx, ly = p->dxymax * g.dy;
    dt = (dt * maxvx > lx) ? lx * (1.0 / maxvx) : dt;
    dt = (dt * maxvy > ly) ? ly * (1.0 / maxvy) : dt;
    dt = (dt * maxvxf > lx) ? lx * (1.0 / maxvxf) : dt;
    dt = (dt * maxvyf > ly) ? ly * (1.0 / maxvyf) : dt;
    dt = (dt * aphimax > p->dphimax) ? p->dphimax * (1.0 / aphimax) : dt;
    return dt;
}

/* compute_stress_strainrate! (E:3839-3925) */
int oracle_stress_strainrate(const ErebusParams *p, ErebusGridHost *G,
                             double dt) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1;
    for (int j = 1; j <= g.Nx; j++)
        for (int i = 1; i <= Ny; i++) {
            double exy = 0.5 * ((AT(G->vx, Ny1, i + 1, j) - AT(G->vx, Ny1, i, j)) / g.dy +
                                (AT(G->vy, Ny1, i, j + 1) - AT(G->vy, Ny1, i, j)) / g.dx);
            AT(G->EXY, Ny, i, j) = exy;
            double e = AT(G->ETA, Ny, i, j), gg = AT(G->GGG, Ny, i, j);
            double sxy = 2 * e * exy * gg * dt / (gg * dt + e) +
                         AT(G->SXY0, Ny, i, j) * e / (gg * dt + e);
            AT(G->SXY, Ny, i, j) = sxy;
            AT(G->DSXY, Ny, i, j) = sxy - AT(G->SXY0, Ny, i, j);
        }
    for (int j = 2; j <= g.Nx; j++)
        for (int i = 2; i <= Ny; i++) {
            double exx = 0.5 * ((AT(G->vx, Ny1, i, j) - AT(G->vx, Ny1, i, j - 1)) / g.dx -
                                (AT(G->vy, Ny1, i, j) - AT(G->vy, Ny1, i - 1, j)) / g.dy);
            AT(G->EXX, Ny1, i, j) = exx;
            double e = AT(G->ETAP, Ny1, i, j), gg = AT(G->GGGP, Ny1, i, j);
            double sxx = 2 * e * exx * gg * dt / (gg * dt + e) +
                         AT(G->SXX0, Ny1, i, j) * e / (gg * dt + e);
            AT(G->SXX, Ny1, i, j) = sxx;
            AT(G->DSXX, Ny1, i, j) = sxx - AT(G->SXX0, Ny1, i, j);
            double ae = grid_average(G->EXY, Ny, i - 1, j - 1);
            double as = grid_average(G->SXY, Ny, i - 1, j - 1);
            AT(G->EII, Ny1, i, j) = sqrt(exx * exx + ae * ae);
            AT(G->SII, Ny1, i, j) = sqrt(sxx * sxx + as * as);
        }
    return 0;
}

/* symmetrize_p_node_observables! (E:3945-3984) */
int oracle_symmetrize(const ErebusParams *p, ErebusGridHost *G) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1, Nx = g.Nx, Nx1 = g.Nx1;
    double *F[5] = {G->SXX, G->APHI, G->PHI, G->pr, G->pf};
    for (int f = 0; f < 5; f++)
        for (int j = 2; j <= Nx; j++) AT(F[f], Ny1, 1, j) = AT(F[f], Ny1, 2, j);
    for (int f = 0; f < 5; f++)
        for (int j = 2; j <= Nx; j++) AT(F[f], Ny1, Ny1, j) = AT(F[f], Ny1, Ny, j);
    for (int f = 0; f < 5; f++)
        for (int i = 1; i <= Ny1; i++) AT(F[f], Ny1, i, 1) = AT(F[f], Ny1, i, 2);
    for (int f = 0; f < 5; f++)
        for (int i = 1; i <= Ny1; i++) AT(F[f], Ny1, i, Nx1) = AT(F[f], Ny1, i, Nx);
    size_t np = (size_t)Nx1 * Ny1;
    for (size_t k = 0; k < np; k++)
        G->ps[k] = (G->pr[k] - G->pf[k] * G->PHI[k]) * (1.0 / (1 - G->PHI[k]));
    return 0;
}

/* compute_nodal_adjustment! (E:4015-4094).  *yerr receives YERRNOD[iplast]
   when ynpl > 0 (unchanged otherwise); returns the convergence flag. */
int oracle_nodal_adjustment(const ErebusParams *p, ErebusGridHost *G,
                            double dt, int iplast, double *yerr, int *ynpl_out) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1;
    size_t nb = (size_t)g.Nx * Ny;
    memcpy(G->ETA5, G->ETA0, nb * 8);
    memset(G->YNY5, 0, nb);
    memset(G->DSY, 0, nb * 8);
    int64_t ynpl = 0;
    double ddd = 0.0;
    for (int j = 1; j <= g.Nx; j++)
        for (int i = 1; i <= Ny; i++) {
            double sxy = AT(G->SXY, Ny, i, j), asxx = grid_average(G->SXX, Ny1, i, j);
            double SIIB = sqrt(sxy * sxy + asxx * asxx);
            double e = AT(G->ETA, Ny, i, j), gg = AT(G->GGG, Ny, i, j);
            double siiel = SIIB * (gg * dt + e) / e;
            double prB = grid_average(G->pr, Ny1, i, j);
            double pfB = grid_average(G->pf, Ny1, i, j);
            double syc = AT(G->COH, Ny, i, j) + AT(G->FRI, Ny, i, j) * (prB - pfB);
            double syt = AT(G->TEN, Ny, i, j) + (prB - pfB);
            double sy = jmax(jmin(syc, syt), 0.0);
            if (AT(G->YNY, Ny, i, j) > 0) {
                double d = SIIB - sy;
                AT(G->DSY, Ny, i, j) = d;
                ddd += d * d;
                ynpl += 1;
            }
            if (sy < siiel) {
                double etapl = dt * gg * sy / (siiel - sy);
                if (etapl < AT(G->ETA0, Ny, i, j)) {
                    double e5 = pow(etapl, 1.0 - p->etawt) * pow(e, p->etawt);
                    if (e5 > p->etamax) e5 = p->etamax;
                    else if (e5 < p->etamin) e5 = p->etamin;
                    AT(G->ETA5, Ny, i, j) = e5;
                    AT(G->YNY5, Ny, i, j) = 1;
                    double d = SIIB - sy;   /* `ynn == false` always holds */
                    AT(G->DSY, Ny, i, j) = d;
                    ddd += d * d;
                    ynpl += 1;
                }
            }
        }
    if (ynpl > 0) *yerr = sqrt(ddd / (double)ynpl);
    if (ynpl_out) *ynpl_out = (int)ynpl;
    return ynpl == 0 || *yerr < p->yerrmax || iplast == p->nplast;
}

/* finalize_plastic_iteration_pass! (E:4142-4169); returns dt */
double oracle_finalize_plastic(const ErebusParams *p, ErebusGridHost *G,
                               double dt, int iplast) {
    Geo g = geo(p);
    size_t nb = (size_t)g.Nx * g.Ny;
    if (iplast % p->dtstep == 0) {
        dt *= p->dtcoefdn;
        memcpy(G->ETA, G->ETA00, nb * 8);
        memcpy(G->YNY, G->YNY00, nb);
    } else {
        memcpy(G->ETA, G->ETA5, nb * 8);
        memcpy(G->YNY, G->YNY5, nb);
    }
    for (size_t k = 0; k < nb; k++) G->YNY_inv_ETA[k] = (double)G->YNY[k] / G->ETA[k];
    return dt;
}

/* ------------------------------------------------------------------------ */
/* heat equation (E:4415-4611)                                              */
/* ------------------------------------------------------------------------ */
/* compute_shear_heating! (E:4415-4433) */
int oracle_shear_heating(const ErebusParams *p, ErebusGridHost *G) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1;
    for (int j = 2; j <= g.Nx; j++)
        for (int i = 2; i <= Ny; i++) {
            double s1 = AT(G->SXY, Ny, i - 1, j - 1), s2 = AT(G->SXY, Ny, i, j - 1);
            double s3 = AT(G->SXY, Ny, i - 1, j), s4 = AT(G->SXY, Ny, i, j);
            double SXYEXY = 0.25 * (s1 * s1 / AT(G->ETA, Ny, i - 1, j - 1) +
                                    s2 * s2 / AT(G->ETA, Ny, i, j - 1) +
                                    s3 * s3 / AT(G->ETA, Ny, i - 1, j) +
                                    s4 * s4 / AT(G->ETA, Ny, i, j));
            double sxx = AT(G->SXX, Ny1, i, j), dp = AT(G->pr, Ny1, i, j) - AT(G->pf, Ny1, i, j);
            double q1 = AT(G->qxD, Ny1, i, j - 1), q2 = AT(G->qxD, Ny1, i, j);
            double q3 = AT(G->qyD, Ny1, i - 1, j), q4 = AT(G->qyD, Ny1, i, j);
            AT(G->HS, Ny1, i, j) =
                sxx * sxx / AT(G->ETAP, Ny1, i, j) + SXYEXY +
                dp * dp / (1 - AT(G->PHI, Ny1, i, j)) / AT(G->ETAPHI, Ny1, i, j) +
                0.5 * (AT(G->RX, Ny1, i, j - 1) * (q1 * q1) + AT(G->RX, Ny1, i, j) * (q2 * q2)) +
                0.5 * (AT(G->RY, Ny1, i - 1, j) * (q3 * q3) + AT(G->RY, Ny1, i, j) * (q4 * q4));
        }
    return 0;
}

/* compute_adiabatic_heating! (E:4458-4501); keeps the reference's use of the
   solid-pressure gradients in the fluid term (E:4492). */
int oracle_adiabatic_heating(const ErebusParams *p, ErebusGridHost *G) {
    Geo g = geo(p);
    int Ny1 = g.Ny1;
    double idx = 1.0 / g.dx, idy = 1.0 / g.dy;
    for (int j = 2; j <= g.Nx; j++)
        for (int i = 2; i <= g.Ny; i++) {
            double VXP = 0.5 * (AT(G->vx, Ny1, i, j) + AT(G->vx, Ny1, i, j - 1));
            double VYP = 0.5 * (AT(G->vy, Ny1, i, j) + AT(G->vy, Ny1, i - 1, j));
            double VXFP = 0.5 * (AT(G->vxf, Ny1, i, j) + AT(G->vxf, Ny1, i, j - 1));
            double VYFP = 0.5 * (AT(G->vyf, Ny1, i, j) + AT(G->vyf, Ny1, i - 1, j));
            double dpsdx = VXP < 0.0 ? (AT(G->ps, Ny1, i, j) - AT(G->ps, Ny1, i, j - 1)) * idx
                                     : (AT(G->ps, Ny1, i, j + 1) - AT(G->ps, Ny1, i, j)) * idx;
            double dpsdy = VYP < 0.0 ? (AT(G->ps, Ny1, i, j) - AT(G->ps, Ny1, i - 1, j)) * idy
                                     : (AT(G->ps, Ny1, i + 1, j) - AT(G->ps, Ny1, i, j)) * idy;
            double dpsdt = VXP * dpsdx + VYP * dpsdy;
            double dpfdt = VXFP * dpsdx + VYFP * dpsdy;
            double ph = AT(G->PHI, Ny1, i, j), tk = AT(G->tk1, Ny1, i, j);
            AT(G->HA, Ny1, i, j) = (1 - ph) * tk * AT(G->ALPHA, Ny1, i, j) * dpsdt +
                                   ph * tk * AT(G->ALPHAF, Ny1, i, j) * dpfdt;
        }
    return 0;
}

/* assemble_thermal_lse! (E:4526-4611).  COO triplets (0-based) and RT. */
int64_t oracle_assemble_thermal(const ErebusParams *p, const ErebusGridHost *G,
                                double dt, int64_t *rows, int64_t *cols,
                                double *vals, double *RT) {
    Geo g = geo(p);
    int Ny1 = g.Ny1, Nx1 = g.Nx1;
    int64_t n = 0;
#define PUT(r, c, v) do { rows[n] = (r); cols[n] = (c); vals[n] = (v); n++; } while (0)
    memset(RT, 0, sizeof(double) * (size_t)Nx1 * Ny1);
    double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
    for (int j = 1; j <= Nx1; j++)
        for (int i = 1; i <= Ny1; i++) {
            int64_t gk = (int64_t)(j - 1) * Ny1 + i - 1;
            if (i == 1 || i == Ny1 || j == 1 || j == Nx1) {
                PUT(gk, gk, 1.0);
                if (j == 1) PUT(gk, gk + Ny1, -1.0);
                if (j == Nx1) PUT(gk, gk - Ny1, -1.0);
                if (i == 1 && 1 < j && j < Nx1) PUT(gk, gk + 1, -1.0);
                if (i == Ny1 && 1 < j && j < Nx1) PUT(gk, gk - 1, -1.0);
            } else {
                double Kx1 = AT(G->KX, Ny1, i, j - 1), Kx2 = AT(G->KX, Ny1, i, j);
                double Ky1 = AT(G->KY, Ny1, i - 1, j), Ky2 = AT(G->KY, Ny1, i, j);
                double rc = AT(G->RHOCP, Ny1, i, j);
                PUT(gk, gk - Ny1, -Kx1 * idx2);
                PUT(gk, gk - 1, -Ky1 * idy2);
                PUT(gk, gk, rc / dt + (Kx1 + Kx2) * idx2 + (Ky1 + Ky2) * idy2);
                PUT(gk, gk + 1, -Ky2 * idy2);
                PUT(gk, gk + Ny1, -Kx2 * idx2);
                RT[gk] = rc / dt * AT(G->tk1, Ny1, i, j) + AT(G->HR, Ny1, i, j) +
                         AT(G->HA, Ny1, i, j) + AT(G->HS, Ny1, i, j) +
                         AT(G->DHP, Ny1, i, j);
            }
        }
#undef PUT
    return n;
}

/* ------------------------------------------------------------------------ */
/* node -> marker (E:6945-7019)                                             */
/* ------------------------------------------------------------------------ */
/* update_marker_viscosity! (E:774-804), update_marker_stress! (E:4354-4388),
   update_marker_temperature! (E:4782-4801), copies E:7011-7012,
   update_marker_porosity! (E:4822-4856), copy E:7014,
   update_p_nodes_melt_composition! (E:1929-1939).  The marker loops the
   reference runs with @threads run with OpenMP here. */
/* apply_subgrid_stress_diffusion! (E:4253-4333): marker-node stress
   differences relaxed over dt (the reference fixes the viscosity factor to
   1, E:4276), markers corrected, the corrections scattered in marker order
   and subtracted from DSXX at inner P nodes and from DSXY at all basic
   nodes.  A no-op when dsubgrids == 0. */
int oracle_subgrid_stress(const ErebusParams *p, ErebusMarkersHost *M, int64_t marknum,
                          ErebusGridHost *G, ErebusSumsHost *s, double dt) {
    if (p->dsubgrids == 0.0) return 0;
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1;
    size_t np = (size_t)g.Nx1 * Ny1, nb = (size_t)g.Nx * Ny;
    memset(s->SXXSUM, 0, np * 8);
    memset(s->WTPSUM, 0, np * 8);
    memset(s->SXYSUM, 0, nb * 8);
    memset(s->WTSUM, 0, nb * 8);
    const double etam = 1.0;
    for (int64_t m = 0; m < marknum; m++) {
        int ip, jp, ib, jb;
        double wp[4], wb[4];
        grid_weights(&g, GP, M->xm[m], M->ym[m], &ip, &jp, wp);
        grid_weights(&g, GB, M->xm[m], M->ym[m], &ib, &jb, wb);
        double dxx = M->sxxm[m] - gather4(G->SXX0, Ny1, ip, jp, wp);
        dxx *= exp(-p->dsubgrids * dt / (etam * M->inv_gggtotalm[m])) - 1.0;
        M->sxxm[m] += dxx;
        add_to_grid(s->SXXSUM, Ny1, ip, jp, wp, dxx);
        add_to_grid(s->WTPSUM, Ny1, ip, jp, wp, 1.0);
        double dxy = M->sxym[m] - gather4(G->SXY0, Ny, ib, jb, wb);
        dxy *= exp(-p->dsubgrids * dt / (etam * M->inv_gggtotalm[m])) - 1.0;
        M->sxym[m] += dxy;
        add_to_grid(s->SXYSUM, Ny, ib, jb, wb, dxy);
        add_to_grid(s->WTSUM, Ny, ib, jb, wb, 1.0);
    }
    for (int j = 2; j <= g.Nx; j++)
        for (int i = 2; i <= Ny; i++)
            if (AT(s->WTPSUM, Ny1, i, j) > 0.0)
                AT(G->DSXX, Ny1, i, j) -= AT(s->SXXSUM, Ny1, i, j) / AT(s->WTPSUM, Ny1, i, j);
    for (size_t k = 0; k < nb; k++)
        if (s->WTSUM[k] > 0.0) G->DSXY[k] -= s->SXYSUM[k] / s->WTSUM[k];
    return 0;
}

/* apply_subgrid_temperature_diffusion! (E:4710-4761): marker-node
   temperature differences relaxed over dt with the marker's conductivity
   and heat capacity, markers corrected, the energy corrections scattered in
   marker order, and DT -= TKSUM / RHOCPSUM.  For rock markers the reference
   body assigns the conductivity to a loop-local name in one branch and
   indexes it in the other, which Julia rejects (UndefVarError) whenever
   dsubgridt > 0; this restatement follows the algorithm its test verifies
   (HTM-planetary.m line 1731ff, T:5480-5545) with the conductivity and heat
   capacity laws of compute_marker_properties!.  A no-op when dsubgridt == 0. */
int oracle_subgrid_temperature(const ErebusParams *p, ErebusMarkersHost *M, int64_t marknum,
                               ErebusGridHost *G, ErebusSumsHost *s, double dt) {
    if (p->dsubgridt == 0.0) return 0;
    Geo g = geo(p);
    int Ny1 = g.Ny1;
    size_t np = (size_t)g.Nx1 * Ny1;
    memset(s->TKSUM, 0, np * 8);
    memset(s->RHOCPSUM, 0, np * 8);
    const double geom = 2.0 * (1.0 / (g.dx * g.dx) + 1.0 / (g.dy * g.dy));
    for (int64_t m = 0; m < marknum; m++) {
        int i, j;
        double w[4];
        grid_weights(&g, GP, M->xm[m], M->ym[m], &i, &j, w);
        double d = M->tkm[m] - gather4(G->tk1, Ny1, i, j, w);
        int t = (int)M->tm[m];
        double tk = M->tkm[m], rcp, k;
        if (t < 3) {
            rcp = total(p->rhocpsolidm[t - 1], rhocpfluid(p, tk), M->phim[m]);
            k = ktotal(ksolid(p, tk), kfluid(p, tk), M->phim[m]);
        } else {
            rcp = p->rhocpsolidm[t - 1];
            k = p->ksolidm[t - 1];
        }
        d *= exp(-p->dsubgridt * k * dt / rcp * geom) - 1.0;
        M->tkm[m] += d;
        add_to_grid(s->TKSUM, Ny1, i, j, w, d * rcp);
        add_to_grid(s->RHOCPSUM, Ny1, i, j, w, rcp);
    }
    for (size_t q = 0; q < np; q++)
        if (s->RHOCPSUM[q] > 0.0) G->DT[q] -= s->TKSUM[q] / s->RHOCPSUM[q];
    return 0;
}

int oracle_nodes_to_markers(const ErebusParams *p, ErebusMarkersHost *M,
                            int64_t marknum, ErebusGridHost *G,
                            ErebusSumsHost *s, double dt, int timestep) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1;
    size_t np = (size_t)g.Nx1 * Ny1;
    memcpy(G->DT0, G->DT, np * 8);
#pragma omp parallel for schedule(static)
    for (int64_t m = 0; m < marknum; m++) {
        int i, j;
        double w[4];
        grid_weights(&g, GB, M->xm[m], M->ym[m], &i, &j, w);
        int t = (int)M->tm[m];
        if (t < 3)
            M->etatotalm[m] = etatotal_rocks(p, M->tkm[m], t,
                                             p->per_marker_eta ? M->etasolidm_m[m] : 0.0);
        if (AT(G->YNY, Ny, i, j) || AT(G->YNY, Ny, i + 1, j) ||
            AT(G->YNY, Ny, i, j + 1) || AT(G->YNY, Ny, i + 1, j + 1)) {
            double v = 1.0 / gather4(G->YNY_inv_ETA, Ny, i, j, w);
            M->etavpm[m] = v > M->etatotalm[m] ? M->etatotalm[m] : v;
        } else {
            M->etavpm[m] = M->etatotalm[m];
        }
    }
    oracle_subgrid_stress(p, M, marknum, G, s, dt);
#pragma omp parallel for schedule(static)
    for (int64_t m = 0; m < marknum; m++) {
        int ip, jp, ib, jb;
        double wp[4], wb[4];
        fix_weights(M->xm[m], M->ym[m], -g.dx / 2, -g.dy / 2, g.dx, g.dy, 2,
                    g.Nx - 1, 2, g.Ny - 1, &ip, &jp, wp);
        fix_weights(M->xm[m], M->ym[m], 0.0, 0.0, g.dx, g.dy, 1, g.Nx - 1, 1,
                    g.Ny - 1, &ib, &jb, wb);
        M->sxxm[m] += gather4(G->DSXX, Ny1, ip, jp, wp);
        M->sxym[m] += gather4(G->DSXY, Ny, ib, jb, wb);
    }
    oracle_subgrid_temperature(p, M, marknum, G, s, dt);
#pragma omp parallel for schedule(static)
    for (int64_t m = 0; m < marknum; m++) {
        int i, j;
        double w[4];
        grid_weights(&g, GP, M->xm[m], M->ym[m], &i, &j, w);
        if (timestep == 1) M->tkm[m] = gather4(G->tk2, Ny1, i, j, w);
        else M->tkm[m] += gather4(G->DT, Ny1, i, j, w);
    }
    memcpy(M->XWsolidm0, M->XWsolidm, (size_t)marknum * 8);
    memcpy(M->phim, M->phinewm, (size_t)marknum * 8);
#pragma omp parallel for schedule(static)
    for (int64_t m = 0; m < marknum; m++) {
        if (M->tm[m] >= 3) continue;
        int i, j;
        double w[4];
        grid_weights(&g, GP, M->xm[m], M->ym[m], &i, &j, w);
        double aphim = gather4(G->APHI, Ny1, i, j, w);
        double ph = M->phim[m];
        M->phim[m] = jmax(p->phimin, jmin(p->phimax, ph / ((1.0 - ph) * exp(aphim * dt) + ph)));
    }
    memcpy(M->phinewm, M->phim, (size_t)marknum * 8);
    oracle_melt_composition(p, M, marknum, G, s);
    return 0;
}

/* update_p_nodes_melt_composition! (E:1929-1939, with E:1883 and E:2239):
   XWsolidm0 scattered to the P nodes in marker order and normalised by the
   weights, zero where no marker contributes. */
void oracle_melt_composition(const ErebusParams *p, const ErebusMarkersHost *M,
                             int64_t marknum, ErebusGridHost *G, ErebusSumsHost *s) {
    Geo g = geo(p);
    int Ny1 = g.Ny1;
    size_t np = (size_t)g.Nx1 * Ny1;
    memset(s->XWSSUM, 0, np * 8);
    memset(s->WTPSUM, 0, np * 8);
    for (int64_t m = 0; m < marknum; m++) {
        int i, j;
        double w[4];
        grid_weights(&g, GP, M->xm[m], M->ym[m], &i, &j, w);
        add_to_grid(s->XWSSUM, Ny1, i, j, w, M->XWsolidm0[m]);
        add_to_grid(s->WTPSUM, Ny1, i, j, w, 1.0);
    }
    for (size_t k = 0; k < np; k++)
        G->XWS[k] = s->WTPSUM[k] > 0.0 ? s->XWSSUM[k] * (1.0 / s->WTPSUM[k]) : 0.0;
}

/* ------------------------------------------------------------------------ */
/* velocities and advection (E:4878-5496)                                   */
/* ------------------------------------------------------------------------ */
/* compute_velocities! (E:4878-4928) */
int oracle_velocities(const ErebusParams *p, ErebusGridHost *G) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1, Nx = g.Nx, Nx1 = g.Nx1;
    for (int j = 2; j <= Nx; j++)
        for (int i = 2; i <= Ny; i++) {
            AT(G->vxp, Ny1, i, j) = 0.5 * (AT(G->vx, Ny1, i, j) + AT(G->vx, Ny1, i, j - 1));
            AT(G->vyp, Ny1, i, j) = 0.5 * (AT(G->vy, Ny1, i, j) + AT(G->vy, Ny1, i - 1, j));
            AT(G->vxpf, Ny1, i, j) = 0.5 * (AT(G->vxf, Ny1, i, j) + AT(G->vxf, Ny1, i, j - 1));
            AT(G->vypf, Ny1, i, j) = 0.5 * (AT(G->vyf, Ny1, i, j) + AT(G->vyf, Ny1, i - 1, j));
        }
    double *V[2] = {G->vxp, G->vxpf};
    double bt[2] = {p->bctop, p->bcftop}, bb[2] = {p->bcbottom, p->bcfbottom};
    for (int f = 0; f < 2; f++) {
        double *a = V[f];
        for (int j = 2; j <= Nx - 1; j++) AT(a, Ny1, 1, j) = -bt[f] * AT(a, Ny1, 2, j);
        for (int j = 2; j <= Nx - 1; j++) AT(a, Ny1, Ny1, j) = -bb[f] * AT(a, Ny1, Ny, j);
        for (int i = 1; i <= Ny1; i++) AT(a, Ny1, i, 1) = 2.0 * g.vxleft - AT(a, Ny1, i, 2);
        for (int i = 1; i <= Ny1; i++) AT(a, Ny1, i, Nx1) = 2.0 * g.vxright - AT(a, Ny1, i, Nx);
    }
    double *W[2] = {G->vyp, G->vypf};
    double bl[2] = {p->bcleft, p->bcfleft}, br[2] = {p->bcright, p->bcfright};
    for (int f = 0; f < 2; f++) {
        double *a = W[f];
        for (int i = 2; i <= Ny - 1; i++) AT(a, Ny1, i, 1) = -bl[f] * AT(a, Ny1, i, 2);
        for (int i = 2; i <= Ny - 1; i++) AT(a, Ny1, i, Nx1) = -br[f] * AT(a, Ny1, i, Nx);
        for (int j = 1; j <= Nx1; j++) AT(a, Ny1, 1, j) = 2.0 * g.vytop - AT(a, Ny1, 2, j);
        for (int j = 1; j <= Nx1; j++) AT(a, Ny1, Ny1, j) = 2.0 * g.vybottom - AT(a, Ny1, Ny, j);
    }
    return 0;
}

/* compute_rotation_rate! (E:4946-4956) */
int oracle_rotation_rate(const ErebusParams *p, ErebusGridHost *G) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1;
    for (int j = 1; j <= g.Nx; j++)
        for (int i = 1; i <= Ny; i++)
            AT(G->wyx, Ny, i, j) =
                0.5 * ((AT(G->vy, Ny1, i, j + 1) - AT(G->vy, Ny1, i, j)) * (1.0 / g.dx) -
                       (AT(G->vx, Ny1, i + 1, j) - AT(G->vx, Ny1, i, j)) * (1.0 / g.dy));
    return 0;
}

/* Interpolated vx at (x,y) with the second-order correction of E:5057-5091.
   `quirk` selects the E:5173 form (vx[i,j] in place of vxf[i,j] in the
   left-half correction of the fluid velocity); vq is then vx. */
static inline double vx_at(const Geo *g, const double *v, const double *vq,
                           int quirk, double x, double y, int form) {
    int i, j, Ny1 = g->Ny1;
    double dxmj, dymi;
    fix_distances(x, y, 0.0, -g->dy / 2, g->dx, g->dy, 1, g->Nx - 1, 1, g->Ny,
                  &i, &j, &dxmj, &dymi);
    double dx = g->dx, dy = g->dy;
    double v13 = AT(v, Ny1, i, j) * (1.0 - dxmj / dx) + AT(v, Ny1, i, j + 1) * dxmj / dx;
    double v24 = AT(v, Ny1, i + 1, j) * (1.0 - dxmj / dx) + AT(v, Ny1, i + 1, j + 1) * dxmj / dx;
    if (dxmj / dx >= 0.5) {
        if (j < g->Nx - 1) {
            double q = dxmj / dx - 0.5;
            v13 += 0.5 * (q * q) * (AT(v, Ny1, i, j) - 2.0 * AT(v, Ny1, i, j + 1) + AT(v, Ny1, i, j + 2));
            v24 += 0.5 * (q * q) * (AT(v, Ny1, i + 1, j) - 2.0 * AT(v, Ny1, i + 1, j + 1) + AT(v, Ny1, i + 1, j + 2));
        }
    } else {
        if (j > 1) {
            double q = dxmj / dx - 0.5;
            const double *c = quirk ? vq : v;
            v13 += 0.5 * (q * q) * (AT(v, Ny1, i, j - 1) - 2.0 * AT(c, Ny1, i, j) + AT(v, Ny1, i, j + 1));
            v24 += 0.5 * (q * q) * (AT(v, Ny1, i + 1, j - 1) - 2.0 * AT(v, Ny1, i + 1, j) + AT(v, Ny1, i + 1, j + 1));
        }
    }
    /* form 0: move_markers_rk4! (E:5091); form 1: backtrace (E:5332) */
    if (form == 0) return v13 * (1.0 - dymi / dy) + v24 * dymi / dy;
    return (1.0 - dymi / dy) * v13 + (dymi / dy) * v24;
}

/* Interpolated vy at (x,y) with the correction of E:5093-5127. */
static inline double vy_at(const Geo *g, const double *v, double x, double y,
                           int form) {
    int i, j, Ny1 = g->Ny1;
    double dxmj, dymi;
    fix_distances(x, y, -g->dx / 2, 0.0, g->dx, g->dy, 1, g->Nx, 1, g->Ny - 1,
                  &i, &j, &dxmj, &dymi);
    double dx = g->dx, dy = g->dy;
    double v12 = AT(v, Ny1, i, j) * (1.0 - dymi / dy) + AT(v, Ny1, i + 1, j) * dymi / dy;
    double v34 = AT(v, Ny1, i, j + 1) * (1.0 - dymi / dy) + AT(v, Ny1, i + 1, j + 1) * dymi / dy;
    if (dymi / dy >= 0.5) {
        if (i < g->Ny - 1) {
            double q = dymi / dy - 0.5;
            v12 += 0.5 * (q * q) * (AT(v, Ny1, i, j) - 2.0 * AT(v, Ny1, i + 1, j) + AT(v, Ny1, i + 2, j));
            v34 += 0.5 * (q * q) * (AT(v, Ny1, i, j + 1) - 2.0 * AT(v, Ny1, i + 1, j + 1) + AT(v, Ny1, i + 2, j + 1));
        }
    } else {
        if (i > 1) {
            double q = dymi / dy - 0.5;
            v12 += 0.5 * (q * q) * (AT(v, Ny1, i - 1, j) - 2.0 * AT(v, Ny1, i, j) + AT(v, Ny1, i + 1, j));
            v34 += 0.5 * (q * q) * (AT(v, Ny1, i - 1, j + 1) - 2.0 * AT(v, Ny1, i, j + 1) + AT(v, Ny1, i + 1, j + 1));
        }
    }
    if (form == 0) return v12 * (1.0 - dxmj / dx) + v34 * dxmj / dx;
    return (1.0 - dxmj / dx) * v12 + (dxmj / dx) * v34;
}

static const double BRK4[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
static const double CRK4[3] = {0.5, 0.5, 1.0};

/* move_markers_rk4! (E:4990-5257).  Serial in the reference; markers are
   independent, so the loop order does not change results. */
int oracle_move_markers_rk4(const ErebusParams *p, ErebusMarkersHost *M,
                            int64_t marknum, const ErebusGridHost *G,
                            double dt) {
    Geo g = geo(p);
    int Ny = g.Ny, Ny1 = g.Ny1;
#pragma omp parallel for schedule(static)
    for (int64_t m = 0; m < marknum; m++) {
        double xmm = M->xm[m], ymm = M->ym[m];
        int i, j;
        double w[4];
        grid_weights(&g, GP, xmm, ymm, &i, &j, w);
        double tksm0 = gather4(G->tk2, Ny1, i, j, w);
        grid_weights(&g, GB, xmm, ymm, &i, &j, w);
        double om = gather4(G->wyx, Ny, i, j, w);
        double th = dt * om;
        double c = cos(th), s = sin(th), s2 = sin(2.0 * th), c2 = cos(2.0 * th);
        double sxx = M->sxxm[m], sxy = M->sxym[m];
        M->sxxm[m] = sxx * (c * c) - sxx * (s * s) - sxy * s2;
        M->sxym[m] = sxx * s2 + sxy * c2;
        double vxr[4] = {0, 0, 0, 0}, vyr[4] = {0, 0, 0, 0};
        double xr = xmm, yr = ymm;
        for (int rk = 0; rk < 4; rk++) {
            vxr[rk] = 0.0 + vx_at(&g, G->vx, G->vx, 0, xr, yr, 0);
            vyr[rk] = 0.0 + vy_at(&g, G->vy, xr, yr, 0);
            if (rk < 3) {
                xr = xmm + dt * CRK4[rk] * vxr[rk];
                yr = ymm + dt * CRK4[rk] * vyr[rk];
            }
        }
        M->xm[m] += dt * (BRK4[0] * vxr[0] + BRK4[1] * vxr[1] + BRK4[2] * vxr[2] + BRK4[3] * vxr[3]);
        M->ym[m] += dt * (BRK4[0] * vyr[0] + BRK4[1] * vyr[1] + BRK4[2] * vyr[2] + BRK4[3] * vyr[3]);
        xmm = xr = M->xm[m];
        ymm = yr = M->ym[m];
        for (int rk = 0; rk < 4; rk++) {
            vxr[rk] = 0.0 + vx_at(&g, G->vxf, G->vx, 1, xr, yr, 0);
            vyr[rk] = 0.0 + vy_at(&g, G->vyf, xr, yr, 0);
            if (rk < 3) {
                xr = xmm - dt * CRK4[rk] * vxr[rk];
                yr = ymm - dt * CRK4[rk] * vyr[rk];
            }
        }
        xr = xmm - dt * (BRK4[0] * vxr[0] + BRK4[1] * vxr[1] + BRK4[2] * vxr[2] + BRK4[3] * vxr[3]);
        yr = ymm - dt * (BRK4[0] * vyr[0] + BRK4[1] * vyr[1] + BRK4[2] * vyr[2] + BRK4[3] * vyr[3]);
        grid_weights(&g, GP, xr, yr, &i, &j, w);
        double tkfm0 = gather4(G->tk2, Ny1, i, j, w);
        double d = tkfm0 - tksm0;
        int t = (int)M->tm[m];
        double ph = M->phim[m], tk = M->tkm[m];
        double rcs = p->rhocpsolidm[t - 1], rcf = rhocpfluid(p, tk);
        M->tkm[m] = ((1.0 - ph) * tk * rcs + ph * (tk + d) * rcf) /
                    ((1.0 - ph) * rcs + ph * rcf);
    }
    return 0;
}

/* backtrace_pressures_rk4! (E:5284-5496) */
int oracle_backtrace_pressures(const ErebusParams *p, ErebusGridHost *G,
                               double dt) {
    Geo g = geo(p);
    int Ny1 = g.Ny1;
    size_t np = (size_t)g.Nx1 * Ny1;
    memcpy(G->pr0, G->pr, np * 8);
    memcpy(G->ps0, G->ps, np * 8);
    for (int pass = 0; pass < 2; pass++) {
        const double *vx = pass == 0 ? G->vx : G->vxf;
        const double *vy = pass == 0 ? G->vy : G->vyf;
        if (pass == 1) memcpy(G->pf0, G->pf, np * 8);
        for (int jj = 2; jj <= g.Nx; jj++)
            for (int ii = 2; ii <= g.Ny; ii++) {
                double xA = ax(-g.dx / 2, g.dx, jj), yA = ax(-g.dy / 2, g.dy, ii);
                double xc = xA, yc = yA, vxm[4], vym[4];
                for (int rk = 0; rk < 4; rk++) {
                    vxm[rk] = vx_at(&g, vx, vx, 0, xc, yc, 1);
                    vym[rk] = vy_at(&g, vy, xc, yc, 1);
                    if (rk == 0 || rk == 1) {
                        xc = xA - 0.5 * dt * vxm[rk];
                        yc = yA - 0.5 * dt * vym[rk];
                    } else if (rk == 2) {
                        xc = xA - dt * vxm[rk];
                        yc = yA - dt * vym[rk];
                    }
                }
                xc = xA - dt * (1.0 / 6.0) * (vxm[0] + 2 * vxm[1] + 2 * vxm[2] + vxm[3]);
                yc = yA - dt * (1.0 / 6.0) * (vym[0] + 2 * vym[1] + 2 * vym[2] + vym[3]);
                int i, j;
                double w[4];
                grid_weights(&g, GP, xc, yc, &i, &j, w);
                if (pass == 0) {
                    AT(G->pr0, Ny1, ii, jj) = gather4(G->pr, Ny1, i, j, w);
                    AT(G->ps0, Ny1, ii, jj) = gather4(G->ps, Ny1, i, j, w);
                } else {
                    AT(G->pf0, Ny1, ii, jj) = gather4(G->pf, Ny1, i, j, w);
                }
            }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* replenishment (E:5518-5698)                                              */
/* ------------------------------------------------------------------------ */
/* counter-based uniform variate in [0,1): the jitter of a replenished marker
   (the reference draws it from its global MersenneTwister, E:5659). */
static inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double oracle_u01(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t z = splitmix64(seed ^ splitmix64(stream ^ splitmix64(idx)));
    return (double)(z >> 11) * 0x1.0p-53;
}

/* replenish_markers! (E:5586-5698).  mdis (Nym*Nxm) and mnum (Nym*Nxm)
   are scratch.  New markers are appended in anchor order; returns the new
   marker count, or -1 if `capacity` would be exceeded. */
int64_t oracle_replenish(const ErebusParams *p, ErebusMarkersHost *M,
                         int64_t marknum, int64_t capacity, double *mdis,
                         int64_t *mnum, int timestep) {
    Geo g = geo(p);
    int Nxm = g.Nxm, Nym = g.Nym;
    size_t na = (size_t)Nxm * Nym;
    for (size_t k = 0; k < na; k++) { mdis[k] = 1.0e30; mnum[k] = 0; }
    double x0 = g.dxm / 2, y0 = g.dym / 2;
    for (int64_t m = 0; m < marknum; m++) {
        int i, j;
        fix(M->xm[m], M->ym[m], x0, y0, g.dxm, g.dym, 1, Nxm - 1, 1, Nym - 1, &i, &j);
        /* update_marker_population_geometry! (E:5518-5544) */
        for (int c = 0; c < 4; c++) {
            int ii = i + (c & 1), jj = j + (c >> 1);
            double ddx = M->xm[m] - ax(x0, g.dxm, jj), ddy = M->ym[m] - ax(y0, g.dym, ii);
            double d = sqrt(ddx * ddx + ddy * ddy);
            if (d < AT(mdis, Nym, ii, jj)) {
                AT(mdis, Nym, ii, jj) = d;
                AT(mnum, Nym, ii, jj) = m + 1;
            }
        }
    }
    int dii = 5 * p->Nymc, djj = 5 * p->Nxmc;
    int64_t n = marknum;
    for (int j = 1; j <= Nxm; j++)
        for (int i = 1; i <= Nym; i++) {
            if (AT(mnum, Nym, i, j) != 0) continue;
            double xa = ax(x0, g.dxm, j), ya = ax(y0, g.dym, i);
            int jlo = j - djj > 1 ? j - djj : 1, jhi = j + djj < Nxm ? j + djj : Nxm;
            int ilo = i - dii > 1 ? i - dii : 1, ihi = i + dii < Nym ? i + dii : Nym;
            for (int jj = jlo; jj <= jhi; jj++)
                for (int ii = ilo; ii <= ihi; ii++) {
                    int64_t mm = AT(mnum, Nym, ii, jj);
                    if (mm > 0) {
                        double ddx = M->xm[mm - 1] - xa, ddy = M->ym[mm - 1] - ya;
                        double d = sqrt(ddx * ddx + ddy * ddy);
                        if (d < AT(mdis, Nym, i, j)) {
                            AT(mdis, Nym, i, j) = d;
                            AT(mnum, Nym, i, j) = -mm;
                        }
                    }
                }
            if (AT(mnum, Nym, i, j) < 0) {
                if (n >= capacity) return -1;
                int64_t src = -AT(mnum, Nym, i, j) - 1;
                uint64_t anchor = (uint64_t)(j - 1) * Nym + (i - 1);
                if (p->random_markers) {
                    M->xm[n] = xa + (oracle_u01(p->seed, 2 * (uint64_t)timestep, anchor) - 0.5) * g.dxm;
                    M->ym[n] = ya + (oracle_u01(p->seed, 2 * (uint64_t)timestep + 1, anchor) - 0.5) * g.dym;
                } else {
                    M->xm[n] = xa;
                    M->ym[n] = ya;
                }
                M->tm[n] = M->tm[src];
                double *F[] = {M->tkm, M->phim, M->sxxm, M->sxym, M->etavpm,
                               M->phinewm, M->pfm0, M->XWsolidm, M->XWsolidm0,
                               M->rhototalm, M->rhocptotalm, M->etatotalm,
                               M->hrtotalm, M->ktotalm, M->inv_gggtotalm,
                               M->fricttotalm, M->cohestotalm, M->tenstotalm,
                               M->rhofluidcur, M->alphasolidcur,
                               M->alphafluidcur, M->tkm_rhocptotalm,
                               M->etafluidcur_inv_kphim, M->etasolidm_m};
                for (size_t f = 0; f < sizeof F / sizeof *F; f++)
                    if (F[f]) F[f][n] = F[f][src];
                n++;
            }
        }
    return n;
}

/* ------------------------------------------------------------------------ */
/* hooks for the tests that re-express the reference's unit tests          */
/* ------------------------------------------------------------------------ */
void oracle_fix_grid(const ErebusParams *p, int grid, double x, double y, int *i, int *j) {
    Geo g = geo(p);
    double w[4];
    grid_weights(&g, grid, x, y, i, j, w);
}
void oracle_weights_grid(const ErebusParams *p, int grid, double x, double y, int *i,
                         int *j, double *w) {
    Geo g = geo(p);
    grid_weights(&g, grid, x, y, i, j, w);
}
double oracle_ktotal(double ks, double kf, double phi) { return ktotal(ks, kf, phi); }
double oracle_total(double s, double f, double phi) { return total(s, f, phi); }
double oracle_etaf_inv_kphi(const ErebusParams *p, double k0, double phi, double etaf) {
    return etaf_inv_kphi(p, k0, phi, etaf);
}
double oracle_Q_radiogenic(double f, double ratio, double E, double tau, double t) {
    return Q_radiogenic(f, ratio, E, tau, t);
}
void oracle_radioactive_heating(const ErebusParams *p, double timesum, double *hrs,
                                double *hrf) {
    Geo g = geo(p);
    radioactive_heating(p, &g, timesum, hrs, hrf);
}
double oracle_dtreaction(const ErebusParams *p, double T, double phi) {
    return dtreaction_of(p, T, phi);
}
double oracle_rhocpfluid(const ErebusParams *p, double T) { return rhocpfluid(p, T); }
double oracle_ksolid(const ErebusParams *p, double T) { return ksolid(p, T); }
double oracle_kfluid(const ErebusParams *p, double T) { return kfluid(p, T); }
double oracle_gibbs(const ErebusParams *p, double T, double pf, double XD, double XW,
                    double dt, double dtr) {
    Geo g = geo(p);
    return gibbs(p, &g, T, pf, XD, XW, dt, dtr);
}
double oracle_rel_enthalpy(const ErebusParams *p, double Xs, double XW) {
    return rel_enthalpy(p, Xs, XW);
}
double oracle_reaction_constant(const ErebusParams *p, double T, double pf, double dG) {
    Geo g = geo(p);
    return reaction_constant(p, &g, T, pf, dG);
}
/* marker_to_{basic,vx,vy,p}_nodes! over given marker properties (no
   compute_marker_properties!), as the reference's scatter tests call them */
void oracle_scatter_only(const ErebusParams *p, const ErebusMarkersHost *M, int64_t n,
                         ErebusSumsHost *s) {
    Geo g = geo(p);
    reset_sums(&g, s);
    for (int64_t m = 0; m < n; m++) scatter_marker(&g, M, m, s);
}
void oracle_node_properties(const ErebusParams *p, const ErebusSumsHost *s,
                            ErebusGridHost *G) {
    Geo g = geo(p);
    node_properties(&g, s, G);
}
void oracle_insulating_bc(const ErebusParams *p, double *t) {
    Geo g = geo(p);
    insulating_bc(&g, t);
}
