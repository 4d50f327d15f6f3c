// common.cuh -- shared device definitions of liberebus_b200.
//
// Grid geometry, the marker->cell index (`fix`, src/Erebus.jl:1456-1470),
// distances and bilinear weights (E:1388-1431) with the reference's exact
// arithmetic order.  The library is compiled with --fmad=false so that every
// a*b+c is rounded twice as in the reference; kernels that want fused
// multiply-adds (the dense LU) call fma() explicitly.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/erebus_b200.h"

#define EREBUS_HD __host__ __device__ __forceinline__

// Column-major element (i,j), 1-based, of an array with `rows` rows.
#define AT(A, rows, i, j) (A)[((int64_t)(j) - 1) * (rows) + ((i) - 1)]

namespace erebus {

constexpr int kThreads = 256;

struct Geo {
    int Nx, Ny, Nx1, Ny1, Nxm, Nym;
    double dx, dy, dxm, dym, xcenter, ycenter;
    double VDs, VWs, VH2Of, VH2Ofi, dVWD, tau_al, tau_fe;
    double vxleft, vxright, vytop, vybottom;
};

// Derived constants of src/constants.jl (C:25-124, C:196-259, C:303-310).
inline Geo make_geo(const ErebusParams &p) {
    Geo g;
    g.Nx = p.Nx; g.Ny = p.Ny; g.Nx1 = p.Nx + 1; g.Ny1 = p.Ny + 1;
    g.dx = p.xsize / (p.Nx - 1);
    g.dy = p.ysize / (p.Ny - 1);
    g.Nxm = (p.Nx - 1) * p.Nxmc;
    g.Nym = (p.Ny - 1) * p.Nymc;
    g.dxm = p.xsize / g.Nxm;
    g.dym = p.ysize / g.Nym;
    g.xcenter = p.xsize / 2;
    g.ycenter = p.ysize / 2;
    g.VDs = p.MD / p.rhoDs;
    g.VWs = (p.MD + p.MH2O) / p.rhoWs;
    g.VH2Of = p.MH2O / p.rhoH2Of;
    g.VH2Ofi = p.MH2O / p.rhoH2Ofi;
    g.dVWD = g.VDs + g.VH2Of - g.VWs;
    g.tau_al = p.t_half_al / log(2.0);
    g.tau_fe = p.t_half_fe / log(2.0);
    g.vxleft = p.strainrate * p.xsize / 2;
    g.vxright = -p.strainrate * p.xsize / 2;
    g.vytop = -p.strainrate * p.ysize / 2;
    g.vybottom = p.strainrate * p.ysize / 2;
    return g;
}

// Axis value: origin + (k-1)*step (all configured steps are exact).
EREBUS_HD double ax(double origin, double step, int k) {
    return origin + (double)(k - 1) * step;
}

// Julia max/min on floats: NaN propagates.
EREBUS_HD double jmax(double a, double b) {
    if (a != a || b != b) return a + b;   // NaN
    return a > b ? a : b;
}
EREBUS_HD double jmin(double a, double b) {
    if (a != a || b != b) return a + b;   // NaN
    return a < b ? a : b;
}

// unsafe_trunc(Int, v); out-of-range and NaN map far below any clamp bound.
EREBUS_HD int64_t jtrunc(double v) {
    if (!(v > -4.0e18 && v < 4.0e18)) return INT64_MIN / 2;
    return (int64_t)v;
}

// fix (E:1456-1470)
EREBUS_HD void fix(double x, double y, double x0, double y0, double dx,
                   double dy, int jmin_, int jmax_, int imin_, int imax_,
                   int &iout, int &jout) {
    int64_t j = jtrunc((x - x0) * (1.0 / dx)) + 1;
    int64_t i = jtrunc((y - y0) * (1.0 / dy)) + 1;
    if (j < jmin_) j = jmin_;
    else if (j > jmax_) j = jmax_;
    if (i < imin_) i = imin_;
    else if (i > imax_) i = imax_;
    iout = (int)i;
    jout = (int)j;
}

// fix_distances (E:1424-1431)
EREBUS_HD void fix_distances(double x, double y, double x0, double y0,
                             double dx, double dy, int jmin_, int jmax_,
                             int imin_, int imax_, int &i, int &j,
                             double &dxmj, double &dymi) {
    fix(x, y, x0, y0, dx, dy, jmin_, jmax_, imin_, imax_, i, j);
    dxmj = x - ax(x0, dx, j);
    dymi = y - ax(y0, dy, i);
}

// fix_weights (E:1388-1397): nodes (i,j),(i+1,j),(i,j+1),(i+1,j+1)
EREBUS_HD void fix_weights(double x, double y, double x0, double y0,
                           double dx, double dy, int jmin_, int jmax_,
                           int imin_, int imax_, int &i, int &j,
                           double w[4]) {
    double dxmj, dymi;
    fix_distances(x, y, x0, y0, dx, dy, jmin_, jmax_, imin_, imax_, i, j,
                  dxmj, dymi);
    w[0] = (1.0 - dymi / dy) * (1.0 - dxmj / dx);
    w[1] = (dymi / dy) * (1.0 - dxmj / dx);
    w[2] = (1.0 - dymi / dy) * (dxmj / dx);
    w[3] = (dymi / dy) * (dxmj / dx);
}

enum Grid { GB = 0, GVX = 1, GVY = 2, GP = 3 };

// Origins and clamp ranges of the four node sets (C:40-101).
struct GridSpec {
    double x0, y0;
    int jmin, jmax, imin, imax, rows, cols;
};

EREBUS_HD GridSpec grid_spec(const Geo &g, int grid) {
    GridSpec s;
    switch (grid) {
    case GB:
        s = {0.0, 0.0, 1, g.Nx - 1, 1, g.Ny - 1, g.Ny, g.Nx};
        break;
    case GVX:
        s = {0.0, -g.dy / 2, 1, g.Nx - 1, 1, g.Ny, g.Ny1, g.Nx1};
        break;
    case GVY:
        s = {-g.dx / 2, 0.0, 1, g.Nx, 1, g.Ny - 1, g.Ny1, g.Nx1};
        break;
    default:
        s = {-g.dx / 2, -g.dy / 2, 1, g.Nx, 1, g.Ny, g.Ny1, g.Nx1};
        break;
    }
    return s;
}

EREBUS_HD void grid_weights(const Geo &g, int grid, double x, double y,
                            int &i, int &j, double w[4]) {
    GridSpec s = grid_spec(g, grid);
    fix_weights(x, y, s.x0, s.y0, g.dx, g.dy, s.jmin, s.jmax, s.imin, s.imax,
                i, j, w);
}

// dot4(grid_vector(i,j,A), w) (E:1137, E:1157)
EREBUS_HD double gather4(const double *A, int rows, int i, int j,
                         const double w[4]) {
    return AT(A, rows, i, j) * w[0] + AT(A, rows, i + 1, j) * w[1] +
           AT(A, rows, i, j + 1) * w[2] + AT(A, rows, i + 1, j + 1) * w[3];
}

// grid_average (E:1176-1180)
EREBUS_HD double grid_average(const double *A, int rows, int i, int j) {
    return 0.25 * (AT(A, rows, i, j) + AT(A, rows, i + 1, j) +
                   AT(A, rows, i, j + 1) + AT(A, rows, i + 1, j + 1));
}

// counter-based uniform variate in [0,1) (splitmix64)
EREBUS_HD uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
EREBUS_HD double u01(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t z = splitmix64(seed ^ splitmix64(stream ^ splitmix64(idx)));
    return (double)(z >> 11) * 0x1.0p-53;
}

// Grid size for n items (at least one block: every kernel checks its
// index against n, and an empty marker set is a valid input).
inline int nblocks(int64_t n, int threads = kThreads) {
    int64_t b = (n + threads - 1) / threads;
    return b > 0 ? (int)b : 1;
}

}  // namespace erebus
