// laws.cuh -- pointwise material laws of the marker properties, and the
// temperature derivatives the adjoint of the heat path needs.
#pragma once
#include "common.cuh"

namespace erebus {

// ---------------------------------------------------------------------------
// material laws (E:1116-1275, E:2272-2397)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double total(double s, double f, double phi) {
    return s * (1.0 - phi) + f * phi;
}
__device__ __forceinline__ double ktotal(double ks, double kf, double phi) {
    double a = ks * (3.0 * phi - 2.0) + kf * (1.0 - 3.0 * phi);
    return sqrt(ks * kf / 2 + (a * a) * (1.0 / 16.0)) -
           0.25 * (ks * (3.0 * phi - 2.0) + kf * (1.0 - 3.0 * phi));
}
// x^3 with one final rounding of a compensated product (Julia evaluates a
// Float64 power with an integral exponent by compensated repeated
// multiplication); x^2 is a single correctly rounded product.
__device__ __forceinline__ double cube(double x) {
    double hi = x * x, lo = fma(x, x, -hi);
    double p = hi * x, e = fma(hi, x, -p);
    return p + (e + lo * x);
}
__device__ __forceinline__ double etaf_inv_kphi(const ErebusParams &p, double k0,
                                                double phi, double etaf) {
    double r = (1.0 - phi) * (1.0 / (1.0 - p.phim0));
    return etaf * (1.0 / k0) * cube(p.phim0 * (1.0 / phi)) * (r * r);
}
__device__ __forceinline__ double rhocpfluid(const ErebusParams &p, double T) {
    if (p.marker_property_mode == 1) {
        double tm = p.tmfluidphase;
        if (T < tm - 5.0) return p.rhoH2Ofi * (7.67 * T);
        if (T < tm) return p.rhoH2Ofi * (7.67 * T + 0.1 * p.Lf);
        if (T < tm + 5.0) return p.rhoH2Of * (4200.0 + 0.1 * p.Lf);
        if (T < 410.0) return p.rhoH2Of * 4200.0;
        return p.rhoH2Of *
               (-4.67e4 + 333 * T - 0.731 * (T * T) + 5.4e-4 * (T * T * T));
    }
    return p.rhocpfluidm[0];
}
__device__ __forceinline__ double ksolid(const ErebusParams &p, double T) {
    if (p.marker_property_mode == 1) return 0.73 + 1293.0 / (T + 77.0);
    return p.ksolidm[0];
}
__device__ __forceinline__ double kfluid(const ErebusParams &p, double T) {
    if (p.marker_property_mode == 1) {
        if (T < p.tmfluidphase) return 0.465 + 488.0 / T;
        if (T < 410) return -0.581 + 6.34e-3 * T - 7.93e-6 * (T * T);
        return -0.142 + 4.12e-3 * T - 5.01e-6 * (T * T);
    }
    return p.kfluidm[0];
}
__device__ __forceinline__ double dtreaction_of(const ErebusParams &p, double T,
                                                double phi) {
    switch (p.reaction_rate_coeff_mode) {
    case 1: {
        double d = T - p.c_I;
        return -p.log_completion_rate / (p.A_I * phi) * exp(p.b_I * (d * d));
    }
    case 2:
        return -p.log_completion_rate / (p.Sxo_B * phi) *
               pow(2.0, (p.To_B - T) / p.Tscl_B);
    case 3:
        return -p.log_completion_rate / (p.Sxo_B * phi) *
               exp(p.Ea_T / p.RG * (1.0 / T - 1.0 / p.To_T));
    default:
        return p.dtreaction;
    }
}

// d/dT of the laws above (zero where a law is constant in T, and in the
// constant-property mode); each piece is the derivative of the branch the law
// takes at T.
__device__ __forceinline__ double rhocpfluid_dT(const ErebusParams &p, double T) {
    if (p.marker_property_mode == 1) {
        double tm = p.tmfluidphase;
        if (T < tm) return p.rhoH2Ofi * 7.67;
        if (T < 410.0) return 0.0;
        return p.rhoH2Of * (333 - 2.0 * 0.731 * T + 3.0 * 5.4e-4 * (T * T));
    }
    return 0.0;
}
__device__ __forceinline__ double ksolid_dT(const ErebusParams &p, double T) {
    if (p.marker_property_mode == 1) return -1293.0 / ((T + 77.0) * (T + 77.0));
    return 0.0;
}
__device__ __forceinline__ double kfluid_dT(const ErebusParams &p, double T) {
    if (p.marker_property_mode == 1) {
        if (T < p.tmfluidphase) return -488.0 / (T * T);
        if (T < 410) return 6.34e-3 - 2.0 * 7.93e-6 * T;
        return 4.12e-3 - 2.0 * 5.01e-6 * T;
    }
    return 0.0;
}
// Partial derivatives of ktotal(ks, kf, phi) (E:1226-1234).
struct KtotalGrad {
    double ks, kf, phi;
};
__device__ __forceinline__ KtotalGrad ktotal_grad(double ks, double kf, double phi) {
    double a = ks * (3.0 * phi - 2.0) + kf * (1.0 - 3.0 * phi);
    double r = sqrt(ks * kf / 2 + (a * a) * (1.0 / 16.0));
    double da = a / (16.0 * r) - 0.25;   // d ktotal / d a
    KtotalGrad gr;
    gr.ks = kf / (4.0 * r) + da * (3.0 * phi - 2.0);
    gr.kf = ks / (4.0 * r) + da * (1.0 - 3.0 * phi);
    gr.phi = da * 3.0 * (ks - kf);
    return gr;
}

}  // namespace erebus
