// device_physics.cuh -- per-bond and per-pair physics of the ChainIntegrator
// step as sm_100a device functions (FP64).
//
// Each function keeps the reference's operand order and grouping; compiled
// with --fmad=false (the plain form) it rounds like the reference's x86-64
// build, up to the CUDA libm (pow/exp/acos/cos/cbrt/sin, <= 2 ulp).
// Citations are relative to the bdsim project root.
#pragma once

#include <math.h>
#include <stdint.h>

#include "bdcu_internal.h"

namespace bdcu {

constexpr double kPi = 3.14159265358979323846;  // src/types.hpp:22
constexpr double kMyEps = 1e-6;                 // src/types.hpp:24

// std::min / std::max semantics (NaN behaviour included).
__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax_(double a, double b) { return (a < b) ? b : a; }

// force_sans_hookean (src/spring.cpp:14-37)
__device__ inline double force_factor(int type, double q, double q0) {
    switch (type) {
        case BDCU_SPRING_HOOK: return 1.0;
        case BDCU_SPRING_FENE: return 1.0 / (1.0 - q * q);
        case BDCU_SPRING_ILC: return (3.0 - q * q) / (1.0 - q * q) / 3.0;
        case BDCU_SPRING_WLC: return 1.0 / (6.0 * q) * (4.0 * q + 1.0 / (1.0 - q) / (1.0 - q) - 1.0);
        case BDCU_SPRING_FRAENKEL: return 1.0 * (1.0 - (q0 / q));
        case BDCU_SPRING_FENE_FRAENKEL: return (1.0 - q0 / q) / (1.0 - (q - q0) * (q - q0));
        case BDCU_SPRING_WLC_BOUNDED: {
            const double t = (q - q0) / (1.0 - q0);
            return (2.0 / (3.0 * q)) * ((pow(1.0 - t, -2.0) - 1.0) / 4.0 + t -
                                        q0 * (pow(1.0 + t, -2.0) - 1.0) / 4.0 + q0 * t);
        }
    }
    return 1.0;
}

__device__ __forceinline__ double cubic_at(const double c[4], double x) {
    return ((c[3] * x + c[2]) * x + c[1]) * x + c[0];
}

// bisect_cubic (src/numerics.cpp:8-23)
__device__ inline double bisect_cubic(const double c[4], double lo, double hi) {
    double flo = cubic_at(c, lo), fhi = cubic_at(c, hi);
    if (flo == 0.0) return lo;
    if (fhi == 0.0) return hi;
    if (flo * fhi > 0.0) return (fabs(flo) < fabs(fhi)) ? lo : hi;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        const double fm = cubic_at(c, mid);
        if (fm == 0.0 || (hi - lo) < 1e-15) return mid;
        if (flo * fm < 0.0) {
            hi = mid;
            fhi = fm;
        } else {
            lo = mid;
            flo = fm;
        }
    }
    return 0.5 * (lo + hi);
}

// find_roots_cubic (src/numerics.cpp:25-59)
__device__ inline double find_roots_cubic(const double c4[4], double lower, double upper) {
    const double a = c4[2] / c4[3];
    const double b = c4[1] / c4[3];
    const double c = c4[0] / c4[3];
    const double Q = (a * a - 3.0 * b) / 9.0;
    const double R = (2.0 * a * a * a - 9.0 * a * b + 27.0 * c) / 54.0;
    double x;
    if (R * R < Q * Q * Q) {
        const double theta = acos(R / sqrt(Q * Q * Q));
        for (int i = -1; i <= 1; ++i) {
            x = -2.0 * sqrt(Q) * cos((theta + (double)i * kPi * 2.0) / 3.0) - a / 3.0;
            if (x >= lower && x <= upper) return x;
        }
        x = -2.0 * sqrt(Q) * cos((theta + kPi * 2.0) / 3.0) - a / 3.0;
    } else {
        const double Au = -copysign(1.0, R) * cbrt(fabs(R) + sqrt(R * R - Q * Q * Q));
        const double Bu = (Au == 0.0) ? 0.0 : Q / Au;
        x = (Au + Bu) - a / 3.0;
    }
    if (x >= lower && x <= upper) return x;
    return bisect_cubic(c4, lower, upper);
}

// polish_poly_root for the cubic (src/numerics.cpp:61-85)
__device__ inline double polish_root(const double c[4], double x0, double atol) {
    double x = x0;
    for (int iter = 0; iter < 30; ++iter) {
        double p = c[3] * x + c[2];
        double p1 = c[3];
        p1 = p + p1 * x;
        p = c[1] + p * x;
        p1 = p + p1 * x;
        p = c[0] + p * x;
        if (fabs(p1) == 0.0) {
            p1 = 6.0 * c[3];
            p1 = 6.0 * p / p1;
            x -= copysign(1.0, p1) * cbrt(fabs(p1));
        } else {
            x -= p / p1;
        }
        if (fabs(p) <= atol) break;
    }
    return x;
}

// cubic_coefficients (src/spring.cpp:55-87)
__device__ inline void cubic_coefficients(int type, double dtby4, double gama, double natscl, double c[4]) {
    c[0] = 0.0;
    c[1] = 0.0;
    c[2] = 0.0;
    c[3] = 1.0;
    switch (type) {
        case BDCU_SPRING_FENE:
            c[0] = gama;
            c[1] = -(1.0 + dtby4);
            c[2] = -gama;
            break;
        case BDCU_SPRING_ILC: {
            const double d = 3.0 + dtby4;
            c[0] = 3.0 * gama / d;
            c[1] = -(3.0 + 3.0 * dtby4) / d;
            c[2] = -3.0 * gama / d;
            break;
        }
        case BDCU_SPRING_WLC: {
            const double d = 2.0 * (1.5 + dtby4);
            c[0] = -3.0 * gama / d;
            c[1] = 3.0 * (1.0 + dtby4 + 2.0 * gama) / d;
            c[2] = -1.5 * (4.0 + 3.0 * dtby4 + 2.0 * gama) / d;
            break;
        }
        case BDCU_SPRING_FENE_FRAENKEL:
            c[0] = dtby4 * natscl + gama * (1.0 - natscl * natscl);
            c[1] = -1.0 + natscl * natscl - dtby4 + 2.0 * gama * natscl;
            c[2] = -(2.0 * natscl + gama);
            break;
        default: break;
    }
}

// asymptotic_guess (src/spring.cpp:90-97)
__device__ inline double asymptotic_guess(int type, double dtby4, double gama) {
    switch (type) {
        case BDCU_SPRING_FENE: return 1.0 - dtby4 / 2.0 / gama;
        case BDCU_SPRING_ILC: return 1.0 - dtby4 / 3.0 / gama;
        case BDCU_SPRING_WLC: return 1.0 - sqrt(dtby4 / 6.0 / gama);
        default: return gama / (1.0 + dtby4);
    }
}

// value_and_deriv of solve_wlc_bounded (src/spring.cpp:107-116)
__device__ inline void wlcb_funcd(double x, double dt, double s, double gama, double& fval, double& fderiv) {
    fval = 6.0 * x / dt + 0.25 * (1.0 - s) * (1.0 - s) / ((1.0 - x) * (1.0 - x)) -
           0.25 + (x - s) / (1.0 - s) -
           s / 4.0 * (1.0 - s) * (1.0 - s) / ((1.0 + x - 2.0 * s) * (1.0 + x - 2.0 * s)) +
           s / 4.0 + s * (x - s) / (1.0 - s) - 6.0 * gama / dt;
    fderiv = 6.0 / dt + 1.0 / (1.0 - s) + s / (1.0 - s) +
             (1.0 - s) * (1.0 - s) / (2.0 * pow(1.0 - x, 3.0)) +
             ((1.0 - s) * (1.0 - s) * s) / (2.0 * pow(1.0 - 2.0 * s + x, 3.0));
}

// rtsafe (src/numerics.hpp:25-73) on the WLC-bounded equation. The reference
// aborts on a missing bracket or MAXIT; here that sets BDCU_ST_RTSAFE_FAIL.
// The iteration cap (10000) bounds the loop.
__device__ inline int rtsafe_wlcb(double dt, double s, double gama, double x1, double x2, double xacc,
                                  double& root) {
    double fl, fh, df;
    wlcb_funcd(x1, dt, s, gama, fl, df);
    wlcb_funcd(x2, dt, s, gama, fh, df);
    if ((fl > 0.0 && fh > 0.0) || (fl < 0.0 && fh < 0.0)) {
        root = 0.5 * (x1 + x2);
        return BDCU_ST_RTSAFE_FAIL;
    }
    if (fl == 0.0) { root = x1; return 0; }
    if (fh == 0.0) { root = x2; return 0; }
    double xl, xh;
    if (fl < 0.0) { xl = x1; xh = x2; } else { xh = x1; xl = x2; }
    double rts = 0.5 * (x1 + x2);
    double dxold = fabs(x2 - x1);
    double dx = dxold;
    double f;
    wlcb_funcd(rts, dt, s, gama, f, df);
    for (int j = 0; j < 10000; ++j) {
        if (((rts - xh) * df - f) * ((rts - xl) * df - f) >= 0.0 || fabs(2.0 * f) > fabs(dxold * df)) {
            dxold = dx;
            dx = 0.5 * (xh - xl);
            rts = xl + dx;
            if (xl == rts) { root = rts; return 0; }
        } else {
            dxold = dx;
            dx = f / df;
            const double temp = rts;
            rts -= dx;
            if (temp == rts) { root = rts; return 0; }
        }
        if (fabs(dx) < xacc) { root = rts; return 0; }
        wlcb_funcd(rts, dt, s, gama, f, df);
        if (f < 0.0) xl = rts; else xh = rts;
    }
    root = rts;
    return BDCU_ST_RTSAFE_FAIL;
}

// solve_implicit_r(...).length (src/spring.cpp:123-172) -- the force factor
// it also returns is unused by solve_connector and not computed here.
__device__ inline double implicit_length(int type, double dtby4, double gama, double natscl, int& st) {
    switch (type) {
        case BDCU_SPRING_HOOK: return gama / (1.0 + dtby4);
        case BDCU_SPRING_FRAENKEL: return (gama + dtby4 * natscl) / (1.0 + dtby4);
        case BDCU_SPRING_WLC_BOUNDED: {
            // solve_wlc_bounded (src/spring.cpp:101-119)
            if (natscl > 1.0) {
                st |= BDCU_ST_BAD_PARAM;
                return 0.0;
            }
            const double dt = dtby4 * 4.0;
            const double eps = 2.220446049250313e-16;
            double r;
            st |= rtsafe_wlcb(dt, natscl, gama, dmax_(0.0, 2.0 * natscl - 1.0 + eps), 1.0 - eps, 1e-15, r);
            return r;
        }
        default: break;
    }
    double c[4];
    cubic_coefficients(type, dtby4, gama, natscl, c);
    double r;
    if (type == BDCU_SPRING_FENE_FRAENKEL) {
        const double lo = dmax_(natscl - 1.0, 0.0), hi = natscl + 1.0;
        r = find_roots_cubic(c, lo, hi);
        r = polish_root(c, r, 1e-14);
        const double margin = 1e-6;
        r = dmin_(dmax_(r, lo + margin), hi - margin);
    } else {
        r = (gama < 1.0) ? gama / (1.0 + dtby4) : asymptotic_guess(type, dtby4, gama);
        if (!(type == BDCU_SPRING_WLC && gama > 100.0)) r = polish_root(c, r, 1e-14);
        const double margin = 1e-6;
        r = dmin_(dmax_(r, 0.0), 1.0 - margin);
    }
    return r;
}

// solve_connector (src/spring.cpp:174-181): new bond from its RHS Gamma.
__device__ inline void solve_connector(const double g[3], double dt, const DevChain& c, double out[3], int& st) {
    const double gmag = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    double r = implicit_length(c.spring_type, dt / 4.0, gmag / c.sqrtb, c.q0, st);
    if (fabs(r - 1.0) < 1e-6) r = 1.0 - 1e-6;
    const double s = r * c.sqrtb / gmag;
    out[0] = s * g[0];
    out[1] = s * g[1];
    out[2] = s * g[2];
}

// Connector force factor at a bond of length len (src/spring.cpp:183-193).
__device__ __forceinline__ double connector_factor(const DevChain& c, double len) {
    double r = len / c.sqrtb;
    if (fabs(r - 1.0) < kMyEps) r = 1.0 - kMyEps;
    return force_factor(c.spring_type, r, c.q0);
}

// clamped_length (src/config.cpp:8-13)
__device__ __forceinline__ double clamped_len(double b0, double b1, double b2) {
    double sq = b0 * b0 + b1 * b1 + b2 * b2;
    if (sq < 1.0e-12) sq = 1.0e-12;
    return sqrt(sq);
}

// gauss_factor / lj_factor / sdk_factor (src/excluded_volume.cpp:36-58)
__device__ inline double ev_factor(const DevChain& c, double r, double phi_pair) {
    switch (c.ev_type) {
        case BDCU_EV_GAUSS: return c.zsbyds5 * exp(-r * r * c.pt5bydssq);
        case BDCU_EV_LJ: {
            const double Rcut = c.equil ? c.Rcutg : c.Rcutp;
            if (r <= Rcut && r >= c.Rmin) return c.LJa / pow(r, 14.0) - c.LJb / pow(r, 8.0);
            if (r < c.Rmin) return c.lj_rmin_fac;
            return 0.0;
        }
        case BDCU_EV_SDK: {
            double fac = 0.0;
            if (r <= c.Rcutg && r >= c.Rmin)
                fac = c.SDKa / pow(r, 14.0) - c.SDKb / pow(r, 8.0);
            else if (r < c.Rmin)
                fac = c.sdk_rmin_fac;
            if (!c.equil && r <= c.RcutpSDK && r > c.Rcutg)
                fac += 1.530633312 * phi_pair * sin(1.530633312 * r * r + 1.213115524);
            return fac;
        }
        default: return 0.0;
    }
}

// Flow::kappa (src/flow.cpp:5-26)
__device__ inline void kappa_at(const DevChain& c, const double* arena, double t, double K[9]) {
    const int n = c.flow_n;
    if (n == 0) {
        for (int k = 0; k < 9; ++k) K[k] = c.K0[k];
        return;
    }
    const double* times = arena + c.flow_off;
    const double* Ks = times + n;
    if (n == 1 || t <= times[0]) {
        for (int k = 0; k < 9; ++k) K[k] = Ks[k];
        return;
    }
    if (t >= times[n - 1]) {
        for (int k = 0; k < 9; ++k) K[k] = Ks[9 * (n - 1) + k];
        return;
    }
    int i = 0;
    while (i < n - 1 && !(t >= times[i] && t < times[i + 1])) ++i;
    const double x0 = times[i], x1 = times[i + 1];
    const double w = (t - x0) / (x1 - x0);
    for (int k = 0; k < 9; ++k) K[k] = Ks[9 * i + k] + w * (Ks[9 * (i + 1) + k] - Ks[9 * i + k]);
}

// ExternalForce::force restricted to bead b (src/external_force.cpp:8-18,44-53):
// entries accumulate in list order.
__device__ inline void external_on_bead(const DevChain& c, const double* arena, int b, double t, double f[3]) {
    f[0] = f[1] = f[2] = 0.0;
    const double* e = arena + c.ext_off;
    const int N = c.N;
    for (int k = 0; k < c.ext_n; ++k) {
        const int bead = (int)e[0];
        const int n = (int)e[5];
        const int i = bead < 0 ? N + bead : bead;
        if (i == b) {
            double v0, v1, v2;
            const double* times = e + 6;
            const double* vals = e + 6 + n;
            if (e[1] != 0.0) {
                v0 = e[2]; v1 = e[3]; v2 = e[4];
            } else if (n == 0) {
                v0 = v1 = v2 = 0.0;
            } else if (n == 1 || t <= times[0]) {
                v0 = vals[0]; v1 = vals[1]; v2 = vals[2];
            } else if (t >= times[n - 1]) {
                v0 = vals[3 * (n - 1)]; v1 = vals[3 * (n - 1) + 1]; v2 = vals[3 * (n - 1) + 2];
            } else {
                int j = 0;
                while (j < n - 1 && !(t >= times[j] && t < times[j + 1])) ++j;
                const double w = (t - times[j]) / (times[j + 1] - times[j]);
                v0 = vals[3 * j] + w * (vals[3 * (j + 1)] - vals[3 * j]);
                v1 = vals[3 * j + 1] + w * (vals[3 * (j + 1) + 1] - vals[3 * j + 1]);
                v2 = vals[3 * j + 2] + w * (vals[3 * (j + 1) + 2] - vals[3 * j + 2]);
            }
            f[0] = f[0] + v0;
            f[1] = f[1] + v1;
            f[2] = f[2] + v2;
        }
        e += 6 + 4 * n;
    }
}

// Bending force on bead m (src/bending.cpp:5-43), from unit bonds u (N-1 x 3),
// bond cosines cs (N-2) and clamped lengths len (N-1).
__device__ inline void bending_on_bead(const DevChain& c, int m, const double* u, const double* cs,
                                       const double* len, double f[3]) {
    const int N = c.N;
    f[0] = f[1] = f[2] = 0.0;
    if (c.bend_type == BDCU_BEND_NONE || N == 2) return;
    const double C = c.C;
#define U_(i, d) u[3 * (i) + (d)]
    if (m == 0) {
        for (int d = 0; d < 3; ++d) f[d] = (C / len[0]) * (cs[0] * U_(0, d) - U_(1, d));
        return;
    }
    if (m == N - 1) {
        for (int d = 0; d < 3; ++d) f[d] = (C / len[N - 2]) * ((-cs[N - 3]) * U_(N - 2, d) + U_(N - 3, d));
        return;
    }
    if (N == 3) {  // m == 1
        for (int d = 0; d < 3; ++d)
            f[d] = C * ((1.0 / len[1]) * (cs[0] * U_(1, d) - U_(0, d)) +
                        (1.0 / len[0]) * ((-cs[0]) * U_(0, d) + U_(1, d)));
        return;
    }
    if (m == 1) {
        for (int d = 0; d < 3; ++d)
            f[d] = C * ((1.0 / len[1]) * (cs[0] * U_(1, d) - U_(0, d)) +
                        (1.0 / len[0]) * ((-cs[0]) * U_(0, d) + U_(1, d)) +
                        (1.0 / len[1]) * (cs[1] * U_(1, d) - U_(2, d)));
        return;
    }
    if (m == N - 2) {
        for (int d = 0; d < 3; ++d)
            f[d] = C * ((1.0 / len[N - 2]) * (cs[N - 3] * U_(N - 2, d) - U_(N - 3, d)) +
                        (1.0 / len[N - 3]) * ((-cs[N - 3]) * U_(N - 3, d) + U_(N - 2, d)) +
                        (1.0 / len[N - 3]) * ((-cs[N - 4]) * U_(N - 3, d) + U_(N - 4, d)));
        return;
    }
    for (int d = 0; d < 3; ++d)
        f[d] = C * ((1.0 / len[m]) * (cs[m - 1] * U_(m, d) - U_(m - 1, d)) +
                    (1.0 / len[m - 1]) * ((-cs[m - 1]) * U_(m - 1, d) + U_(m, d)) +
                    (1.0 / len[m - 1]) * ((-cs[m - 2]) * U_(m - 1, d) + U_(m - 2, d)) +
                    (1.0 / len[m]) * (cs[m] * U_(m, d) - U_(m + 1, d)));
#undef U_
}

// RPY pair weights (src/hydrodynamics.cpp:36-43): omega1 (isotropic) and
// omega2 (dyadic) for bead separation b with |b|^2 = sq (unclamped).
__device__ __forceinline__ void rpy_weights(double hstar, double sq, double& om1, double& om2) {
    const double RPI = sqrt(kPi), TRPI = 2.0 * RPI, TPI = 2.0 * kPi;
    const double C1 = TPI / 3.0, C3 = 0.75 / RPI * 0.375, C7 = 0.09375 / RPI;
    const double RPI3by4 = RPI * 0.75;
    if (sq < 1.0e-12) sq = 1.0e-12;
    const double rs = sqrt(sq);
    const double hsbyrs = hstar / rs, rsbyhs = rs / hstar;
    const double hsbyrs2 = hsbyrs * hsbyrs;
    if (rsbyhs >= TRPI) {
        om1 = RPI3by4 * hsbyrs * (1.0 + C1 * hsbyrs2);
        om2 = RPI3by4 * (hsbyrs / (rs * rs)) * (1.0 - TPI * hsbyrs2);
    } else {
        om1 = 1.0 - C3 * rsbyhs;
        om2 = C7 * rsbyhs / (rs * rs);
    }
}

}  // namespace bdcu
