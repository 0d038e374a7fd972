/*
 * bd_oracle.c -- CPU restatement of bdsim's ChainIntegrator step.
 *
 * TEST INFRASTRUCTURE ONLY (see bd_oracle.h). Written as plain C over flat
 * row-major arrays. Every expression keeps the reference's operand order and
 * grouping so that, compiled without FMA contraction (-ffp-contract=off, as
 * the reference's default x86-64 Release build has no FMA), it reproduces the
 * reference bit for bit up to libm.
 *
 * File:line citations are relative to the bdsim project root.
 */
#include "bd_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define PI_D 3.14159265358979323846 /* src/types.hpp:22 */
#define MYEPS_D 1e-6                /* src/types.hpp:24 */
#define MAXCHEB_I 500               /* src/types.hpp:20 */
#define LANCZOS_COLD_I 30           /* src/hydrodynamics.cpp:79 */
#define LANCZOS_WARM_I 8            /* src/hydrodynamics.cpp:80 */

/* std::min / std::max semantics, NaN behaviour included. */
static double mind(double a, double b) { return (b < a) ? b : a; }
static double maxd(double a, double b) { return (a < b) ? b : a; }
static int mini(int a, int b) { return (b < a) ? b : a; }
static int maxi(int a, int b) { return (a < b) ? b : a; }

/* ------------------------------------------------------------------ RNG */

/* am = nextafterf(1,-1)/float(IM) in single precision (src/rng.cpp:24-28). */
static float rng_scale(void) { return nextafterf(1.0f, -1.0f) / (float)2147483647; }

/* Rng::maybe_init + Rng::ran_1 (src/rng.cpp:31-70). */
void bdo_ran1(int32_t st[3], int n, double* out) {
    int32_t ix = st[0], iy = st[1], seed = st[2];
    if (seed <= 0 || iy < 0) {
        const int32_t s = seed < 0 ? -seed : seed;
        iy = (888889999 ^ s) | 1;
        ix = 777755555 ^ s;
        seed = s + 1;
    }
    const float am = rng_scale();
    uint32_t ux = (uint32_t)ix;
    for (int c = 0; c < n; ++c) {
        ux ^= (ux << 13);
        ux ^= (ux >> 17);
        ux ^= (ux << 5);
        const int32_t k = iy / 127773;
        iy = 16807 * (iy - k * 127773) - 2836 * k;
        if (iy < 0) iy += 2147483647;
        const uint32_t mixed = ux ^ (uint32_t)iy;
        const int32_t res = (int32_t)((mixed & 0x7fffffffu) | 1u);
        out[c] = (double)(am * (float)res);
    }
    st[0] = (int32_t)ux;
    st[1] = iy;
    st[2] = seed;
}

/* raw_noise: Ottinger deviate per draw, 3 draws per bead (src/mobility.cpp:18-29). */
static void raw_noise(int32_t rng[3], int N, double* x) {
    const double c1 = 14.14855378, c2 = 1.21569221;
    double u[3];
    for (int mu = 0; mu < N; ++mu) {
        bdo_ran1(rng, 3, u);
        for (int d = 0; d < 3; ++d) {
            const double y = u[d] - 0.5;
            x[3 * mu + d] = (c1 * y * y + c2) * y;
        }
    }
}

/* ------------------------------------------------------------- geometry */

static double norm2_3(const double* a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }

/* clamped_length (src/config.cpp:8-13) */
static double clamped_len(const double* b) {
    double sq = norm2_3(b);
    if (sq < 1.0e-12) sq = 1.0e-12;
    return sqrt(sq);
}

/* chain_geometry (src/config.cpp:15-25): bonds (N-1 x 3) and lengths. */
static void geometry(const double* R, int N, double* bond, double* len) {
    for (int i = 0; i < N - 1; ++i) {
        for (int d = 0; d < 3; ++d) bond[3 * i + d] = R[3 * (i + 1) + d] - R[3 * i + d];
        len[i] = clamped_len(bond + 3 * i);
    }
}

void bdo_unit_bonds_and_cosines(const double* R, int N, double* unit, double* cosines) {
    double* bond = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    double* len = (double*)malloc(sizeof(double) * (size_t)N);
    geometry(R, N, bond, len);
    /* unit_bonds (src/config.cpp:35-39), bond_cosines (:41-45) */
    for (int i = 0; i < N - 1; ++i)
        for (int d = 0; d < 3; ++d) unit[3 * i + d] = (1.0 / len[i]) * bond[3 * i + d];
    for (int i = 0; i + 1 < N - 1; ++i) cosines[i] = unit[3 * (i + 1)] * unit[3 * i] + unit[3 * (i + 1) + 1] * unit[3 * i + 1] + unit[3 * (i + 1) + 2] * unit[3 * i + 2];
    free(bond);
    free(len);
}

/* --------------------------------------------------------------- springs */

/* force_sans_hookean (src/spring.cpp:14-37) */
static double force_factor(int type, double q, double q0) {
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

/* bisect_cubic (src/numerics.cpp:8-23) */
static double cubic_eval(const double c[4], double x) { return ((c[3] * x + c[2]) * x + c[1]) * x + c[0]; }
static double bisect_cubic(const double c[4], double lo, double hi) {
    double flo = cubic_eval(c, lo), fhi = cubic_eval(c, hi);
    if (flo == 0.0) return lo;
    if (fhi == 0.0) return hi;
    if (flo * fhi > 0.0) return (fabs(flo) < fabs(fhi)) ? lo : hi;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        const double fm = cubic_eval(c, mid);
        if (fm == 0.0 || (hi - lo) < 1e-15) return mid;
        if (flo * fm < 0.0) {
            hi = mid;
            fhi = fm;
        } else {
            lo = mid;
            flo = fm;
        }
    }
    (void)fhi;
    return 0.5 * (lo + hi);
}

/* find_roots_cubic (src/numerics.cpp:25-59) */
static double find_roots_cubic(const double c4[4], double lower, double upper) {
    const double a = c4[2] / c4[3];
    const double b = c4[1] / c4[3];
    const double c = c4[0] / c4[3];
    const double Q = (a * a - 3.0 * b) / 9.0;
    const double R = (2.0 * a * a * a - 9.0 * a * b + 27.0 * c) / 54.0;
    double x;
    if (R * R < Q * Q * Q) {
        const double theta = acos(R / sqrt(Q * Q * Q));
        for (int i = -1; i <= 1; ++i) {
            x = -2.0 * sqrt(Q) * cos((theta + (double)i * PI_D * 2.0) / 3.0) - a / 3.0;
            if (x >= lower && x <= upper) return x;
        }
        x = -2.0 * sqrt(Q) * cos((theta + PI_D * 2.0) / 3.0) - a / 3.0;
    } else {
        const double Au = -copysign(1.0, R) * cbrt(fabs(R) + sqrt(R * R - Q * Q * Q));
        const double Bu = (Au == 0.0) ? 0.0 : Q / Au;
        x = (Au + Bu) - a / 3.0;
    }
    if (x >= lower && x <= upper) return x;
    return bisect_cubic(c4, lower, upper);
}

/* polish_poly_root (src/numerics.cpp:61-85) */
static double polish_root(const double c[4], double x0, double atol) {
    double x = x0;
    for (int iter = 0; iter < 30; ++iter) {
        double p = c[3] * x + c[2];
        double p1 = c[3];
        for (int i = 1; i >= 0; --i) {
            p1 = p + p1 * x;
            p = c[i] + p * x;
        }
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

/* cubic_coefficients (src/spring.cpp:55-87) */
static void cubic_coefficients(int type, double dtby4, double gama, double natscl, double c[4]) {
    c[0] = c[1] = c[2] = 0.0;
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

/* asymptotic_guess (src/spring.cpp:90-97) */
static double asymptotic_guess(int type, double dtby4, double gama) {
    switch (type) {
        case BDCU_SPRING_FENE: return 1.0 - dtby4 / 2.0 / gama;
        case BDCU_SPRING_ILC: return 1.0 - dtby4 / 3.0 / gama;
        case BDCU_SPRING_WLC: return 1.0 - sqrt(dtby4 / 6.0 / gama);
        default: return gama / (1.0 + dtby4);
    }
}

/* value_and_deriv of solve_wlc_bounded (src/spring.cpp:107-116) */
static void wlcb_funcd(double x, double dt, double s, double gama, double* fval, double* fderiv) {
    *fval = 6.0 * x / dt + 0.25 * (1.0 - s) * (1.0 - s) / ((1.0 - x) * (1.0 - x)) -
            0.25 + (x - s) / (1.0 - s) -
            s / 4.0 * (1.0 - s) * (1.0 - s) / ((1.0 + x - 2.0 * s) * (1.0 + x - 2.0 * s)) +
            s / 4.0 + s * (x - s) / (1.0 - s) - 6.0 * gama / dt;
    *fderiv = 6.0 / dt + 1.0 / (1.0 - s) + s / (1.0 - s) +
              (1.0 - s) * (1.0 - s) / (2.0 * pow(1.0 - x, 3.0)) +
              ((1.0 - s) * (1.0 - s) * s) / (2.0 * pow(1.0 - 2.0 * s + x, 3.0));
}

/* rtsafe (src/numerics.hpp:25-73). The reference aborts on a missing bracket
   or on MAXIT; here that is reported as BDCU_ST_RTSAFE_FAIL. */
static int rtsafe_wlcb(double dt, double s, double gama, double x1, double x2, double xacc, double* root) {
    double fl, fh, df;
    wlcb_funcd(x1, dt, s, gama, &fl, &df);
    wlcb_funcd(x2, dt, s, gama, &fh, &df);
    if ((fl > 0.0 && fh > 0.0) || (fl < 0.0 && fh < 0.0)) {
        *root = 0.5 * (x1 + x2);
        return BDCU_ST_RTSAFE_FAIL;
    }
    if (fl == 0.0) { *root = x1; return 0; }
    if (fh == 0.0) { *root = x2; return 0; }
    double xl, xh;
    if (fl < 0.0) { xl = x1; xh = x2; } else { xh = x1; xl = x2; }
    double rts = 0.5 * (x1 + x2);
    double dxold = fabs(x2 - x1);
    double dx = dxold;
    double f;
    wlcb_funcd(rts, dt, s, gama, &f, &df);
    for (int j = 0; j < 10000; ++j) {
        if (((rts - xh) * df - f) * ((rts - xl) * df - f) >= 0.0 || fabs(2.0 * f) > fabs(dxold * df)) {
            dxold = dx;
            dx = 0.5 * (xh - xl);
            rts = xl + dx;
            if (xl == rts) { *root = rts; return 0; }
        } else {
            dxold = dx;
            dx = f / df;
            const double temp = rts;
            rts -= dx;
            if (temp == rts) { *root = rts; return 0; }
        }
        if (fabs(dx) < xacc) { *root = rts; return 0; }
        wlcb_funcd(rts, dt, s, gama, &f, &df);
        if (f < 0.0) xl = rts; else xh = rts;
    }
    *root = rts;
    return BDCU_ST_RTSAFE_FAIL;
}

/* solve_wlc_bounded (src/spring.cpp:101-119) */
static int solve_wlc_bounded(double dtby4, double gama, double sigma, double* r) {
    if (sigma > 1.0) { *r = 0.0; return BDCU_ST_BAD_PARAM; }
    const double dt = dtby4 * 4.0;
    const double eps = 2.220446049250313e-16; /* numeric_limits<double>::epsilon */
    return rtsafe_wlcb(dt, sigma, gama, maxd(0.0, 2.0 * sigma - 1.0 + eps), 1.0 - eps, 1e-15, r);
}

/* solve_implicit_r (src/spring.cpp:174-223) */
int bdo_solve_implicit_r(int type, double dtby4, double gama, double natscl, double* length, double* ff) {
    int st = 0;
    double r;
    switch (type) {
        case BDCU_SPRING_HOOK:
            *length = gama / (1.0 + dtby4);
            *ff = 1.0;
            return 0;
        case BDCU_SPRING_FRAENKEL:
            r = (gama + dtby4 * natscl) / (1.0 + dtby4);
            *length = r;
            *ff = 1.0 - natscl / r;
            return 0;
        case BDCU_SPRING_WLC_BOUNDED:
            st = solve_wlc_bounded(dtby4, gama, natscl, &r);
            *length = r;
            *ff = force_factor(type, r, natscl);
            return st;
        default: break;
    }
    double c[4];
    cubic_coefficients(type, dtby4, gama, natscl, c);
    if (type == BDCU_SPRING_FENE_FRAENKEL) {
        const double lo = maxd(natscl - 1.0, 0.0), hi = natscl + 1.0;
        r = find_roots_cubic(c, lo, hi);
        r = polish_root(c, r, 1e-14);
        const double margin = 1e-6;
        r = mind(maxd(r, lo + margin), hi - margin);
    } else {
        r = (gama < 1.0) ? gama / (1.0 + dtby4) : asymptotic_guess(type, dtby4, gama);
        if (!(type == BDCU_SPRING_WLC && gama > 100.0)) r = polish_root(c, r, 1e-14);
        const double margin = 1e-6;
        r = mind(maxd(r, 0.0), 1.0 - margin);
    }
    *length = r;
    *ff = force_factor(type, r, natscl);
    return 0;
}

/* solve_connector (src/spring.cpp:225-232) */
int bdo_solve_connector(const double gamma[3], double dt, const bdcu_phys* p, double out[3]) {
    const double sqrtb = p->sqrtb;
    const double q0 = p->natural_length / sqrtb;
    const double gmag = sqrt(norm2_3(gamma));
    double r, ff;
    const int st = bdo_solve_implicit_r(p->spring_type, dt / 4.0, gmag / sqrtb, q0, &r, &ff);
    if (fabs(r - 1.0) < 1e-6) r = 1.0 - 1e-6;
    for (int d = 0; d < 3; ++d) out[d] = (r * sqrtb / gmag) * gamma[d];
    return st;
}

/* connector_forces (src/spring.cpp:183-193) from bonds/lengths. */
static void connector_forces(const double* bond, const double* len, int nb, const bdcu_phys* p, double* Fb) {
    const double sqrtb = p->sqrtb;
    const double q0 = p->natural_length / sqrtb;
    for (int i = 0; i < nb; ++i) {
        double r = len[i] / sqrtb;
        if (fabs(r - 1.0) < MYEPS_D) r = 1.0 - MYEPS_D;
        const double f = force_factor(p->spring_type, r, q0);
        for (int d = 0; d < 3; ++d) Fb[3 * i + d] = f * bond[3 * i + d];
    }
}

/* bead_forces_from_connectors (src/spring.cpp:195-203) */
static void bead_forces(const double* Fb, int N, double* F) {
    memset(F, 0, sizeof(double) * 3 * (size_t)N);
    if (N == 1) return;
    for (int d = 0; d < 3; ++d) F[d] = Fb[d];
    for (int nu = 1; nu < N - 1; ++nu)
        for (int d = 0; d < 3; ++d) F[3 * nu + d] = Fb[3 * nu + d] - Fb[3 * (nu - 1) + d];
    for (int d = 0; d < 3; ++d) F[3 * (N - 1) + d] = (-1.0) * Fb[3 * (N - 2) + d];
}

void bdo_spring_force(const double* R, int N, const bdcu_phys* p, double* F) {
    double* bond = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    double* len = (double*)malloc(sizeof(double) * (size_t)N);
    double* Fb = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    geometry(R, N, bond, len);
    connector_forces(bond, len, N - 1, p, Fb);
    bead_forces(Fb, N, F);
    free(bond);
    free(len);
    free(Fb);
}

/* ------------------------------------------------------------- bending */

/* BendingForce::force (src/bending.cpp:5-43) from bonds/lengths. */
static void bending_from_geom(const double* bond, const double* len, int N, const bdcu_phys* p, double* F) {
    memset(F, 0, sizeof(double) * 3 * (size_t)N);
    if (p->bend_type == BDCU_BEND_NONE) return;
    if (N == 2) return;
    const double C = p->bend_stiffness;
    double* u = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    double* cs = (double*)malloc(sizeof(double) * (size_t)N);
    for (int i = 0; i < N - 1; ++i)
        for (int d = 0; d < 3; ++d) u[3 * i + d] = (1.0 / len[i]) * bond[3 * i + d];
    for (int i = 0; i + 1 < N - 1; ++i)
        cs[i] = u[3 * (i + 1)] * u[3 * i] + u[3 * (i + 1) + 1] * u[3 * i + 1] + u[3 * (i + 1) + 2] * u[3 * i + 2];
#define U(i, d) u[3 * (i) + (d)]
    for (int d = 0; d < 3; ++d) {
        F[d] = (C / len[0]) * (cs[0] * U(0, d) - U(1, d));
        F[3 * (N - 1) + d] = (C / len[N - 2]) * ((-cs[N - 3]) * U(N - 2, d) + U(N - 3, d));
    }
    if (N == 3) {
        for (int d = 0; d < 3; ++d)
            F[3 + d] = C * ((1.0 / len[1]) * (cs[0] * U(1, d) - U(0, d)) +
                            (1.0 / len[0]) * ((-cs[0]) * U(0, d) + U(1, d)));
    } else {
        for (int d = 0; d < 3; ++d) {
            F[3 + d] = C * ((1.0 / len[1]) * (cs[0] * U(1, d) - U(0, d)) +
                            (1.0 / len[0]) * ((-cs[0]) * U(0, d) + U(1, d)) +
                            (1.0 / len[1]) * (cs[1] * U(1, d) - U(2, d)));
            F[3 * (N - 2) + d] = C * ((1.0 / len[N - 2]) * (cs[N - 3] * U(N - 2, d) - U(N - 3, d)) +
                                      (1.0 / len[N - 3]) * ((-cs[N - 3]) * U(N - 3, d) + U(N - 2, d)) +
                                      (1.0 / len[N - 3]) * ((-cs[N - 4]) * U(N - 3, d) + U(N - 4, d)));
        }
        for (int m = 2; m <= N - 3; ++m)
            for (int d = 0; d < 3; ++d)
                F[3 * m + d] = C * ((1.0 / len[m]) * (cs[m - 1] * U(m, d) - U(m - 1, d)) +
                                    (1.0 / len[m - 1]) * ((-cs[m - 1]) * U(m - 1, d) + U(m, d)) +
                                    (1.0 / len[m - 1]) * ((-cs[m - 2]) * U(m - 1, d) + U(m - 2, d)) +
                                    (1.0 / len[m]) * (cs[m] * U(m, d) - U(m + 1, d)));
    }
#undef U
    free(u);
    free(cs);
}

void bdo_bending_force(const double* R, int N, const bdcu_phys* p, double* F) {
    double* bond = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    double* len = (double*)malloc(sizeof(double) * (size_t)N);
    geometry(R, N, bond, len);
    bending_from_geom(bond, len, N, p, F);
    free(bond);
    free(len);
}

/* ----------------------------------------------------- excluded volume */

/* Constants of the ExcludedVolume constructor (src/excluded_volume.cpp:14-34). */
typedef struct {
    double zsbyds5, pt5bydssq, LJa, LJb, SDKa, SDKb, Rmin, Rcutp, RcutpSDK, Rcutg;
} ev_consts;

static void ev_make(const bdcu_phys* p, ev_consts* e) {
    const double z = p->zstar, d = p->dstar;
    e->zsbyds5 = z / pow(d, 5.0);
    e->pt5bydssq = 0.5 / (d * d);
    e->LJa = 12.0 * 4.0 * z * pow(d, 12.0);
    e->LJb = 6.0 * 4.0 * z * pow(d, 6.0);
    e->SDKa = 12.0 * 4.0 * pow(d, 12.0);
    e->SDKb = 6.0 * 4.0 * pow(d, 6.0);
    e->Rmin = p->min_cutoff;
    e->Rcutp = p->max_cutoff;
    e->RcutpSDK = p->max_cutoff;
    e->Rcutg = d * pow(2.0, 1.0 / 6.0);
}

/* gauss_factor / lj_factor / sdk_factor (src/excluded_volume.cpp:36-58) */
static double ev_factor(int type, const ev_consts* e, int equil, double r, double phi_pair) {
    switch (type) {
        case BDCU_EV_GAUSS: return e->zsbyds5 * exp(-r * r * e->pt5bydssq);
        case BDCU_EV_LJ: {
            const double Rcut = equil ? e->Rcutg : e->Rcutp;
            if (r <= Rcut && r >= e->Rmin) return e->LJa / pow(r, 14.0) - e->LJb / pow(r, 8.0);
            if (r < e->Rmin) return e->LJa / pow(e->Rmin, 14.0) - e->LJb / pow(e->Rmin, 8.0);
            return 0.0;
        }
        case BDCU_EV_SDK: {
            double fac = 0.0;
            if (r <= e->Rcutg && r >= e->Rmin)
                fac = e->SDKa / pow(r, 14.0) - e->SDKb / pow(r, 8.0);
            else if (r < e->Rmin)
                fac = e->SDKa / pow(e->Rmin, 14.0) - e->SDKb / pow(e->Rmin, 8.0);
            if (!equil && r <= e->RcutpSDK && r > e->Rcutg)
                fac += 1.530633312 * phi_pair * sin(1.530633312 * r * r + 1.213115524);
            return fac;
        }
        default: return 0.0;
    }
}

/* ExcludedVolume::force (src/excluded_volume.cpp:60-89) */
void bdo_ev_force(const double* R, int N, const bdcu_phys* p, const double* arena, double* F) {
    memset(F, 0, sizeof(double) * 3 * (size_t)N);
    if (p->ev_type == BDCU_EV_NONE) return;
    ev_consts e;
    ev_make(p, &e);
    const double* phi = (p->ev_type == BDCU_EV_SDK && p->phi_offset >= 0) ? arena + p->phi_offset : NULL;
    for (int nu = 1; nu < N; ++nu) {
        for (int mu = 0; mu < nu; ++mu) {
            if ((nu - mu) < p->contour_dist_for_ev) continue;
            double q[3];
            for (int d = 0; d < 3; ++d) q[d] = R[3 * nu + d] - R[3 * mu + d];
            double sq = norm2_3(q);
            if (sq < 1.0e-12) sq = 1.0e-12;
            const double r = sqrt(sq);
            const double fac = ev_factor(p->ev_type, &e, p->equilibration, r, phi ? phi[mu * N + nu] : 0.0);
            for (int d = 0; d < 3; ++d) {
                const double f = (-fac) * q[d];
                F[3 * mu + d] = F[3 * mu + d] + f;
                F[3 * nu + d] = F[3 * nu + d] - f;
            }
        }
    }
}

/* ------------------------------------------------- external force, flow */

/* sample / ExternalForce::force (src/external_force.cpp:8-18,44-53) */
void bdo_external_force(int N, const bdcu_phys* p, const double* arena, double t, double* F) {
    memset(F, 0, sizeof(double) * 3 * (size_t)N);
    const double* e = arena + p->ext_offset;
    for (int k = 0; k < p->ext_n_entries; ++k) {
        const int bead = (int)e[0];
        const int is_const = (int)e[1];
        const int n = (int)e[5];
        const double* times = e + 6;
        const double* vals = e + 6 + n;
        int i = bead < 0 ? N + bead : bead;
        if (!(i < 0 || i >= N)) {
            double v[3];
            if (is_const) {
                v[0] = e[2]; v[1] = e[3]; v[2] = e[4];
            } else if (n == 0) {
                v[0] = v[1] = v[2] = 0.0;
            } else if (n == 1 || t <= times[0]) {
                v[0] = vals[0]; v[1] = vals[1]; v[2] = vals[2];
            } else if (t >= times[n - 1]) {
                v[0] = vals[3 * (n - 1)]; v[1] = vals[3 * (n - 1) + 1]; v[2] = vals[3 * (n - 1) + 2];
            } else {
                int j = 0;
                while (j < n - 1 && !(t >= times[j] && t < times[j + 1])) ++j;
                const double w = (t - times[j]) / (times[j + 1] - times[j]);
                for (int d = 0; d < 3; ++d) v[d] = vals[3 * j + d] + w * (vals[3 * (j + 1) + d] - vals[3 * j + d]);
            }
            for (int d = 0; d < 3; ++d) F[3 * i + d] = F[3 * i + d] + v[d];
        }
        e += 6 + 4 * n;
    }
}

/* Flow::kappa (src/flow.cpp:5-26) */
void bdo_kappa(const bdcu_phys* p, const double* arena, double t, double K[9]) {
    const int n = p->flow_n_times;
    if (n == 0) {
        memcpy(K, p->flow_kappa, sizeof(double) * 9);
        return;
    }
    const double* times = arena + p->flow_offset;
    const double* Ks = times + n;
    if (n == 1 || t <= times[0]) { memcpy(K, Ks, sizeof(double) * 9); return; }
    if (t >= times[n - 1]) { memcpy(K, Ks + 9 * (n - 1), sizeof(double) * 9); return; }
    int i = 0;
    while (i < n - 1 && !(t >= times[i] && t < times[i + 1])) ++i;
    const double x0 = times[i], x1 = times[i + 1];
    const double w = (t - x0) / (x1 - x0);
    for (int k = 0; k < 9; ++k) K[k] = Ks[9 * i + k] + w * (Ks[9 * (i + 1) + k] - Ks[9 * i + k]);
}

/* flow_velocity (src/integrator.cpp:53-58): out = K . R per bead. */
static void flow_velocity(const double K[9], const double* R, int N, double* out) {
    for (int i = 0; i < N; ++i) {
        const double* v = R + 3 * i;
        for (int r = 0; r < 3; ++r) out[3 * i + r] = K[3 * r] * v[0] + K[3 * r + 1] * v[1] + K[3 * r + 2] * v[2];
    }
}

void bdo_total_force(const double* R, int N, const bdcu_phys* p, const double* arena, double* F) {
    double* Fe = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    double* Fb = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    bdo_spring_force(R, N, p, F);
    bdo_ev_force(R, N, p, arena, Fe);
    bdo_bending_force(R, N, p, Fb);
    /* non_spring_force = ev + bending (src/model.hpp:56-58), then F + Fe */
    for (int i = 0; i < 3 * N; ++i) F[i] = F[i] + (Fe[i] + Fb[i]);
    free(Fe);
    free(Fb);
}

/* ---------------------------------------------------------------- RPY */

void bdo_rpy_matrix(const double* R, int N, double hstar, double* D) {
    const int n = 3 * N;
    memset(D, 0, sizeof(double) * (size_t)n * (size_t)n);
    for (int i = 0; i < n; ++i) D[(size_t)i * n + i] = 1.0;
    if (hstar <= 0.0) return;
    const double RPI = sqrt(PI_D), TRPI = 2.0 * RPI, TPI = 2.0 * PI_D;
    const double C1 = TPI / 3.0, C3 = 0.75 / RPI * 0.375, C7 = 0.09375 / RPI;
    const double RPI3by4 = RPI * 0.75;
    for (int nu = 1; nu < N; ++nu) {
        for (int mu = 0; mu < nu; ++mu) {
            double b[3];
            for (int d = 0; d < 3; ++d) b[d] = R[3 * nu + d] - R[3 * mu + d];
            double sq = norm2_3(b);
            if (sq < 1.0e-12) sq = 1.0e-12;
            const double rs = sqrt(sq);
            const double hsbyrs = hstar / rs, rsbyhs = rs / hstar;
            const double hsbyrs2 = hsbyrs * hsbyrs;
            double om1, om2;
            if (rsbyhs >= TRPI) {
                om1 = RPI3by4 * hsbyrs * (1.0 + C1 * hsbyrs2);
                om2 = RPI3by4 * (hsbyrs / (rs * rs)) * (1.0 - TPI * hsbyrs2);
            } else {
                om1 = 1.0 - C3 * rsbyhs;
                om2 = C7 * rsbyhs / (rs * rs);
            }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double val = om2 * b[i] * b[j] + (i == j ? om1 : 0.0);
                    D[(size_t)(3 * mu + i) * n + 3 * nu + j] = val;
                    D[(size_t)(3 * nu + j) * n + 3 * mu + i] = val;
                }
        }
    }
}

/* matvec, hand-rolled backend (src/linalg.cpp:79-89) */
static void matvec(const double* M, int n, const double* x, double* y) {
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += M[(size_t)i * n + j] * x[j];
        y[i] = s;
    }
}

/* cholesky_lower (src/linalg.cpp:91-107) */
int bdo_cholesky(const double* M, int n, double* L) {
    memset(L, 0, sizeof(double) * (size_t)n * (size_t)n);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j <= i; ++j) {
            double sum = M[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) sum -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
            if (i == j) {
                if (!(sum > 0.0)) return BDCU_ST_NOT_PD;
                L[(size_t)i * n + j] = sqrt(sum);
            } else {
                L[(size_t)i * n + j] = sum / L[(size_t)j * n + j];
            }
        }
    }
    return 0;
}

/* lower_matvec (src/linalg.cpp:109-117) */
static void lower_matvec(const double* L, int n, const double* x, double* y) {
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 0; j <= i; ++j) s += L[(size_t)i * n + j] * x[j];
        y[i] = s;
    }
}

static double dotv(const double* a, const double* b, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* -------------------------------------------------------- Lanczos bounds */

/* default_seed (src/hydrodynamics.cpp:83-87) */
static void default_seed(int n, double* v) {
    for (int i = 0; i < n; ++i) v[i] = sin(0.7654321 * (i + 1)) + 0.5;
}

/* sturm_count (src/hydrodynamics.cpp:91-104) */
static int sturm_count(const double* a, const double* b, int m, double x) {
    int count = 0;
    double d = a[0] - x;
    if (d < 0.0) ++count;
    for (int i = 1; i < m; ++i) {
        if (d == 0.0) d = 1.0e-300;
        d = (a[i] - x) - b[i - 1] * b[i - 1] / d;
        if (d < 0.0) ++count;
    }
    return count;
}

/* tridiag_eigenvector (src/hydrodynamics.cpp:106-136) */
static void tridiag_eigenvector(const double* a, const double* b, int m, double lambda, double* y) {
    const double scale = maxd(fabs(lambda), 1.0);
    const double shift = lambda - 1.0e-7 * scale;
    double c[LANCZOS_COLD_I], d[LANCZOS_COLD_I];
    for (int i = 0; i < m; ++i) y[i] = 1.0 / sqrt((double)m);
    for (int it = 0; it < 2; ++it) {
        double beta0 = a[0] - shift;
        if (fabs(beta0) < 1.0e-300) beta0 = 1.0e-300;
        c[0] = (m > 1 ? b[0] / beta0 : 0.0);
        d[0] = y[0] / beta0;
        for (int i = 1; i < m; ++i) {
            double beta = (a[i] - shift) - b[i - 1] * c[i - 1];
            if (fabs(beta) < 1.0e-300) beta = 1.0e-300;
            c[i] = (i < m - 1 ? b[i] / beta : 0.0);
            d[i] = (y[i] - b[i - 1] * d[i - 1]) / beta;
        }
        y[m - 1] = d[m - 1];
        for (int i = m - 2; i >= 0; --i) y[i] = d[i] - c[i] * y[i + 1];
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += y[i] * y[i];
        nrm = sqrt(nrm);
        if (!(nrm > 0.0) || !isfinite(nrm)) {
            for (int i = 0; i < m; ++i) y[i] = 1.0 / sqrt((double)m);
            return;
        }
        for (int i = 0; i < m; ++i) y[i] /= nrm;
    }
}

typedef struct {
    double rmin, rmax;
    int steps;
} lanczos_out;

/* lanczos_extremes (src/hydrodynamics.cpp:146-221). seed == NULL => default.
   vmin/vmax: n outputs. V: scratch m*n. Counts D.x in *ndx. */
static lanczos_out lanczos_extremes(const double* D, int n, int m, const double* seed,
                                    double* vmin, double* vmax, double* V, long* ndx) {
    if (n < m) m = n;
    double* v = (double*)malloc(sizeof(double) * (size_t)n);
    double* w = (double*)malloc(sizeof(double) * (size_t)n);
    double* vprev = (double*)calloc((size_t)n, sizeof(double));
    double alpha[LANCZOS_COLD_I], beta[LANCZOS_COLD_I];
    if (seed) memcpy(v, seed, sizeof(double) * (size_t)n); else default_seed(n, v);
    {
        double nv = sqrt(dotv(v, v, n));
        if (!(nv > 0.0)) { default_seed(n, v); nv = sqrt(dotv(v, v, n)); }
        for (int i = 0; i < n; ++i) v[i] /= nv;
    }
    int k = 0, nbeta = 0;
    double b = 0.0;
    for (int j = 0; j < m; ++j) {
        memcpy(V + (size_t)j * n, v, sizeof(double) * (size_t)n);
        matvec(D, n, v, w);
        ++*ndx;
        const double a = dotv(v, w, n);
        alpha[k++] = a;
        for (int i = 0; i < n; ++i) w[i] -= a * v[i] + b * vprev[i];
        for (int u = 0; u <= j; ++u) {
            const double* uu = V + (size_t)u * n;
            const double dd = dotv(w, uu, n);
            for (int i = 0; i < n; ++i) w[i] -= dd * uu[i];
        }
        b = sqrt(dotv(w, w, n));
        if (b < 1.0e-10) break;
        memcpy(vprev, v, sizeof(double) * (size_t)n);
        for (int i = 0; i < n; ++i) v[i] = w[i] / b;
        beta[nbeta++] = b;
    }
    lanczos_out out;
    out.steps = k;
    if (k == 1) {
        out.rmin = out.rmax = alpha[0];
        memcpy(vmin, V, sizeof(double) * (size_t)n);
        memcpy(vmax, V, sizeof(double) * (size_t)n);
        free(v); free(w); free(vprev);
        return out;
    }
    const double* bb = beta; /* first k-1 entries */
    double lo = alpha[0], hi = alpha[0];
    for (int i = 0; i < k; ++i) {
        const double rad = (i > 0 ? fabs(bb[i - 1]) : 0.0) + (i < k - 1 ? fabs(bb[i]) : 0.0);
        lo = mind(lo, alpha[i] - rad);
        hi = maxd(hi, alpha[i] + rad);
    }
    double a1 = lo, b1 = hi;
    for (int it = 0; it < 100; ++it) {
        const double mid = 0.5 * (a1 + b1);
        if (sturm_count(alpha, bb, k, mid) >= 1) b1 = mid; else a1 = mid;
    }
    double a2 = lo, b2 = hi;
    for (int it = 0; it < 100; ++it) {
        const double mid = 0.5 * (a2 + b2);
        if (sturm_count(alpha, bb, k, mid) >= k) b2 = mid; else a2 = mid;
    }
    out.rmin = 0.5 * (a1 + b1);
    out.rmax = 0.5 * (a2 + b2);
    double ymin[LANCZOS_COLD_I], ymax[LANCZOS_COLD_I];
    tridiag_eigenvector(alpha, bb, k, out.rmin, ymin);
    tridiag_eigenvector(alpha, bb, k, out.rmax, ymax);
    for (int i = 0; i < n; ++i) { vmin[i] = 0.0; vmax[i] = 0.0; }
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < n; ++i) {
            vmin[i] += ymin[j] * V[(size_t)j * n + i];
            vmax[i] += ymax[j] * V[(size_t)j * n + i];
        }
    free(v); free(w); free(vprev);
    return out;
}

/* spectral_bounds (src/hydrodynamics.cpp:224-264). Counters may be NULL. */
static void spectral_bounds_counted(const double* D, int n, double* cache_vec, int* cache_valid,
                                    double* lmin_out, double* lmax_out, int* steps_out,
                                    bdcu_counters* cnt) {
    const int can_warm = (cache_vec != NULL && *cache_valid);
    double* vmin = (double*)malloc(sizeof(double) * (size_t)n);
    double* vmax = (double*)malloc(sizeof(double) * (size_t)n);
    double* V = (double*)malloc(sizeof(double) * (size_t)n * LANCZOS_COLD_I);
    long ndx = 0;
    lanczos_out r = lanczos_extremes(D, n, can_warm ? LANCZOS_WARM_I : LANCZOS_COLD_I,
                                     can_warm ? cache_vec : NULL, vmin, vmax, V, &ndx);
    if (can_warm && r.steps < 4) {
        r = lanczos_extremes(D, n, LANCZOS_COLD_I, NULL, vmin, vmax, V, &ndx);
        if (cnt) cnt->lanczos_cold++;
    } else if (cnt) {
        if (can_warm) cnt->lanczos_warm++; else cnt->lanczos_cold++;
    }
    if (cnt) cnt->dx_products += ndx;
    if (cache_vec) {
        double* u = (double*)malloc(sizeof(double) * (size_t)n);
        double* s = (double*)malloc(sizeof(double) * (size_t)n);
        default_seed(n, u);
        const double un = sqrt(dotv(u, u, n));
        for (int i = 0; i < n; ++i) s[i] = vmin[i] + vmax[i] + 0.01 * u[i] / un;
        const double sn = sqrt(dotv(s, s, n));
        if (sn > 0.0 && isfinite(sn)) {
            for (int i = 0; i < n; ++i) cache_vec[i] = s[i] / sn;
            *cache_valid = 1;
        } else {
            *cache_valid = 0;
        }
        free(u);
        free(s);
    }
    double lmin = 0.5 * r.rmin;
    const double lmax = 1.02 * r.rmax;
    if (lmin < 1.0e-12) lmin = 1.0e-12;
    if (lmin >= lmax) lmin = lmax * 1.0e-6;
    *lmin_out = lmin;
    *lmax_out = lmax;
    if (steps_out) *steps_out = r.steps;
    free(vmin); free(vmax); free(V);
}

void bdo_spectral_bounds(const double* D, int n, double* cache_vec, int* cache_valid,
                         double* lmin, double* lmax, int* steps_out) {
    spectral_bounds_counted(D, n, cache_vec, cache_valid, lmin, lmax, steps_out, NULL);
}

/* sqrt_chebyshev_coefficients (src/hydrodynamics.cpp:267-280) */
static void cheb_coefficients(int L, double da, double db, double* a) {
    double xks[MAXCHEB_I + 1];
    for (int j = 0; j <= L; ++j) a[j] = 0.0;
    for (int k = 0; k <= L; ++k) xks[k] = cos(PI_D * (k + 0.5) / (L + 1)) / da - db / da;
    for (int j = 0; j <= L; ++j) {
        for (int k = 0; k <= L; ++k) a[j] += sqrt(xks[k]) * cos(j * (k + 0.5) * PI_D / (L + 1));
        a[j] *= 2.0 / (L + 1);
    }
    a[0] /= 2.0;
}

/* chebyshev_series (src/hydrodynamics.cpp:284-312) */
static void cheb_series(const double* D, int n, const double* x0, int L, double lmin, double lmax,
                        double* result, long* ndx) {
    const double da = 2.0 / (lmax - lmin);
    const double db = -(lmax + lmin) / (lmax - lmin);
    double a[MAXCHEB_I + 1];
    cheb_coefficients(L, da, db, a);
    double* tp = (double*)malloc(sizeof(double) * (size_t)n);
    double* tc = (double*)malloc(sizeof(double) * (size_t)n);
    double* tn = (double*)malloc(sizeof(double) * (size_t)n);
    double* Dv = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) result[i] = a[0] * x0[i];
    memcpy(tp, x0, sizeof(double) * (size_t)n);
    matvec(D, n, x0, Dv);
    ++*ndx;
    for (int i = 0; i < n; ++i) tc[i] = da * Dv[i] + db * x0[i];
    for (int i = 0; i < n; ++i) result[i] += a[1] * tc[i];
    for (int l = 2; l <= L; ++l) {
        matvec(D, n, tc, Dv);
        ++*ndx;
        for (int i = 0; i < n; ++i) tn[i] = da * Dv[i] + db * tc[i];
        for (int i = 0; i < n; ++i) tn[i] = 2.0 * tn[i] - tp[i];
        double* t = tp; tp = tc; tc = tn; tn = t;
        for (int i = 0; i < n; ++i) result[i] += a[l] * tc[i];
    }
    free(tp); free(tc); free(tn); free(Dv);
}

/* chebyshev_sqrt_times (src/hydrodynamics.cpp:317-337) */
static void cheb_sqrt_counted(const double* D, int n, const double* x0, double mult, double fd_tol,
                              double* cache_vec, int* cache_valid, double* out, int* nterms,
                              double* fd_err_out, bdcu_counters* cnt) {
    double lmin, lmax;
    spectral_bounds_counted(D, n, cache_vec, cache_valid, &lmin, &lmax, NULL, cnt);
    double* Dx0 = (double*)malloc(sizeof(double) * (size_t)n);
    long ndx = 0;
    matvec(D, n, x0, Dx0);
    ++ndx;
    const double x0Dx0 = dotv(x0, Dx0, n);
    int L = (int)(sqrt(lmax / lmin) * mult + 0.5) + 1;
    L = maxi(2, mini(L, MAXCHEB_I));
    double fd_err = 0.0;
    for (;;) {
        cheb_series(D, n, x0, L, lmin, lmax, out, &ndx);
        if (cnt) cnt->cheb_terms += L;
        fd_err = fabs(dotv(out, out, n) - x0Dx0) / x0Dx0;
        if (fd_err <= fd_tol || L >= MAXCHEB_I) break;
        L = mini(MAXCHEB_I, L + maxi(1, L / 4));
    }
    if (cnt) cnt->dx_products += ndx;
    *nterms = L;
    *fd_err_out = fd_err;
    free(Dx0);
}

void bdo_chebyshev_sqrt_times(const double* D, int n, const double* x0, double mult, double fd_tol,
                              double* cache_vec, int* cache_valid, double* out, int* nterms,
                              double* fd_err) {
    cheb_sqrt_counted(D, n, x0, mult, fd_tol, cache_vec, cache_valid, out, nterms, fd_err, NULL);
}

/* ------------------------------------------------------------ integrator */

typedef struct {
    const bdcu_phys* p;
    const double* arena;
    int N, n;
    int hi; /* hstar > 0 */
    double* D;
    double* L; /* Cholesky factor (Cholesky method) */
    double* tmp;
} chain_ws;

/* Diffusion::apply (src/mobility.cpp:53-56): identity => copy. */
static void apply_D(chain_ws* w, const double* x, double* y, bdcu_counters* cnt) {
    if (!w->hi) {
        memcpy(y, x, sizeof(double) * (size_t)w->n);
        return;
    }
    matvec(w->D, w->n, x, y);
    if (cnt) cnt->dx_products++;
}

/* Fe = (EV + bending)(R) + external(t) (src/model.hpp:56-64, src/integrator.cpp:75-76). */
static void explicit_force(chain_ws* w, const double* R, double t, double* Fe) {
    const int N = w->N;
    double* a = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    double* b = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    double* bond = (double*)malloc(sizeof(double) * 3 * (size_t)N);
    double* len = (double*)malloc(sizeof(double) * (size_t)N);
    bdo_ev_force(R, N, w->p, w->arena, a);
    geometry(R, N, bond, len);
    bending_from_geom(bond, len, N, w->p, b);
    if (w->p->ext_n_entries > 0) {
        double* c = (double*)malloc(sizeof(double) * 3 * (size_t)N);
        bdo_external_force(N, w->p, w->arena, t, c);
        for (int i = 0; i < 3 * N; ++i) Fe[i] = (a[i] + b[i]) + c[i];
        free(c);
    } else {
        for (int i = 0; i < 3 * N; ++i) Fe[i] = (a[i] + b[i]) + 0.0;
    }
    free(a); free(b); free(bond); free(len);
}

int bdo_integrate(double* R, const bdcu_phys* p, const bdcu_sim* s, const double* arena,
                  int32_t rng[3], double* cache_vec_in, int* cache_valid_in,
                  bdcu_counters* cnt) {
    const int N = p->n_beads, n = 3 * N;
    const double dt = s->dt;
    const double sqrt2inv = 1.0 / sqrt(2.0);
    int status = 0;
    if (p->hstar > 0.0 && p->hi_method == BDCU_HI_EXACT_SQRT) return BDCU_ST_BAD_PARAM;

    chain_ws w;
    w.p = p; w.arena = arena; w.N = N; w.n = n; w.hi = (p->hstar > 0.0);
    w.D = w.hi ? (double*)malloc(sizeof(double) * (size_t)n * n) : NULL;
    w.L = w.hi ? (double*)malloc(sizeof(double) * (size_t)n * n) : NULL;

    double* own_cache = NULL;
    int own_valid = 0;
    double* cache_vec = cache_vec_in;
    int* cache_valid = cache_valid_in;
    if (!cache_vec) {
        own_cache = (double*)malloc(sizeof(double) * (size_t)n);
        cache_vec = own_cache;
        cache_valid = &own_valid;
    }
#define ALLOC(nm) double* nm = (double*)malloc(sizeof(double) * (size_t)n)
    ALLOC(Fs); ALLOC(Fe); ALLOC(dW); ALLOC(x0); ALLOC(Rp); ALLOC(ups); ALLOC(tmp); ALLOC(tmp2);
    ALLOC(DF); ALLOC(fl1); ALLOC(fl2); ALLOC(Fep); ALLOC(DFs); ALLOC(DFe);
    ALLOC(bond); ALLOC(len); ALLOC(Fc); ALLOC(dups); ALLOC(Rc); ALLOC(Rprev); ALLOC(Fbead);
#undef ALLOC

    for (double t = s->time_start; t <= s->time_end + s->dt / 2.0; t += s->dt) {
        /* recenter (src/integrator.cpp:88-93) */
        if (s->update_center_of_mass) {
            double com[3] = {0, 0, 0};
            for (int i = 0; i < N; ++i)
                for (int d = 0; d < 3; ++d) com[d] = com[d] + R[3 * i + d];
            for (int d = 0; d < 3; ++d) com[d] = (1.0 / N) * com[d];
            for (int i = 0; i < N; ++i)
                for (int d = 0; d < 3; ++d) R[3 * i + d] = R[3 * i + d] - com[d];
        }
        /* Fs, Fe (src/integrator.cpp:70-76) */
        bdo_spring_force(R, N, p, Fs);
        explicit_force(&w, R, t, Fe);
        /* D (src/mobility.cpp:39-51) */
        if (w.hi) {
            bdo_rpy_matrix(R, N, p->hstar, w.D);
            if (p->hi_method == BDCU_HI_CHOLESKY) {
                status |= bdo_cholesky(w.D, n, w.L);
                if (status & BDCU_ST_NOT_PD) break;
            }
        }
        /* brownian_step (src/mobility.cpp:58-88) */
        raw_noise(rng, N, x0);
        const double sqrt_dt = sqrt(dt);
        if (!w.hi) {
            for (int i = 0; i < n; ++i) dW[i] = sqrt_dt * x0[i];
        } else if (p->hi_method == BDCU_HI_CHOLESKY) {
            lower_matvec(w.L, n, x0, tmp);
            for (int i = 0; i < n; ++i) dW[i] = sqrt_dt * tmp[i];
        } else {
            int nterms;
            double fd_err;
            cheb_sqrt_counted(w.D, n, x0, p->ncheb_multiplier, p->fd_err_max, cache_vec, cache_valid,
                              tmp, &nterms, &fd_err, cnt);
            if (!(fd_err <= p->fd_err_max)) {
                status |= BDCU_ST_CHEB_FALLBACK;
                if (cnt) cnt->cheb_fallbacks++;
                int st = bdo_cholesky(w.D, n, w.L);
                if (st) { status |= st; break; }
                lower_matvec(w.L, n, x0, tmp);
            }
            for (int i = 0; i < n; ++i) dW[i] = sqrt_dt * tmp[i];
        }
        /* predictor (src/integrator.cpp:96-101) */
        double K[9], K2[9];
        bdo_kappa(p, arena, t, K);
        for (int i = 0; i < n; ++i) tmp[i] = Fs[i] + Fe[i];
        apply_D(&w, tmp, DF, cnt);
        flow_velocity(K, R, N, fl1);
        for (int i = 0; i < n; ++i) Rp[i] = R[i] + dt * (fl1[i] + 0.25 * DF[i]) + sqrt2inv * dW[i];
        /* upsilon (src/integrator.cpp:107-119) */
        explicit_force(&w, Rp, t + dt, Fep);
        bdo_kappa(p, arena, t + dt, K2);
        flow_velocity(K2, Rp, N, fl2);
        apply_D(&w, Fs, DFs, cnt);
        for (int i = 0; i < n; ++i) tmp[i] = Fe[i] + Fep[i];
        apply_D(&w, tmp, DFe, cnt);
        for (int i = 0; i < n; ++i) {
            const double flow = 0.5 * (fl1[i] + fl2[i]);
            ups[i] = R[i] + dt * (flow + 0.125 * DFs[i] + 0.125 * DFe[i]) + sqrt2inv * dW[i];
        }
        /* solve_connectors (src/integrator.cpp:125-165) */
        const int nb = N - 1;
        for (int mu = 0; mu < nb; ++mu)
            for (int d = 0; d < 3; ++d) {
                dups[3 * mu + d] = ups[3 * (mu + 1) + d] - ups[3 * mu + d];
                bond[3 * mu + d] = Rp[3 * (mu + 1) + d] - Rp[3 * mu + d];
            }
        memcpy(Rprev, Rp, sizeof(double) * (size_t)n);
        const int max_iter = 100 * N;
        double increment = 0.0;
        int iter = 0;
        for (; iter <= max_iter; ++iter) {
            for (int mu = 0; mu < nb; ++mu) len[mu] = clamped_len(bond + 3 * mu);
            connector_forces(bond, len, nb, p, Fc);
            bead_forces(Fc, N, Fbead);
            apply_D(&w, Fbead, DFs, cnt);
            for (int d = 0; d < 3; ++d) Rc[d] = Rp[d];
            for (int mu = 0; mu < nb; ++mu) {
                double g[3];
                for (int d = 0; d < 3; ++d)
                    g[d] = dups[3 * mu + d] + (0.125 * dt) * (DFs[3 * (mu + 1) + d] - DFs[3 * mu + d]) +
                           (0.25 * dt) * Fc[3 * mu + d];
                status |= bdo_solve_connector(g, dt, p, bond + 3 * mu);
                for (int d = 0; d < 3; ++d) Rc[3 * (mu + 1) + d] = Rc[3 * mu + d] + bond[3 * mu + d];
            }
            double ssum = 0.0;
            for (int i = 0; i < N; ++i) {
                double dd[3];
                for (int d = 0; d < 3; ++d) dd[d] = Rc[3 * i + d] - Rprev[3 * i + d];
                ssum += norm2_3(dd);
            }
            increment = sqrt(ssum) / N;
            if (cnt) cnt->corrector_iters++;
            if (increment < s->implicit_loop_tol) break;
            memcpy(Rprev, Rc, sizeof(double) * (size_t)n);
        }
        if (iter > max_iter) {
            status |= BDCU_ST_NONCONVERGED;
            if (cnt) cnt->nonconverged++;
        }
        if (status & BDCU_ST_FATAL_MASK) break;
        memcpy(R, Rc, sizeof(double) * (size_t)n);
        if (cnt) cnt->steps++;
    }
    free(Fs); free(Fe); free(dW); free(x0); free(Rp); free(ups); free(tmp); free(tmp2);
    free(DF); free(fl1); free(fl2); free(Fep); free(DFs); free(DFe);
    free(bond); free(len); free(Fc); free(dups); free(Rc); free(Rprev); free(Fbead);
    free(w.D); free(w.L); free(own_cache);
    return status;
}

/* ------------------------------------------------------------ threads */

typedef struct {
    double* R;
    const int64_t* off;
    const bdcu_phys* p;
    const bdcu_sim* s;
    const double* arena;
    int32_t* rng;
    int32_t* status;
    int n_chains;
    int* next;
    pthread_mutex_t* mu;
} pool_arg;

static void* pool_worker(void* vp) {
    pool_arg* a = (pool_arg*)vp;
    for (;;) {
        pthread_mutex_lock(a->mu);
        const int c = (*a->next)++;
        pthread_mutex_unlock(a->mu);
        if (c >= a->n_chains) break;
        a->status[c] = bdo_integrate(a->R + 3 * a->off[c], &a->p[c], &a->s[c], a->arena,
                                     a->rng + 3 * c, NULL, NULL, NULL);
    }
    return NULL;
}

int bdo_integrate_many(double* R, const int64_t* bead_offset, int n_chains,
                       const bdcu_phys* p, const bdcu_sim* s, const double* arena,
                       int32_t* rng, int32_t* status, int n_threads) {
    if (n_threads < 1) n_threads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
    pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
    int next = 0;
    pool_arg a = {R, bead_offset, p, s, arena, rng, status, n_chains, &next, &mu};
    for (int i = 0; i < n_threads; ++i) pthread_create(&th[i], NULL, pool_worker, &a);
    for (int i = 0; i < n_threads; ++i) pthread_join(th[i], NULL);
    free(th);
    return 0;
}
