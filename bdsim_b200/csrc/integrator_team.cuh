// integrator_team.cuh -- the FP32-mixed form with one chain per TEAM of T
// warps (T = 1, 2, 4, 8), for chains of up to 64*T beads. Each team claims
// chains from the device work queue and owns one chain at a time; team thread
// u owns beads u and u + 32T, holding their positions, forces and noise in
// registers. There is no block-wide barrier: neighbour data (bonds, prefix
// sums) goes through the team's own shared-memory area under the team barrier
// (__syncwarp for T = 1, a named barrier otherwise); reductions are warp
// shuffles followed, for T > 1, by a fixed-order sum over the team's warps.
//
// Precision (the mixed form): D.x recomputed pairwise in FP32 from shared FP32
// bead coordinates, FP32 excluded volume and Chebyshev recurrence; FP64
// positions, spring/bending forces, connector solve, Lanczos vectors and
// tridiagonal bounds, and the (rare) Cholesky fallback. The noise stream is
// the reference's ran_1 stream bit for bit, drawn by all team threads at once
// with a jump-ahead (GF(2) powers of the xorshift step, powers of 16807 mod
// 2^31-1).
//
// Reference: src/integrator.cpp:61-170 of the bdsim project and the physics it
// calls; each stage cites its reference function.
#pragma once

#include "integrator.cuh"
#include "team_layout.h"

namespace bdcu {

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Barrier over one team: __syncwarp for a single warp, else named barrier
// 1 + team (barrier 0 is __syncthreads') over the team's 32T threads.
template <int T>
__device__ __forceinline__ void team_sync(int team) {
    if constexpr (T == 1) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(32 * T) : "memory");
    }
}

// Number of eigenvalues of the tridiagonal (a, b) below x, from the signs of
// the leading principal minors p_i = (a_i - x) p_{i-1} - b_{i-1}^2 p_{i-2}
// (divide-free Sturm sequence, rescaled against overflow). The mixed form
// uses it in place of sturm_count (src/hydrodynamics.cpp:91-104).
__device__ __forceinline__ int sturm_count_products(const double* a, const double* b, int m, double x) {
    double pm = 1.0, p = a[0] - x;
    int count = (p < 0.0) ? 1 : 0;
    for (int i = 1; i < m; ++i) {
        const double pn = (a[i] - x) * p - b[i - 1] * b[i - 1] * pm;
        count += ((pn < 0.0) != (p < 0.0)) ? 1 : 0;
        pm = p;
        p = pn;
        if (fabs(p) > 1e150) {
            p *= 1e-150;
            pm *= 1e-150;
        }
    }
    return count;
}

// Bisection for the target-th eigenvalue boundary on a half warp (16 lanes,
// depth-4 speculative tree), the iteration of src/hydrodynamics.cpp:196-207.
static __device__ void halfwarp_bisect(const double* al, const double* bb, int k, int target, double& lo, double& hi) {
    const int lane = threadIdx.x & 15;
    const int lvl = 31 - __clz(lane + 1);
    const int p = lane + 1 - (1 << lvl);
    for (int it = 0; it < 100; it += 4) {
        int dec = 0;
        if (lane < 15) {
            double a = lo, b = hi;
            for (int l = 0; l < lvl; ++l) {
                const int bit = (p >> (lvl - 1 - l)) & 1;
                const double m = 0.5 * (a + b);
                if (bit == 0) b = m; else a = m;
            }
            const double mid = 0.5 * (a + b);
            dec = (sturm_count_products(al, bb, k, mid) >= target) ? 0 : 1;
        }
        int node = 0;
        double na = lo, nb = hi;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int d = __shfl_sync(kFull, dec, node, 16);
            const double m = 0.5 * (na + nb);
            if (d == 0) nb = m; else na = m;
            node = 2 * node + 1 + d;
        }
        // settled: the interval stopped shrinking or is within 1e-10 relative
        // (the bounds are padded by 2x / 2% downstream)
        const bool done = (na == lo && nb == hi) || (nb - na) <= 1e-10 * fmax(fabs(na), fabs(nb));
        lo = na;
        hi = nb;
        if (__all_sync(kFull, done)) break;
    }
}

// Sturm count below x for a tridiagonal of k <= kLanczosWarm entries held in
// registers (a: diagonal, b: off-diagonal), the divide-free recurrence of
// sturm_count_products fully unrolled.
__device__ __forceinline__ int sturm_count_reg(const double (&a)[kLanczosWarm], const double (&b)[kLanczosWarm], int k,
                                               double x) {
    double pm = 1.0, p = a[0] - x;
    int count = (p < 0.0) ? 1 : 0;
#pragma unroll
    for (int i = 1; i < kLanczosWarm; ++i) {
        if (i < k) {
            const double pn = (a[i] - x) * p - (b[i - 1] * b[i - 1]) * pm;
            count += ((pn < 0.0) != (p < 0.0)) ? 1 : 0;
            pm = p;
            p = pn;
            if (fabs(p) > 1e150) {
                p *= 1e-150;
                pm *= 1e-150;
            }
        }
    }
    return count;
}

// Multisection for the target-th eigenvalue boundary on a half warp: 15 lanes
// evaluate the Sturm count at 15 evenly spaced interior points of [lo, hi], a
// ballot finds the sixteenth that holds the boundary (4 bits per round), the
// iteration of src/hydrodynamics.cpp:196-207 in place of its halvings. Every
// lane of the half warp ends with the same lo, hi.
static __device__ void halfwarp_multisect(const double (&a)[kLanczosWarm], const double (&b)[kLanczosWarm], int k,
                                          int target, double& lo, double& hi) {
    const int h = threadIdx.x & 15;
    const int shift = threadIdx.x & 16;
    for (int it = 0; it < 25; ++it) {
        const double w = hi - lo;
        const bool ge = h < 15 && sturm_count_reg(a, b, k, lo + w * ((double)(h + 1) * 0.0625)) >= target;
        const unsigned bal = (__ballot_sync(kFull, ge) >> shift) & 0xffffu;
        const int f = bal ? __ffs(bal) - 1 : 15;
        const double nlo = f == 0 ? lo : lo + w * ((double)f * 0.0625);
        const double nhi = f == 15 ? hi : lo + w * ((double)(f + 1) * 0.0625);
        // settled: the interval stopped shrinking or is within 1e-6 relative
        // (the bounds are padded by 2x / 2% downstream, and the FD check
        // polices the Chebyshev result)
        const bool done = (nlo == lo && nhi == hi) || (nhi - nlo) <= 1e-6 * fmax(fabs(nlo), fabs(nhi));
        lo = nlo;
        hi = nhi;
        if (__all_sync(kFull, done)) break;
    }
}

// 1/x for |x| in [1e-30, 1e30]: a single-precision seed refined by two
// Newton-Raphson steps r <- r (2 - x r) (quadratic convergence: 2^-23 ->
// 2^-46 -> below double rounding).
__device__ __forceinline__ double rcp_newton(double x) {
    double r = (double)__frcp_rn((float)x);
    r = r * (2.0 - x * r);
    r = r * (2.0 - x * r);
    return r;
}

// Inverse iteration for a Ritz vector (src/hydrodynamics.cpp:106-136) with the
// tridiagonal (k <= kLanczosWarm) in registers; every lane that calls it
// computes the same y.
static __device__ void tridiag_vec_reg(const double (&a)[kLanczosWarm], const double (&b)[kLanczosWarm], int m,
                                       double lambda, double (&y)[kLanczosWarm]) {
    const double scale = dmax_(fabs(lambda), 1.0);
    const double shift = lambda - 1.0e-7 * scale;
    const double y0 = rsqrt((double)m);
    double c[kLanczosWarm];
#pragma unroll
    for (int i = 0; i < kLanczosWarm; ++i) y[i] = i < m ? y0 : 0.0;
    // one pass: the shift is within 1e-6 relative of the eigenvalue, so a
    // single solve already amplifies its eigenvector by ~1e5 over the others
    // (the vector only seeds the next step's Lanczos)
    for (int it = 0; it < 1; ++it) {
        // pivots: the reference's tiny-pivot guard (1e-300) raised to 1e-30 so
        // that the reciprocal's single-precision seed stays in range (the
        // vector only seeds the next step's Lanczos)
        double beta = a[0] - shift;
        if (fabs(beta) < 1.0e-30) beta = 1.0e-30;
        double ib = rcp_newton(beta);
        c[0] = (m > 1 ? b[0] * ib : 0.0);
        y[0] = y[0] * ib;
#pragma unroll
        for (int i = 1; i < kLanczosWarm; ++i) {
            if (i < m) {
                beta = (a[i] - shift) - b[i - 1] * c[i - 1];
                if (fabs(beta) < 1.0e-30) beta = 1.0e-30;
                ib = rcp_newton(beta);
                c[i] = (i < m - 1 ? b[i] * ib : 0.0);
                y[i] = (y[i] - b[i - 1] * y[i - 1]) * ib;
            }
        }
#pragma unroll
        for (int i = kLanczosWarm - 2; i >= 0; --i)
            if (i < m - 1) y[i] = y[i] - c[i] * y[i + 1];
        double nrm = 0.0;
#pragma unroll
        for (int i = 0; i < kLanczosWarm; ++i) nrm += y[i] * y[i];
        nrm = sqrt(nrm);
        if (!(nrm > 0.0) || !isfinite(nrm)) {
#pragma unroll
            for (int i = 0; i < kLanczosWarm; ++i) y[i] = i < m ? y0 : 0.0;
            return;
        }
        const double inr = 1.0 / nrm;
#pragma unroll
        for (int i = 0; i < kLanczosWarm; ++i) y[i] *= inr;
    }
}

// Inverse iteration for a Ritz vector (src/hydrodynamics.cpp:106-136), one lane.
static __device__ void wk_tridiag_vec(const double* a, const double* b, int m, double lambda, double* y, double* c,
                                      double* d) {
    const double scale = dmax_(fabs(lambda), 1.0);
    const double shift = lambda - 1.0e-7 * scale;
    const double y0 = rsqrt((double)m);
    for (int i = 0; i < m; ++i) y[i] = y0;
    for (int it = 0; it < 2; ++it) {
        double beta0 = a[0] - shift;
        if (fabs(beta0) < 1.0e-300) beta0 = 1.0e-300;
        double ib = 1.0 / beta0;
        c[0] = (m > 1 ? b[0] * ib : 0.0);
        d[0] = y[0] * ib;
        for (int i = 1; i < m; ++i) {
            double beta = (a[i] - shift) - b[i - 1] * c[i - 1];
            if (fabs(beta) < 1.0e-300) beta = 1.0e-300;
            ib = 1.0 / beta;
            c[i] = (i < m - 1 ? b[i] * ib : 0.0);
            d[i] = (y[i] - b[i - 1] * d[i - 1]) * ib;
        }
        y[m - 1] = d[m - 1];
        for (int i = m - 2; i >= 0; --i) y[i] = d[i] - c[i] * y[i + 1];
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += y[i] * y[i];
        nrm = sqrt(nrm);
        if (!(nrm > 0.0) || !isfinite(nrm)) {
            for (int i = 0; i < m; ++i) y[i] = y0;
            return;
        }
        const double inr = 1.0 / nrm;
        for (int i = 0; i < m; ++i) y[i] *= inr;
    }
}


template <int T, int Q>
struct TeamChain {
    static constexpr int TT = 32 * T;  // threads of the team
    const RunArgs& a;
    TeamShared<T, Q>& S;
    const DevChain& ch;
    double* V;      // warm Lanczos basis in shared memory (kLanczosWarm x nv)
    float* sqx;     // Chebyshev node values, aliasing V (dead after the bounds)
    float* coef;    // Chebyshev coefficients, aliasing V
    double* Vg;     // cold basis in global scratch (kLanczosCold x nv)
    double* Lt;     // Cholesky factor in global scratch (n x n)
    int nv;
    int tid;        // thread in the team
    int wl, wi;     // lane in its warp, warp in the team
    int team;       // team in the thread block (named barrier 1 + team)
    int N, n;
    bool hi;
    int32_t cnt[8];  // this call's counts for the chain (added to the 64-bit counters at the end)
    int status;
    // RPY constants (FP32). Bead coordinates are staged divided by `scale`
    // (= h* under HI), which turns the RPY weights into functions of
    // rho = h*/r alone.
    float scale, iscale, K1, K2, K3, C3, C7;

    __device__ TeamChain(const RunArgs& a_, TeamShared<T, Q>& S_, const DevChain& ch_) : a(a_), S(S_), ch(ch_) {}

    __device__ __forceinline__ bool valid(int q) const { return tid + TT * q < N; }
    __device__ __forceinline__ int bead(int q) const { return tid + TT * q; }
    __device__ __forceinline__ void sync() const { team_sync<T>(team); }

    // Sum over the team, the same bits in every thread: warp butterflies, then
    // the warps' partial sums added in warp order.
    __device__ double tsum(double v) const {
        v = wsum(v);
        if constexpr (T == 1) {
            return v;
        } else {
            sync();
            if (wl == 0) S.red[wi] = v;
            sync();
            double s = S.red[0];
#pragma unroll
            for (int w = 1; w < T; ++w) s += S.red[w];
            return s;
        }
    }

    // Eight team sums at once (the batched projections of the warm Lanczos),
    // the same bits in every thread. In each warp a transposed reduction:
    // exchange halves of the vector with lane^16, ^8, ^4 (each lane keeps the
    // half its lane bit selects), then a butterfly over lane^2, ^1, leaves sum
    // u = 4*b4 + 2*b3 + b2 in the lanes whose bits 4, 3, 2 are b4, b3, b2;
    // lanes 0, 4, ..., 28 publish the warp's eight sums in shared memory and
    // the warps' partials are added in warp order.
    __device__ void tsum8(double (&c)[kLanczosWarm]) const {
        static_assert(kLanczosWarm == 8, "tsum8 reduces eight values");
        const bool u16 = wl & 16, u8 = wl & 8, u4 = wl & 4;
        double k4[4], k2[2];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double send = u16 ? c[u] : c[u + 4];
            k4[u] = (u16 ? c[u + 4] : c[u]) + __shfl_xor_sync(kFull, send, 16);
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const double send = u8 ? k4[u] : k4[u + 2];
            k2[u] = (u8 ? k4[u + 2] : k4[u]) + __shfl_xor_sync(kFull, send, 8);
        }
        double s = (u4 ? k2[1] : k2[0]) + __shfl_xor_sync(kFull, u4 ? k2[0] : k2[1], 4);
        s += __shfl_xor_sync(kFull, s, 2);
        s += __shfl_xor_sync(kFull, s, 1);
        const int idx = (u16 ? 4 : 0) + (u8 ? 2 : 0) + (u4 ? 1 : 0);
        if constexpr (T == 1) {
            if ((wl & 3) == 0) S.red[idx] = s;
            __syncwarp();
#pragma unroll
            for (int u = 0; u < kLanczosWarm; ++u) c[u] = S.red[u];
            __syncwarp();
        } else {
            sync();
            if ((wl & 3) == 0) S.red[kLanczosWarm * wi + idx] = s;
            sync();
#pragma unroll
            for (int u = 0; u < kLanczosWarm; ++u) {
                double v = S.red[u];
#pragma unroll
                for (int w = 1; w < T; ++w) v += S.red[kLanczosWarm * w + u];
                c[u] = v;
            }
        }
    }

    // OR of status bits over the team.
    __device__ int tor(int v) const {
        v = __reduce_or_sync(kFull, v);
        if constexpr (T == 1) {
            return v;
        } else {
            sync();
            if (wl == 0) S.flag[wi] = v;
            sync();
            int s = 0;
#pragma unroll
            for (int w = 0; w < T; ++w) s |= S.flag[w];
            return s;
        }
    }

    // ---- FP32 matrix-free D.x (Diffusion::apply, src/mobility.cpp:53-56;
    // RPY weights src/hydrodynamics.cpp:36-43). x, y: the thread's beads.
    // K products against the same D in one pass over the bead pairs: the
    // pair geometry and weights are computed once for all K inputs (K = 3
    // for the products of a step that do not depend on one another).
    //
    // The single products (K = 1, most of the step's passes) take the
    // partner beads j two at a time in packed FP32x2 arithmetic (sm_100's
    // FADD2 / FMUL2 / FFMA2: one issue slot for the pair; the FP32 pipe rate
    // is that of scalar FFMA, measured 73 TFLOP/s on one B200 either way),
    // from coordinates and inputs staged by component in shared memory, so
    // one 64-bit broadcast load brings (j, j+1) of a component. Each bead's
    // sum is kept as two interleaved partial sums (even and odd j), added at
    // the end. An odd N is padded with one zero input (whose contribution
    // om1 * 0 + om2 (d . 0) d is exactly zero).
    template <int K>
    __device__ void applyK(const float (&x)[K][Q][3], float (&acc)[K][Q][3]) {
        static_assert(K >= 1 && K <= 3, "applyK stages at most three inputs");
        cnt[C_DX] += K;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (valid(q))
#pragma unroll
                for (int r = 0; r < K; ++r)
#pragma unroll
                    for (int d = 0; d < 3; ++d) S.xk[r][d][bead(q)] = x[r][q][d];
        if ((N & 1) && tid < 3 * K) S.xk[tid / 3][tid % 3][N] = 0.f;
        sync();
        // In units of h*: with d = (R_j - R_b)/h*, s = |d|^2, rho = s^-1/2,
        //   far  (s >= 4 pi): om1 = rho (K1 + K2 rho^2), om2 = rho^3 (K1 - K3 rho^2)
        //   near (s <  4 pi): om1 = 1 - C3 s rho,         om2 = C7 rho
        // and y_b += om1 x_j + om2 (d.x_j) d; both branches' weights are
        // computed and each is selected once. The self
        // pair (d = 0, s clamped to 1e-24) takes the near branch with om1 = 1
        // exactly in FP32 and om2 d = 0: it contributes the identity block.
        bool one_slot = false;
        if constexpr (Q == 2) one_slot = __all_sync(kFull, !valid(1));
        const int nq = one_slot ? 1 : Q;
        {
            // every product (the Lanczos, Chebyshev, upsilon and corrector
            // ones, and the fused sets of K = 2, 3): partner beads two at a
            // time in packed FP32x2
            float2 nb[Q][3], a[K][Q][3];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const float v = valid(q) ? -S.ps[d][bead(q)] : 0.f;
                    nb[q][d] = make_float2(v, v);
                    for (int r = 0; r < K; ++r) a[r][q][d] = make_float2(0.f, 0.f);
                }
            const float2 k1 = make_float2(K1, K1), k2 = make_float2(K2, K2), mk3 = make_float2(-K3, -K3);
            const float2 mc3 = make_float2(-C3, -C3), c7 = make_float2(C7, C7), one = make_float2(1.f, 1.f);
            const int n2 = (N + 1) & ~1;
            // not unrolled: this loop is inlined at every product's call site
#pragma unroll 1
            for (int j = 0; j < n2; j += 2) {
                float2 pj[3], xj[K][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    pj[d] = *reinterpret_cast<const float2*>(&S.ps[d][j]);
                    for (int r = 0; r < K; ++r) xj[r][d] = *reinterpret_cast<const float2*>(&S.xk[r][d][j]);
                }
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    if (q < nq) {
                        const float2 dx = __fadd2_rn(pj[0], nb[q][0]);
                        const float2 dy = __fadd2_rn(pj[1], nb[q][1]);
                        const float2 dz = __fadd2_rn(pj[2], nb[q][2]);
                        float2 sq = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                        sq = make_float2(fmaxf(sq.x, 1e-24f), fmaxf(sq.y, 1e-24f));
                        const float2 rho = make_float2(rsqrtf(sq.x), rsqrtf(sq.y));
                        const float2 t = __fmul2_rn(rho, rho);
                        const float2 u = __ffma2_rn(k2, t, k1), v = __ffma2_rn(mk3, t, k1);
                        const float2 r = __fmul2_rn(sq, rho), rt = __fmul2_rn(rho, t);
                        const bool fx = sq.x >= 12.566370614359172f, fy = sq.y >= 12.566370614359172f;
                        // both branches' weights, then one select each (a far
                        // weight of the clamped self pair may be infinite: it
                        // is not selected)
                        const float2 f1 = __fmul2_rn(rho, u), f2 = __fmul2_rn(rt, v);
                        const float2 n1 = __ffma2_rn(mc3, r, one), n2 = __fmul2_rn(c7, rho);
                        const float2 om1 = make_float2(fx ? f1.x : n1.x, fy ? f1.y : n1.y);
                        const float2 om2 = make_float2(fx ? f2.x : n2.x, fy ? f2.y : n2.y);
#pragma unroll
                        for (int r = 0; r < K; ++r) {
                            const float2 tt = __fmul2_rn(
                                om2, __ffma2_rn(dz, xj[r][2], __ffma2_rn(dy, xj[r][1], __fmul2_rn(dx, xj[r][0]))));
                            a[r][q][0] = __ffma2_rn(tt, dx, __ffma2_rn(om1, xj[r][0], a[r][q][0]));
                            a[r][q][1] = __ffma2_rn(tt, dy, __ffma2_rn(om1, xj[r][1], a[r][q][1]));
                            a[r][q][2] = __ffma2_rn(tt, dz, __ffma2_rn(om1, xj[r][2], a[r][q][2]));
                        }
                    }
                }
            }
            sync();
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    for (int r = 0; r < K; ++r) acc[r][q][d] = valid(q) ? a[r][q][d].x + a[r][q][d].y : 0.f;
        }
    }

    __device__ void apply32(const float (&x)[Q][3], float (&acc)[Q][3]) {
        applyK<1>(reinterpret_cast<const float(&)[1][Q][3]>(x), reinterpret_cast<float(&)[1][Q][3]>(acc));
    }

    __device__ void apply(const double (&x)[Q][3], double (&y)[Q][3]) {
        if (!hi) {
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) y[q][d] = x[q][d];
            return;
        }
        float xf[Q][3], yf[Q][3];
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) xf[q][d] = (float)x[q][d];
        apply32(xf, yf);
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) y[q][d] = (double)yf[q][d];
    }

    // D.x on FP32 thread vectors (identity without HI).
    __device__ void applyF(const float (&x)[Q][3], float (&y)[Q][3]) {
        if (!hi) {
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) y[q][d] = x[q][d];
            return;
        }
        apply32(x, y);
    }

    __device__ double dotf(const float (&x)[Q][3], const float (&y)[Q][3]) const {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) s += (double)x[q][d] * (double)y[q][d];
        return tsum(s);
    }

    __device__ double dot(const double (&x)[Q][3], const double (&y)[Q][3]) const {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) s += x[q][d] * y[q][d];
        return tsum(s);
    }

    __device__ void stage_pos(const double (&R)[Q][3]) {
        sync();
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (valid(q)) {
                const float x = (float)(R[q][0] * iscale), y = (float)(R[q][1] * iscale), z = (float)(R[q][2] * iscale);
                S.pos[bead(q)] = make_float4(x, y, z, 0.f);
                S.ps[0][bead(q)] = x;
                S.ps[1][bead(q)] = y;
                S.ps[2][bead(q)] = z;
            }
        if ((N & 1) && tid < 3) S.ps[tid][N] = 0.f;  // the odd-N pad bead (zero input in every pass)
        sync();
    }

    __device__ void to_smem(double* buf, const double (&x)[Q][3]) const {
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (valid(q))
#pragma unroll
                for (int d = 0; d < 3; ++d) buf[3 * bead(q) + d] = x[q][d];
    }

    // ---- forces at R (FP64 springs/bending/external, FP32 EV) ------------
    // Fs: spring bead forces (src/spring.cpp:195-207). Fe: (EV + bending) +
    // external(t) (src/model.hpp:56-64). Positions must be staged (S.pos).
    __device__ void forces(const double (&R)[Q][3], double t, float (&Fs)[Q][3], float (&Fe)[Q][3], bool spring) {
        const bool bend = ch.bend_type != BDCU_BEND_NONE && N > 2;
        const bool bonds = spring || bend;  // bond forces, unit bonds, lengths: springs and bending only
        if (bonds) to_smem(S.s0, R);
        sync();
        // bonds b = bead(0), bead(1) (b < N-1): Fc -> s1, unit bonds -> s2, lengths -> s3
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int b = bead(q);
            if (bonds && b < N - 1) {
                const double b0 = S.s0[3 * b + 3] - S.s0[3 * b], b1 = S.s0[3 * b + 4] - S.s0[3 * b + 1],
                             b2 = S.s0[3 * b + 5] - S.s0[3 * b + 2];
                const double len = clamped_len(b0, b1, b2);
                const double f = connector_factor(ch, len);
                S.s1[3 * b] = f * b0;
                S.s1[3 * b + 1] = f * b1;
                S.s1[3 * b + 2] = f * b2;
                const double il = 1.0 / len;
                S.s2[3 * b] = il * b0;
                S.s2[3 * b + 1] = il * b1;
                S.s2[3 * b + 2] = il * b2;
                S.s3[b] = len;
            }
        }
        sync();
        if (bend) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int b = bead(q);
                if (b < N - 2)
                    S.s4[b] = S.s2[3 * (b + 1)] * S.s2[3 * b] + S.s2[3 * (b + 1) + 1] * S.s2[3 * b + 1] +
                              S.s2[3 * (b + 1) + 2] * S.s2[3 * b + 2];
            }
            sync();
        }
        // EV on the scaled coordinates: r = scale*|d|, force -fac(r) * scale * d
        const float zs = (float)(ch.zsbyds5 * scale), p5 = (float)(ch.pt5bydssq * (double)scale * scale);
        const double* phi = (ch.ev_type == BDCU_EV_SDK && ch.phi_off >= 0) ? a.arena + ch.phi_off : nullptr;
        // excluded volume, FP32 pair sums over both bead slots at once: the
        // force on m from j is -fac(r) (R_j - R_m), |j - m| >= contour distance
        float fev[Q][3] = {};
        if (ch.ev_type == BDCU_EV_GAUSS) {
            float4 pm[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) pm[q] = valid(q) ? S.pos[bead(q)] : make_float4(0.f, 0.f, 0.f, 0.f);
            const int cd = ch.cd;
#pragma unroll 2
            for (int j = 0; j < N; ++j) {
                const float4 pj = S.pos[j];
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int m = bead(q);
                    const float dx = pj.x - pm[q].x, dy = pj.y - pm[q].y, dz = pj.z - pm[q].z;
                    const float sq = dx * dx + dy * dy + dz * dz;
                    const int dj = j > m ? j - m : m - j;
                    const float fac = (dj >= cd && j != m) ? zs * __expf(-sq * p5) : 0.f;
                    fev[q][0] -= fac * dx;
                    fev[q][1] -= fac * dy;
                    fev[q][2] -= fac * dz;
                }
            }
        } else if (ch.ev_type != BDCU_EV_NONE) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int m = bead(q);
                if (!valid(q)) continue;
                const float4 pm = S.pos[m];
                for (int j = 0; j < N; ++j) {
                    const int dj = j > m ? j - m : m - j;
                    if (dj < ch.cd || j == m) continue;
                    const float4 pj = S.pos[j];
                    const float dx = pj.x - pm.x, dy = pj.y - pm.y, dz = pj.z - pm.z;
                    const float sq = fmaxf(dx * dx + dy * dy + dz * dz, 1e-12f);
                    const int mu = j < m ? j : m, nu = j < m ? m : j;
                    const float fac =
                        (float)(ev_factor(ch, sqrt((double)sq) * scale, phi ? phi[mu * N + nu] : 0.0) * scale);
                    fev[q][0] -= fac * dx;
                    fev[q][1] -= fac * dy;
                    fev[q][2] -= fac * dz;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int m = bead(q);
            if (!valid(q)) {
                for (int d = 0; d < 3; ++d) Fs[q][d] = Fe[q][d] = 0.f;
                continue;
            }
            if (spring) {
                for (int d = 0; d < 3; ++d) {
                    double v;
                    if (m == 0) v = S.s1[d];
                    else if (m == N - 1) v = -S.s1[3 * (N - 2) + d];
                    else v = S.s1[3 * m + d] - S.s1[3 * (m - 1) + d];
                    Fs[q][d] = (float)v;
                }
            }
            double fb[3] = {0.0, 0.0, 0.0}, fx[3] = {0.0, 0.0, 0.0};
            if (bend) bending_on_bead(ch, m, S.s2, S.s4, S.s3, fb);
            if (ch.ext_n > 0) external_on_bead(ch, a.arena, m, t, fx);
            Fe[q][0] = (float)(((double)fev[q][0] + fb[0]) + fx[0]);
            Fe[q][1] = (float)(((double)fev[q][1] + fb[1]) + fx[1]);
            Fe[q][2] = (float)(((double)fev[q][2] + fb[2]) + fx[2]);
        }
        sync();
    }

    // ---- noise: the 3N draws of raw_noise (src/mobility.cpp:18-29) -------
    // The team's threads draw contiguous blocks of the stream; thread u jumps
    // to draw u*c with the tabulated powers, so the uniforms equal ran_1's,
    // bit for bit.
    __device__ void noise(uint32_t& ux0, int32_t& iy0, int32_t& seed, float (&X)[Q][3]) {
        if (seed <= 0 || iy0 < 0) {
            const int32_t s = seed < 0 ? -seed : seed;
            iy0 = (888889999 ^ s) | 1;
            ux0 = (uint32_t)(777755555 ^ s);
            seed = s + 1;
        }
        const int c = (n + TT - 1) / TT;
        const int k0 = tid * c;
        const int k1 = min(n, k0 + c);
        uint32_t ux = 0;
        int32_t iy = 0;
        if (k0 < n) {
            const uint32_t* cols = a.xs_pow + 32 * (int64_t)k0;
#pragma unroll 8
            for (int i = 0; i < 32; ++i) ux ^= cols[i] & (0u - ((ux0 >> i) & 1u));
            iy = (int32_t)(((uint64_t)a.a_pow[k0] * (uint64_t)(uint32_t)iy0) % 2147483647ull);
            const float am = __fdiv_rn(__int_as_float(0x3f7fffff), 2147483648.0f);
            for (int k = k0; k < k1; ++k) {
                ux ^= (ux << 13);
                ux ^= (ux >> 17);
                ux ^= (ux << 5);
                const int32_t kk = iy / 127773;
                iy = 16807 * (iy - kk * 127773) - 2836 * kk;
                if (iy < 0) iy += 2147483647;
                const uint32_t mixed = ux ^ (uint32_t)iy;
                const int32_t res = (int32_t)((mixed & 0x7fffffffu) | 1u);
                S.s0[k] = (double)__fmul_rn(am, __int2float_rn(res));
            }
        }
        // the state after the last draw, from the thread that made it
        const int last = (n - 1) / c;
        if constexpr (T == 1) {
            ux0 = __shfl_sync(kFull, ux, last);
            iy0 = __shfl_sync(kFull, iy, last);
            __syncwarp();
        } else {
            if (tid == last) {
                S.bu = ux;
                S.bi = iy;
            }
            sync();
            ux0 = S.bu;
            iy0 = S.bi;
        }
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double v = 0.0;
                if (valid(q)) {
                    const double y = S.s0[3 * bead(q) + d] - 0.5;
                    v = (14.14855378 * y * y + 1.21569221) * y;
                }
                X[q][d] = (float)v;
            }
        sync();
    }

    // ---- Lanczos extreme eigenvalues (src/hydrodynamics.cpp:146-264) ----
    __device__ double* basis(int j, int m) { return (m <= kLanczosWarm ? V : Vg) + (int64_t)j * nv; }
    __device__ void load(const double* vec, double (&x)[Q][3]) const {
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) x[q][d] = valid(q) ? vec[3 * bead(q) + d] : 0.0;
    }
    __device__ void store(double* vec, const double (&x)[Q][3]) const {
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (valid(q))
#pragma unroll
                for (int d = 0; d < 3; ++d) vec[3 * bead(q) + d] = x[q][d];
    }

    // Lanczos start vector (src/hydrodynamics.cpp:152-155): the normalised
    // warm-start cache, or the normalised default seed when cold or when the
    // cache is zero.
    __device__ void start_vector(bool warm, const double* cache, double (&v)[Q][3]) const {
        double nv2 = 0.0;
        if (warm) {
            load(cache, v);
            nv2 = sqrt(dot(v, v));
        }
        if (!(nv2 > 0.0)) {
            load(a.seed_table, v);
            nv2 = ch.seed_norm;
        }
        const double inv = 1.0 / nv2;
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) v[q][d] *= inv;
    }

    // Returns the number of Lanczos steps; sets rmin/rmax and the Ritz vectors.
    // v0: the start vector; if have_dv0, dv0 = D v0 (computed by the caller
    // together with the step's other independent products).
    __device__ int lanczos(int m, bool warm, const double (&v0)[Q][3], const double (&dv0)[Q][3], bool have_dv0,
                           double (&vmin)[Q][3], double (&vmax)[Q][3], double& rmin, double& rmax) {
        if (n < m) m = n;
        double v[Q][3], w[Q][3], vp[Q][3];
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) v[q][d] = v0[q][d];
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) vp[q][d] = 0.0;
        int k = 0;
        double b = 0.0;
        if (m <= kLanczosWarm) {
            // warm runs (8 steps from the previous step's Ritz vectors): the
            // three-term recurrence without reorthogonalisation. In 8 FP64
            // steps the loss of orthogonality (of order eps over the accuracy
            // of the converged Ritz values) leaves the extreme Ritz values far
            // inside the 2x / 2% padding of the bounds, and the Chebyshev
            // fluctuation-dissipation check polices the result. One batched
            // team sum per step gives alpha = v.w and |w|^2, so beta^2 =
            // |w|^2 - alpha^2 (Pythagoras, |v| = 1); when that cancels by more
            // than 99% beta comes from an explicit norm. The last step's beta
            // is not needed (it is not an entry of T).
            for (int j = 0; j < m; ++j) {
                store(basis(j, m), v);
                if (j == 0 && have_dv0) {
#pragma unroll
                    for (int q = 0; q < Q; ++q)
#pragma unroll
                        for (int d = 0; d < 3; ++d) w[q][d] = dv0[q][d];
                } else {
                    apply(v, w);
                }
                if (j > 0)
#pragma unroll
                    for (int q = 0; q < Q; ++q)
#pragma unroll
                        for (int d = 0; d < 3; ++d) w[q][d] -= b * vp[q][d];
                double c[kLanczosWarm];
#pragma unroll
                for (int u = 0; u < kLanczosWarm; ++u) c[u] = 0.0;
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        c[0] += v[q][d] * w[q][d];
                        c[1] += w[q][d] * w[q][d];
                    }
                tsum8(c);
                const double al = c[0];
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) w[q][d] -= al * v[q][d];
                if (tid == 0) S.alpha[k] = al;
                ++k;
                if (j == m - 1) break;
                double bsq = c[1] - al * al;
                if (!(bsq >= 0.01 * c[1])) bsq = dot(w, w);
                b = sqrt(bsq);
                if (b < 1.0e-10) break;
                const double ib = 1.0 / b;
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        vp[q][d] = v[q][d];
                        v[q][d] = w[q][d] * ib;
                    }
                if (tid == 0) S.beta[j] = b;
            }
        } else {
            // cold runs (first step of a call): the reference's modified Gram-Schmidt
            for (int j = 0; j < m; ++j) {
                store(basis(j, m), v);
                if (j == 0 && have_dv0) {
#pragma unroll
                    for (int q = 0; q < Q; ++q)
#pragma unroll
                        for (int d = 0; d < 3; ++d) w[q][d] = dv0[q][d];
                } else {
                    apply(v, w);
                }
                const double al = dot(v, w);
                if (tid == 0) S.alpha[k] = al;
                ++k;
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) w[q][d] -= al * v[q][d] + b * vp[q][d];
                sync();
                for (int u = 0; u <= j; ++u) {
                    double uu[Q][3];
                    load(basis(u, m), uu);
                    const double dd = dot(w, uu);
#pragma unroll
                    for (int q = 0; q < Q; ++q)
#pragma unroll
                        for (int d = 0; d < 3; ++d) w[q][d] -= dd * uu[q][d];
                }
                b = sqrt(dot(w, w));
                if (b < 1.0e-10) break;
                const double ib = 1.0 / b;
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        vp[q][d] = v[q][d];
                        v[q][d] = w[q][d] * ib;
                    }
                if (tid == 0) S.beta[j] = b;
            }
        }
        sync();
        if (k == 1) {
            rmin = rmax = S.alpha[0];
            load(basis(0, m), vmin);
            load(basis(0, m), vmax);
            return 1;
        }
        if (wi == 0 && k <= kLanczosWarm) {
            // warm-sized tridiagonal in registers: Gershgorin bracket, then
            // lanes 0-15 find the smallest eigenvalue and its Ritz vector,
            // lanes 16-31 the largest
            double ar[kLanczosWarm], br[kLanczosWarm];
#pragma unroll
            for (int i = 0; i < kLanczosWarm; ++i) {
                ar[i] = i < k ? S.alpha[i] : 0.0;
                br[i] = i < k - 1 ? S.beta[i] : 0.0;
            }
            double lo = ar[0], hi2 = ar[0];
#pragma unroll
            for (int i = 0; i < kLanczosWarm; ++i) {
                if (i < k) {
                    const double rad = (i > 0 ? fabs(br[i - 1]) : 0.0) + fabs(br[i]);
                    lo = dmin_(lo, ar[i] - rad);
                    hi2 = dmax_(hi2, ar[i] + rad);
                }
            }
            halfwarp_multisect(ar, br, k, wl < 16 ? 1 : k, lo, hi2);
            const double r = 0.5 * (lo + hi2);
            double y[kLanczosWarm];
            tridiag_vec_reg(ar, br, k, r, y);
            if ((wl & 15) == 0) {
                double* dst = wl == 0 ? S.ymin : S.ymax;
#pragma unroll
                for (int i = 0; i < kLanczosWarm; ++i)
                    if (i < k) dst[i] = y[i];
                S.rr[wl >> 4] = r;
            }
        } else if (wi == 0) {
            double lo = S.alpha[0], hi2 = S.alpha[0];
            for (int i = 0; i < k; ++i) {
                const double rad = (i > 0 ? fabs(S.beta[i - 1]) : 0.0) + (i < k - 1 ? fabs(S.beta[i]) : 0.0);
                lo = dmin_(lo, S.alpha[i] - rad);
                hi2 = dmax_(hi2, S.alpha[i] + rad);
            }
            // lanes 0-15 of the first warp bracket the smallest eigenvalue,
            // lanes 16-31 the largest
            double l2 = lo, h2 = hi2;
            halfwarp_bisect(S.alpha, S.beta, k, wl < 16 ? 1 : k, l2, h2);
            const double r = 0.5 * (l2 + h2);
            const double r0 = __shfl_sync(kFull, r, 0);
            const double r1 = __shfl_sync(kFull, r, 16);
            if (wl == 0 || wl == 16) {
                const bool lo_end = wl == 0;
                wk_tridiag_vec(S.alpha, S.beta, k, lo_end ? r0 : r1, lo_end ? S.ymin : S.ymax,
                               lo_end ? S.s3 : S.s3 + 32, lo_end ? S.s4 : S.s4 + 32);
            }
            if (wl == 0) {
                S.rr[0] = r0;
                S.rr[1] = r1;
            }
        }
        sync();
        rmin = S.rr[0];
        rmax = S.rr[1];
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) vmin[q][d] = vmax[q][d] = 0.0;
        for (int j = 0; j < k; ++j) {
            double vj[Q][3];
            load(basis(j, m), vj);
            const double y1 = S.ymin[j], y2 = S.ymax[j];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    vmin[q][d] += y1 * vj[q][d];
                    vmax[q][d] += y2 * vj[q][d];
                }
        }
        sync();
        return k;
    }

    // spectral_bounds (src/hydrodynamics.cpp:224-264): the warm-start vector
    // lives in the chain's cache slice.
    // The step's three mutually independent products against D(R) run in
    // one pass first: D v0 (the Lanczos start vector), D X0 (the noise, for
    // the Chebyshev series) and D A (A = Fs + Fe, the predictor's force).
    // fuse: also form DX0 = D X0 and DA = D A in the start vector's pass;
    // otherwise the caller has them and the Lanczos forms D v0 itself.
    __device__ void bounds(double* cache, int& cache_valid, double& lmin, double& lmax, const float (&X0)[Q][3],
                           const float (&A)[Q][3], float (&DX0)[Q][3], float (&DA)[Q][3], bool fuse = true) {
        double vmin[Q][3], vmax[Q][3], rmin, rmax;
        const bool can_warm = cache_valid != 0;
        double v0[Q][3], dv0[Q][3];
        start_vector(can_warm, cache, v0);
        if (fuse) {
            float x3[3][Q][3], y3[3][Q][3];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    x3[0][q][d] = (float)v0[q][d];
                    x3[1][q][d] = X0[q][d];
                    x3[2][q][d] = A[q][d];
                }
            applyK<3>(x3, y3);
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    dv0[q][d] = (double)y3[0][q][d];
                    DX0[q][d] = y3[1][q][d];
                    DA[q][d] = y3[2][q][d];
                }
        }
        const int steps =
            lanczos(can_warm ? kLanczosWarm : kLanczosCold, can_warm, v0, dv0, fuse, vmin, vmax, rmin, rmax);
        if (can_warm && steps < 4) {
            start_vector(false, cache, v0);
            lanczos(kLanczosCold, false, v0, dv0, false, vmin, vmax, rmin, rmax);
            cnt[C_LZCOLD] += 1;
        } else {
            cnt[can_warm ? C_LZWARM : C_LZCOLD] += 1;
        }
        double s[Q][3], u[Q][3];
        load(a.seed_table, u);
        const double iun = 1.0 / ch.seed_norm;
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) s[q][d] = vmin[q][d] + vmax[q][d] + 0.01 * u[q][d] * iun;
        const double sn = sqrt(dot(s, s));
        if (sn > 0.0 && isfinite(sn)) {
            const double is = 1.0 / sn;
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) s[q][d] *= is;
            store(cache, s);
            cache_valid = 1;
        } else {
            cache_valid = 0;
        }
        lmin = 0.5 * rmin;
        lmax = 1.02 * rmax;
        if (lmin < 1.0e-12) lmin = 1.0e-12;
        if (lmin >= lmax) lmin = lmax * 1.0e-6;
    }

    // ---- Chebyshev square root, FP32 recurrence (src/hydrodynamics.cpp:267-337)
    // Returns the FD error; out = approx D^{1/2} x0.
    // Dx0 = D x0 (computed by the caller). grow: the FD growth loop of the
    // reference; without it a failed check returns at once (bounds kept from
    // an earlier step are refreshed first).
    __device__ double chebyshev(const float (&x0)[Q][3], const float (&Dx0)[Q][3], double lmin, double lmax,
                                float (&out)[Q][3], bool grow = true) {
        const double x0Dx0 = dotf(x0, Dx0);
        double Lr = sqrt(lmax / lmin) * ch.mult + 0.5;
        int L = !(Lr < 2.0e9) ? kMaxCheb : (int)Lr + 1;
        L = L > kMaxCheb ? kMaxCheb : (L < 2 ? 2 : L);
        const float da = (float)(2.0 / (lmax - lmin));
        const float db = (float)(-(lmax + lmin) / (lmax - lmin));
        double fd = 0.0;
        for (;;) {
            const float inv = 1.f / (float)(L + 1);
            const float ida = 1.f / da;
            for (int k = tid; k <= L; k += TT) {
                const float xk = (cospif(((float)k + 0.5f) * inv) - db) * ida;
                sqx[k] = sqrtf(xk);
            }
            sync();
            for (int j = tid; j <= L; j += TT) {
                float s = 0.f;
                for (int k = 0; k <= L; ++k) s += sqx[k] * cospif((float)j * ((float)k + 0.5f) * inv);
                s *= 2.f * inv;
                if (j == 0) s *= 0.5f;
                coef[j] = s;
            }
            sync();
            float tp[Q][3], tc[Q][3], o[Q][3];
            const float c0 = coef[0], c1 = coef[1];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    tp[q][d] = x0[q][d];
                    tc[q][d] = da * Dx0[q][d] + db * tp[q][d];
                    o[q][d] = c0 * tp[q][d] + c1 * tc[q][d];
                }
            for (int l = 2; l <= L; ++l) {
                float Dv[Q][3];
                apply32(tc, Dv);
                const float cl = coef[l];
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const float tn = 2.f * (da * Dv[q][d] + db * tc[q][d]) - tp[q][d];
                        tp[q][d] = tc[q][d];
                        tc[q][d] = tn;
                        o[q][d] += cl * tn;
                    }
            }
            cnt[C_CHEB] += L;
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) out[q][d] = valid(q) ? o[q][d] : 0.f;
            const double rr = dotf(out, out);
            fd = fabs(rr - x0Dx0) / x0Dx0;
            sync();
            if (fd <= ch.fd_tol || L >= kMaxCheb || !grow) break;
            const int grow = L / 4 > 1 ? L / 4 : 1;
            L = (L + grow) > kMaxCheb ? kMaxCheb : L + grow;
        }
        return fd;
    }

    // ---- Cholesky fallback (src/mobility.cpp:69-81): dense FP64 D in global
    // scratch, right-looking factor, L x0. Returns false if not PD.
    __device__ bool cholesky_noise(const double (&R)[Q][3], const float (&x0)[Q][3], float (&out)[Q][3]) {
        to_smem(S.s0, R);
        sync();
        double* L = Lt;
        for (int idx = tid; idx < 9 * N; idx += TT) {
            const int mu = idx / 9, i = (idx % 9) / 3, j = idx % 3;
            L[(int64_t)(3 * mu + i) * n + 3 * mu + j] = (i == j) ? 1.0 : 0.0;
        }
        const int npairs = N * (N - 1) / 2;
        for (int pidx = tid; pidx < npairs; pidx += TT) {
            int nu = (int)((1.0 + sqrt(1.0 + 8.0 * (double)pidx)) * 0.5);
            while (nu * (nu - 1) / 2 > pidx) --nu;
            while ((nu + 1) * nu / 2 <= pidx) ++nu;
            const int mu = pidx - nu * (nu - 1) / 2;
            double b[3];
            for (int d = 0; d < 3; ++d) b[d] = S.s0[3 * nu + d] - S.s0[3 * mu + d];
            double om1, om2;
            rpy_weights(ch.hstar, b[0] * b[0] + b[1] * b[1] + b[2] * b[2], om1, om2);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double val = om2 * b[i] * b[j] + (i == j ? om1 : 0.0);
                    L[(int64_t)(3 * mu + i) * n + 3 * nu + j] = val;
                    L[(int64_t)(3 * nu + j) * n + 3 * mu + i] = val;
                }
        }
        __threadfence_block();
        sync();
        for (int k = 0; k < n; ++k) {
            const double s = L[(int64_t)k * n + k];
            if (!(s > 0.0)) return false;
            const double dk = sqrt(s);
            sync();
            if (tid == 0) L[(int64_t)k * n + k] = dk;
            const double idk = 1.0 / dk;
            for (int i = k + 1 + tid; i < n; i += TT) L[(int64_t)k * n + i] *= idk;
            __threadfence_block();
            sync();
            const double* colk = L + (int64_t)k * n;
            for (int j = k + 1; j < n; ++j) {
                const double ljk = colk[j];
                for (int i = j + tid; i < n; i += TT) L[(int64_t)j * n + i] -= colk[i] * ljk;
            }
            __threadfence_block();
            sync();
        }
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (valid(q))
#pragma unroll
                for (int d = 0; d < 3; ++d) S.s1[3 * bead(q) + d] = (double)x0[q][d];
        sync();
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const int i = 3 * bead(q) + d;
                double s = 0.0;
                if (valid(q))
                    for (int j = 0; j <= i; ++j) s += L[(int64_t)j * n + i] * S.s1[j];
                out[q][d] = (float)s;
            }
        sync();
        return true;
    }
};

// -------------------------------------------------------------- the kernel

template <int T, int Q>
__global__ void __launch_bounds__(TeamCfg<T, Q>::kCtaThreads, TeamCfg<T, Q>::kMinBlocks)
    integrate_team_kernel(const RunArgs a) {
    extern __shared__ __align__(16) unsigned char wsm[];
    constexpr int TT = TeamCfg<T, Q>::kThreads;
    const int team = threadIdx.x / TT;
    const int tid = threadIdx.x % TT;
    const int64_t stride = team_area_stride<T, Q>(a.n_max);
    TeamShared<T, Q>& S = *reinterpret_cast<TeamShared<T, Q>*>(wsm + stride * team);
    double* Vs = reinterpret_cast<double*>(wsm + stride * team + (sizeof(TeamShared<T, Q>) + 15) / 16 * 16);
    const int64_t gw = (int64_t)blockIdx.x * TeamCfg<T, Q>::kTeamsPerCta + team;
    double* scr = a.scratch + gw * a.scratch_stride;
    const int nvr = (int)round_up8(a.n_max);
    const uint64_t t_launch = global_ns();

    for (;;) {
        if (tid == 0) {
            const int item = atomicAdd(a.work_counter, 1);
            S.item = item >= a.n_work ? -1 : (a.order ? a.order[item] : item);
        }
        team_sync<T>(team);
        const int c = S.item;
        if (c < 0) break;
        {
            const int nw = (int)(sizeof(DevChain) / 8);
            const double* src = reinterpret_cast<const double*>(a.chains + c);
            double* dst = reinterpret_cast<double*>(&S.ch);
            for (int i = tid; i < nw; i += TT) dst[i] = src[i];
        }
        team_sync<T>(team);
        const DevChain& ch = S.ch;
        int status = a.status[c];
        if ((status & BDCU_ST_FATAL_MASK) || ch.bad_param) {
            if (tid == 0 && ch.bad_param) a.status[c] = status | BDCU_ST_BAD_PARAM;
            team_sync<T>(team);
            continue;
        }
        TeamChain<T, Q> W(a, S, ch);
        W.V = Vs;
        W.sqx = reinterpret_cast<float*>(Vs);
        W.coef = reinterpret_cast<float*>(Vs) + kCoefCap;
        W.Vg = scr;
        W.Lt = scr + (int64_t)kLanczosCold * nvr;
        W.nv = nvr;
        W.tid = tid;
        W.wl = tid & 31;
        W.wi = tid >> 5;
        W.team = team;
        W.N = ch.N;
        W.n = 3 * ch.N;
        W.hi = ch.hstar > 0.0;
        W.status = status;
        for (int k = 0; k < 8; ++k) W.cnt[k] = 0;
        {
            const double RPI = 1.7724538509055160, TPI = 6.283185307179586;
            const double K1 = RPI * 0.75;
            W.scale = ch.hstar > 0.0 ? (float)ch.hstar : 1.f;
            W.iscale = 1.f / W.scale;
            W.K1 = (float)K1;
            W.K2 = (float)(K1 * (TPI / 3.0));
            W.K3 = (float)(K1 * TPI);
            W.C3 = (float)(0.75 / RPI * 0.375);
            W.C7 = (float)(0.09375 / RPI);
        }
        const int N = W.N;
        double* gR = a.R + 3 * ch.bead_off;
        double* gcache = a.cache + 3 * ch.bead_off;
        int cache_valid = (a.cache_mode == BDCU_CACHE_PERSIST) ? a.cache_valid[c] : 0;
        uint32_t ux = (uint32_t)a.rng[3 * c];
        int32_t iy = a.rng[3 * c + 1], seed = a.rng[3 * c + 2];
        double R[Q][3];
        W.load(gR, R);
        const int nsteps = a.n_steps[c];
        double t = a.t_start[c];
        const double dt = ch.dt;
        const double sqrt2inv = 1.0 / sqrt(2.0);
        const double sqrt_dt = sqrt(dt);
        // spectral bounds kept between refreshes (a launch starts with a refresh)
        const int bounds_every = a.bounds_every > 1 ? a.bounds_every : 1;
        int since_bounds = bounds_every;
        double lmin = 0.0, lmax = 0.0;
        int step = 0;
        for (; step < nsteps; ++step) {
            // time slice: no new step past the budget (thread 0 decides for the team)
            if (a.budget_ns > 0 && W.tor(tid == 0 && (int64_t)(global_ns() - t_launch) >= a.budget_ns)) break;
            // recenter (src/integrator.cpp:88-93)
            if (ch.update_com) {
                double com[3];
                for (int d = 0; d < 3; ++d) {
                    double s = 0.0;
#pragma unroll
                    for (int q = 0; q < Q; ++q) s += R[q][d];
                    com[d] = (1.0 / N) * W.tsum(s);
                }
#pragma unroll
                for (int q = 0; q < Q; ++q)
                    if (W.valid(q))
                        for (int d = 0; d < 3; ++d) R[q][d] -= com[d];
            }
            W.stage_pos(R);
            float Fs[Q][3], Fe[Q][3];
            W.forces(R, t, Fs, Fe, true);
            float X0[Q][3], dW[Q][3], A[Q][3], DF[Q][3];
            W.noise(ux, iy, seed, X0);
            // brownian_step (src/mobility.cpp:58-88)
            if (!W.hi) {
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) dW[q][d] = (float)(sqrt_dt * X0[q][d]);
            } else {
                float bx[Q][3], DX0[Q][3];
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) A[q][d] = Fs[q][d] + Fe[q][d];
                double fd;
                if (since_bounds >= bounds_every) {
                    W.bounds(gcache, cache_valid, lmin, lmax, X0, A, DX0, DF);
                    since_bounds = 0;
                    fd = W.chebyshev(X0, DX0, lmin, lmax, bx);
                } else {
                    // bounds kept from an earlier step: the two products in one pass
                    float x2[2][Q][3], y2[2][Q][3];
#pragma unroll
                    for (int q = 0; q < Q; ++q)
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            x2[0][q][d] = X0[q][d];
                            x2[1][q][d] = A[q][d];
                        }
                    W.template applyK<2>(x2, y2);
#pragma unroll
                    for (int q = 0; q < Q; ++q)
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            DX0[q][d] = y2[0][q][d];
                            DF[q][d] = y2[1][q][d];
                        }
                    fd = W.chebyshev(X0, DX0, lmin, lmax, bx, false);
                    if (!(fd <= ch.fd_tol)) {  // the kept bounds no longer hold: refresh and redo
                        W.bounds(gcache, cache_valid, lmin, lmax, X0, A, DX0, DF, false);
                        since_bounds = 0;
                        fd = W.chebyshev(X0, DX0, lmin, lmax, bx);
                    }
                }
                ++since_bounds;
                if (!(fd <= ch.fd_tol)) {
                    W.status |= BDCU_ST_CHEB_FALLBACK;
                    W.cnt[C_FALLBACK] += 1;
                    if (!W.cholesky_noise(R, X0, bx)) {
                        W.status |= BDCU_ST_NOT_PD;
                        break;
                    }
                }
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) dW[q][d] = (float)(sqrt_dt * bx[q][d]);
            }
            // predictor (src/integrator.cpp:96-101)
            double K1[9], K2[9];
            kappa_at(ch, a.arena, t, K1);
            kappa_at(ch, a.arena, t + dt, K2);
            double Rp[Q][3];
            if (!W.hi)  // without HI D = I; with HI, bounds() formed D (Fs + Fe)
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) DF[q][d] = Fs[q][d] + Fe[q][d];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const double fl1 = K1[3 * r] * R[q][0] + K1[3 * r + 1] * R[q][1] + K1[3 * r + 2] * R[q][2];
                    Rp[q][r] = W.valid(q) ? R[q][r] + dt * (fl1 + 0.25 * DF[q][r]) + sqrt2inv * dW[q][r] : 0.0;
                }
            // upsilon (src/integrator.cpp:107-119): forces at R~ with R~'s coordinates staged
            W.stage_pos(Rp);
            float Fep[Q][3], dummy[Q][3];
            W.forces(Rp, t + dt, dummy, Fep, false);
            // D Fs + D (Fe + Fe~) = D (Fs + Fe) + D Fe~: the predictor's
            // product plus one more (the reference forms both sums anew)
            W.stage_pos(R);
            // solve_connectors (src/integrator.cpp:125-165): thread owns bonds
            // bead(0), bead(1). Its first iteration's bonds are those of R~,
            // so that iteration's product D Fb is formed in one pass with
            // upsilon's D Fe~.
            W.to_smem(S.s1, Rp);
            team_sync<T>(team);
            double bond[Q][3];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int b = W.bead(q);
#pragma unroll
                for (int d = 0; d < 3; ++d) bond[q][d] = b < N - 1 ? S.s1[3 * (b + 1) + d] - S.s1[3 * b + d] : 0.0;
            }
            const double anchor0 = S.s1[0], anchor1 = S.s1[1], anchor2 = S.s1[2];
            team_sync<T>(team);
            double Fc[Q][3];
            float Fb[Q][3], DFb[Q][3];
            // connector forces (src/spring.cpp:183-193) into s1, then the bead forces
            auto connector_and_bead_forces = [&]() {
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int b = W.bead(q);
                    const double f =
                        b < N - 1 ? connector_factor(ch, clamped_len(bond[q][0], bond[q][1], bond[q][2])) : 0.0;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        Fc[q][d] = f * bond[q][d];
                        if (b < N - 1) S.s1[3 * b + d] = Fc[q][d];
                    }
                }
                team_sync<T>(team);
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int m = W.bead(q);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        double v = 0.0;
                        if (m < N) {
                            if (m == 0) v = S.s1[d];
                            else if (m == N - 1) v = -S.s1[3 * (N - 2) + d];
                            else v = S.s1[3 * m + d] - S.s1[3 * (m - 1) + d];
                        }
                        Fb[q][d] = (float)v;
                    }
                }
                team_sync<T>(team);
            };
            connector_and_bead_forces();
            float DFep[Q][3];
            if (W.hi) {
                float x2[2][Q][3], y2[2][Q][3];
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        x2[0][q][d] = Fep[q][d];
                        x2[1][q][d] = Fb[q][d];
                    }
                W.template applyK<2>(x2, y2);
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        DFep[q][d] = y2[0][q][d];
                        DFb[q][d] = y2[1][q][d];
                    }
            } else {
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        DFep[q][d] = Fep[q][d];
                        DFb[q][d] = Fb[q][d];
                    }
            }
            double ups[Q][3];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const double fl1 = K1[3 * r] * R[q][0] + K1[3 * r + 1] * R[q][1] + K1[3 * r + 2] * R[q][2];
                    const double fl2 = K2[3 * r] * Rp[q][0] + K2[3 * r + 1] * Rp[q][1] + K2[3 * r + 2] * Rp[q][2];
                    ups[q][r] = R[q][r] + dt * (0.5 * (fl1 + fl2) + 0.125 * ((double)DF[q][r] + (double)DFep[q][r])) +
                                sqrt2inv * dW[q][r];
                }
            W.to_smem(S.s0, ups);
            team_sync<T>(team);
            double dups[Q][3];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int b = W.bead(q);
#pragma unroll
                for (int d = 0; d < 3; ++d) dups[q][d] = b < N - 1 ? S.s0[3 * (b + 1) + d] - S.s0[3 * b + d] : 0.0;
            }
            team_sync<T>(team);
            double Rprev[Q][3], Rc[Q][3];
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) Rprev[q][d] = Rp[q][d];
            const int max_iter = 100 * N;
            const double c8 = 0.125 * dt, c4 = 0.25 * dt;
            int lstat = 0;
            for (int iter = 0;; ++iter) {
                if (iter > 0) {  // (the first iteration's Fc, Fb and D Fb are formed above)
                    connector_and_bead_forces();
                    W.applyF(Fb, DFb);
                }
#pragma unroll
                for (int q = 0; q < Q; ++q)
                    if (W.valid(q))
#pragma unroll
                        for (int d = 0; d < 3; ++d) S.s2[3 * W.bead(q) + d] = (double)DFb[q][d];
                team_sync<T>(team);
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int b = W.bead(q);
                    if (b < N - 1) {
                        double g[3], qv[3];
                        for (int d = 0; d < 3; ++d)
                            g[d] = dups[q][d] + c8 * (S.s2[3 * (b + 1) + d] - S.s2[3 * b + d]) + c4 * Fc[q][d];
                        solve_connector(g, dt, ch, qv, lstat);
                        for (int d = 0; d < 3; ++d) bond[q][d] = qv[d];
                    }
                }
                // R_corr = anchor + prefix sums of the bonds: inclusive scan in
                // each warp, then the totals of the warps before it (slot 0 of
                // the whole team precedes slot 1)
                double scan[Q][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    double v[Q];
#pragma unroll
                    for (int q = 0; q < Q; ++q) v[q] = bond[q][d];
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
                        for (int q = 0; q < Q; ++q) {
                            const double tq = __shfl_up_sync(kFull, v[q], o);
                            if (W.wl >= o) v[q] += tq;
                        }
                    }
#pragma unroll
                    for (int q = 0; q < Q; ++q) scan[q][d] = v[q];
                }
                if constexpr (T == 1) {
                    if constexpr (Q == 2) {
#pragma unroll
                        for (int d = 0; d < 3; ++d) scan[1][d] += __shfl_sync(kFull, scan[0][d], 31);
                    }
                    __syncwarp();
                } else {
                    if (W.wl == 31)
#pragma unroll
                        for (int q = 0; q < Q; ++q)
#pragma unroll
                            for (int d = 0; d < 3; ++d) S.tot[(q * 3 + d) * T + W.wi] = scan[q][d];
                    team_sync<T>(team);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        double off0 = 0.0, all0 = 0.0, off1 = 0.0;
#pragma unroll
                        for (int w = 0; w < T; ++w) {
                            const double t0 = S.tot[d * T + w];
                            const double t1 = Q == 2 ? S.tot[(3 + d) * T + w] : 0.0;
                            if (w < W.wi) {
                                off0 += t0;
                                off1 += t1;
                            }
                            all0 += t0;
                        }
                        scan[0][d] += off0;
                        if constexpr (Q == 2) scan[1][d] += all0 + off1;
                    }
                }
                team_sync<T>(team);
                if (tid == 0) {
                    S.s1[0] = anchor0;
                    S.s1[1] = anchor1;
                    S.s1[2] = anchor2;
                }
                const double an[3] = {anchor0, anchor1, anchor2};
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int b = W.bead(q);
                    if (b < N - 1)
                        for (int d = 0; d < 3; ++d) S.s1[3 * (b + 1) + d] = an[d] + scan[q][d];
                }
                team_sync<T>(team);
                W.load(S.s1, Rc);
                team_sync<T>(team);
                double s = 0.0;
#pragma unroll
                for (int q = 0; q < Q; ++q)
                    if (W.valid(q)) {
                        const double e0 = Rc[q][0] - Rprev[q][0], e1 = Rc[q][1] - Rprev[q][1],
                                     e2 = Rc[q][2] - Rprev[q][2];
                        s += e0 * e0 + e1 * e1 + e2 * e2;
                    }
                const double incr = sqrt(W.tsum(s)) / N;
                W.cnt[C_CORR] += 1;
                if (incr < ch.tol) break;
                if (!(incr == incr) || isinf(incr)) {
                    W.status |= BDCU_ST_NONFINITE;
                    break;
                }
                if (iter >= max_iter) {
                    W.status |= BDCU_ST_NONCONVERGED;
                    W.cnt[C_NONCONV] += 1;
                    break;
                }
#pragma unroll
                for (int q = 0; q < Q; ++q)
#pragma unroll
                    for (int d = 0; d < 3; ++d) Rprev[q][d] = Rc[q][d];
            }
            // every thread's connector status, then a team-uniform fatal test
            W.status |= W.tor(lstat);
            if (W.status & BDCU_ST_FATAL_MASK) break;
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) R[q][d] = Rc[q][d];
            W.cnt[C_STEPS] += 1;
            t += dt;
        }
        if (!(W.status & BDCU_ST_FATAL_MASK)) W.store(gR, R);
        if (tid == 0) {
            a.rng[3 * c] = (int32_t)ux;
            a.rng[3 * c + 1] = iy;
            a.rng[3 * c + 2] = seed;
            a.cache_valid[c] = cache_valid;
            a.status[c] = W.status;
            int64_t* cc = reinterpret_cast<int64_t*>(a.counters + c);
            for (int k = 0; k < 8; ++k) cc[k] += (int64_t)W.cnt[k];
            if (a.steps_done) a.steps_done[c] = step;
            if (a.t_end) a.t_end[c] = t;
        }
        team_sync<T>(team);
    }
}

}  // namespace bdcu
