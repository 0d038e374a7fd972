// integrator.cuh -- the ChainIntegrator step loop as one persistent sm_100a
// kernel: one chain per thread block, chains claimed from a device work queue,
// chain state resident in shared memory for all steps of a call.
//
// FORM == BDCU_FORM_PLAIN_FP64: the reference algorithm in FP64. The dense RPY
//   tensor D lives in shared memory (global scratch when 3N is too large);
//   D.x is a row-sequential sum per thread, EV forces are accumulated per bead
//   in the reference's pair order, Cholesky is right-looking with the
//   reference's per-element subtraction order. Only block dot products
//   (Lanczos, FD check) use a tree order.
// FORM == BDCU_FORM_MIXED_FP32: D.x recomputed pairwise in FP32 from
//   shared-memory bead coordinates (no stored D), FP32 excluded volume; FP64
//   positions, connector solve, Lanczos bounds and Cholesky.
//
// Reference: src/integrator.cpp:61-170 of the bdsim project and the physics
// it calls (cited per function).
#pragma once

#include <stdint.h>

#include "bdcu_internal.h"
#include "device_physics.cuh"

namespace bdcu {

constexpr int kSlots = 16;     // n-vectors in shared memory
constexpr int kCoefCap = 504;  // >= kMaxCheb + 1
// Blocked Cholesky (3N >= kBlockedCholMin): column blocks of up to
// kCholMaxBlock columns, each factored as sub-panels of up to kCholMaxPanel
// columns (rows solved with the sub-panel in registers); trailing updates in
// kCholTile x kCholTile tiles whose panel rows are staged in shared memory
// with row stride kCholTileStride (padded against bank conflicts), in vector
// slots kCholFirstSlot.. (free while D is factored).
constexpr int kBlockedCholMin = 300;
constexpr int kCholTile = 64;
constexpr int kCholTileStride = kCholTile + 4;
constexpr int kCholMaxPanel = 32;
constexpr int kCholMaxBlock = 64;
constexpr int kCholFirstSlot = 7;

// Block-shared control state.
struct Ctl {
    double com[3];
    double lmin, lmax, x0Dx0, fd_err, incr, rmin, rmax, glo, ghi, nv, bval;
    int32_t chain, k, L, status, cache_valid, lz_steps, brk, stop;
    int64_t cnt[8];  // bdcu_counters order
};
enum { C_STEPS = 0, C_DX, C_CHEB, C_CORR, C_LZCOLD, C_LZWARM, C_FALLBACK, C_NONCONV };

struct SmemLayout {
    int64_t ctl, chain, red, alpha, beta, ymin, ymax, coef, sqx, slots, V, D, f32, total;  // in doubles
};

__host__ __device__ inline int64_t round_up8(int64_t x) { return (x + 7) / 8 * 8; }

// Shared-memory layout (in doubles) for a launch whose largest chain has
// 3N = n_max. Host and device compute it with the same function.
__host__ __device__ inline SmemLayout smem_layout(int n_max, int d_in_smem, int v_cap, int mixed) {
    SmemLayout s;
    int64_t o = 0;
    s.ctl = o;   o += round_up8((int64_t)(sizeof(Ctl) + 7) / 8);
    s.chain = o; o += round_up8((int64_t)(sizeof(DevChain) + 7) / 8);
    s.red = o;   o += 32;
    s.alpha = o; o += 32;
    s.beta = o;  o += 32;
    s.ymin = o;  o += 32;
    s.ymax = o;  o += 32;
    s.coef = o;  o += kCoefCap;
    s.sqx = o;   o += kCoefCap;
    const int64_t nv = round_up8(n_max);
    s.slots = o; o += (int64_t)kSlots * nv;
    s.V = o;     o += (int64_t)v_cap * nv;
    s.D = o;     if (d_in_smem) o += (int64_t)n_max * n_max;
    s.f32 = o;   if (mixed) o += 2 * nv;  // float4 bead coordinates + float4 staged vector (N <= n/3 each)
    s.total = o;
    return s;
}

// Leading dimension of the Cholesky factor Lt (column k of L at Lt + k*ld):
// n rounded up to 16 doubles, so that every column, and every 64-row segment
// of it starting at a multiple of 8 rows, begins on a 128-byte line (the
// bulk copies of the blocked factorisation need 16-byte alignment).
__host__ __device__ inline int chol_ld(int n) { return (n + 15) / 16 * 16; }

// Global scratch per thread block (doubles): dense D when it is not in shared
// memory (plain form), the Cholesky factor, and the cold Lanczos basis.
struct ScratchLayout {
    int64_t D, Lt, V, total;
};
__host__ __device__ inline ScratchLayout scratch_layout(int n_max, int d_in_smem, int v_cap, int need_chol,
                                                        int mixed, int need_d, int need_lz) {
    // every region a whole number of 128-byte lines (16 doubles), so that a
    // block's D and factor start on a line of their own (discard.global.L2)
    ScratchLayout s;
    int64_t o = 0;
    const int64_t nn = (int64_t)n_max * n_max, nn16 = (nn + 15) / 16 * 16;
    s.D = o;  if (!mixed && need_d && !d_in_smem) o += nn16;
    s.Lt = o; if (need_chol) o += (int64_t)n_max * chol_ld(n_max);
    s.V = o;  if (need_lz && v_cap < kLanczosCold) o += ((int64_t)kLanczosCold * round_up8(n_max) + 15) / 16 * 16;
    s.total = o;
    return s;
}

// ---------------------------------------------------------------- helpers

__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Dot product over the block, same value returned to every thread, in one
// fixed order whatever the block size (so a chain's result does not depend on
// the launch shape its bucket was given): 64 partial sums, partial v adding
// a[i]*b[i] for i = v, v+64, ... in order, then a butterfly within each half
// and the two halves added. Not the reference's sequential order; the
// difference is at the last bit of each sum. Needs blockDim.x >= 64.
static __device__ double block_dot(const double* a, const double* b, int n, double* red) {
    double s = 0.0;
    if (threadIdx.x < 64)
        for (int i = threadIdx.x; i < n; i += 64) s += a[i] * b[i];
    __syncthreads();
    if (threadIdx.x < 64) {
        s = warp_allsum(s);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    }
    __syncthreads();
    return red[0] + red[1];
}

// y_r = D x_r for K vectors in one read of D: one row per thread, each
// product summed over j in order exactly as matvec does
// (src/linalg.cpp:81-89), so every y_r equals its own single product bit for
// bit. The plain form reads D (L2-resident) once for the step's K mutually
// independent products instead of K times.
template <int K>
__device__ __forceinline__ void matvec_dense_k(const double* __restrict__ D, int ld, const double* const (&x)[K],
                                               double* const (&y)[K], int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s[K];
#pragma unroll
        for (int r = 0; r < K; ++r) s[r] = 0.0;
        const double* col = D + i;
#pragma unroll 8
        for (int j = 0; j < n; ++j) {
            const double d = col[(int64_t)j * ld];
#pragma unroll
            for (int r = 0; r < K; ++r) s[r] += d * x[r][j];
        }
#pragma unroll
        for (int r = 0; r < K; ++r) y[r][i] = s[r];
    }
}

// Drop the L2 lines of [p, p + doubles) without writing them back: the dense
// D (and a factor) are rebuilt every step, so after a step's last read the
// data is dead. p must start a 128-byte line and the range must end at the
// end of its allocation's last line (scratch_layout rounds every region to
// whole lines); a misaligned p is left alone.
__device__ __forceinline__ void discard_l2(const double* p, int64_t doubles) {
    if ((reinterpret_cast<uintptr_t>(p) & 127) != 0) return;
    const int64_t lines = (doubles * 8 + 127) / 128;
    const char* base = reinterpret_cast<const char*>(p);
    for (int64_t l = threadIdx.x; l < lines; l += blockDim.x)
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(base + 128 * l) : "memory");
}

// y = D x, one row per thread, summed over j in order (matvec,
// src/linalg.cpp:81-89). D is exactly symmetric (rpy_diffusion_matrix writes
// both halves from one value), so row i is read as column i for coalescing.
__device__ __forceinline__ void matvec_dense(const double* __restrict__ D, int ld, const double* __restrict__ x,
                                             double* __restrict__ y, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        const double* col = D + i;
#pragma unroll 16  // (16 loads of D in flight per row: +4.5% on the plain form over 8; 32 was slower)
        for (int j = 0; j < n; ++j) s += col[(int64_t)j * ld] * x[j];
        y[i] = s;
    }
}

// sturm_count (src/hydrodynamics.cpp:91-104)
__device__ __forceinline__ int sturm_count(const double* a, const double* b, int m, double x) {
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

// The 100-step bisection of lanczos_extremes (src/hydrodynamics.cpp:196-207),
//   mid = 0.5*(lo+hi); if (sturm(mid) >= target) hi = mid; else lo = mid;
// evaluated five levels at a time by one warp: lane l owns node l of a
// depth-5 decision tree, replays the midpoints on its path with the same
// arithmetic, and evaluates its own Sturm count; the warp then walks the
// resolved path. A round that leaves (lo, hi) unchanged has reached the fixed
// point of the iteration, so the remaining rounds are skipped. The result is
// the sequential algorithm's, bit for bit.
static __device__ void warp_bisect(const double* al, const double* bb, int k, int target, double& lo, double& hi) {
    const int lane = threadIdx.x & 31;
    const int lvl = 31 - __clz(lane + 1);
    const int p = lane + 1 - (1 << lvl);
    for (int it = 0; it < 100; it += 5) {
        int dec = 0;
        if (lane < 31) {
            double a = lo, b = hi;
            for (int l = 0; l < lvl; ++l) {
                const int bit = (p >> (lvl - 1 - l)) & 1;
                const double m = 0.5 * (a + b);
                if (bit == 0) b = m; else a = m;
            }
            const double mid = 0.5 * (a + b);
            dec = (sturm_count(al, bb, k, mid) >= target) ? 0 : 1;
        }
        int node = 0;
        double na = lo, nb = hi;
#pragma unroll
        for (int l = 0; l < 5; ++l) {
            const int d = __shfl_sync(0xffffffffu, dec, node);
            const double m = 0.5 * (na + nb);
            if (d == 0) nb = m; else na = m;
            node = 2 * node + 1 + d;
        }
        const bool same = (na == lo && nb == hi);
        lo = na;
        hi = nb;
        if (same) break;
    }
}

// tridiag_eigenvector (src/hydrodynamics.cpp:106-136), one thread.
static __device__ void tridiag_eigenvector(const double* a, const double* b, int m, double lambda, double* y) {
    const double scale = dmax_(fabs(lambda), 1.0);
    const double shift = lambda - 1.0e-7 * scale;
    double c[kLanczosCold], d[kLanczosCold];
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

// --------------------------------------------------------- the block state

template <int FORM>
struct Block {
    static constexpr bool kMixed = (FORM == BDCU_FORM_MIXED_FP32);
    const RunArgs& a;
    Ctl& ctl;
    const DevChain& ch;
    double* red;
    double* alpha;
    double* beta;
    double* ymin;
    double* ymax;
    double* coef;
    double* sqx;
    double* slot[kSlots];
    double* Vs;        // shared Lanczos basis (v_cap vectors)
    double* Vg;        // global Lanczos basis (kLanczosCold vectors)
    double* D;         // plain: dense D (shared or global)
    int ldd;
    double* Lt;        // transposed Cholesky factor, global scratch (leading dimension ldl)
    int ldl;           // chol_ld(n)
    double* stage;     // blocked Cholesky tile staging (vector slots kCholFirstSlot..)
    int64_t stage_cap; // doubles available at stage
    float4* pos32;     // mixed: FP32 bead coordinates
    float4* vec32;     // mixed: FP32 staged vector
    int ldv;           // stride of Lanczos basis vectors
    int N, n;
    bool hi;

    __device__ Block(const RunArgs& a_, Ctl& c_, const DevChain& ch_) : a(a_), ctl(c_), ch(ch_) {}

    __device__ __forceinline__ void sync() { __syncthreads(); }

    __device__ __forceinline__ void count(int which, int64_t v) {
        if (threadIdx.x == 0) ctl.cnt[which] += v;
    }

    // ---- D.x (Diffusion::apply, src/mobility.cpp:53-56) -----------------
    // Caller syncs before (x ready) and after (y ready). Identity => copy.
    __device__ void apply_D(const double* x, double* y) {
        if (!hi) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = x[i];
            return;
        }
        count(C_DX, 1);
        if constexpr (!kMixed) {
            matvec_dense(D, ldd, x, y, n);
        } else {
            apply_D_pairwise(x, y);
        }
    }

    // K products against D at once (K = 1..4): the plain form reads D once,
    // the mixed form runs its matrix-free products one after another. Caller
    // syncs before and after, as for apply_D.
    template <int K>
    __device__ void apply_D_multi(const double* const (&x)[K], double* const (&y)[K]) {
        if (!hi) {
#pragma unroll
            for (int r = 0; r < K; ++r)
                for (int i = threadIdx.x; i < n; i += blockDim.x) y[r][i] = x[r][i];
            return;
        }
        if constexpr (!kMixed) {
            count(C_DX, K);
            matvec_dense_k<K>(D, ldd, x, y, n);
        } else {
#pragma unroll
            for (int r = 0; r < K; ++r) {
                if (r > 0) __syncthreads();
                apply_D(x[r], y[r]);
            }
        }
    }
    // the same with the count of products known only at run time (1 + extra)
    __device__ void apply_D_n(int k, const double* const* x, double* const* y) {
        switch (k) {
            case 1: { const double* const xs[1] = {x[0]}; double* const ys[1] = {y[0]}; apply_D_multi<1>(xs, ys); break; }
            case 2: { const double* const xs[2] = {x[0], x[1]}; double* const ys[2] = {y[0], y[1]};
                      apply_D_multi<2>(xs, ys); break; }
            case 3: { const double* const xs[3] = {x[0], x[1], x[2]}; double* const ys[3] = {y[0], y[1], y[2]};
                      apply_D_multi<3>(xs, ys); break; }
            default: { const double* const xs[4] = {x[0], x[1], x[2], x[3]};
                       double* const ys[4] = {y[0], y[1], y[2], y[3]}; apply_D_multi<4>(xs, ys); break; }
        }
    }

    // Matrix-free FP32 D.x: y_b = x_b + sum_{j != b} (om1 x_j + om2 (d.x_j) d),
    // d = R_j - R_b, with omega from the RPY formula (src/hydrodynamics.cpp:36-43).
    __device__ void apply_D_pairwise(const double* x, double* y) {
        for (int b = threadIdx.x; b < N; b += blockDim.x)
            vec32[b] = make_float4((float)x[3 * b], (float)x[3 * b + 1], (float)x[3 * b + 2], 0.f);
        __syncthreads();
        const float hs = (float)ch.hstar;
        const float RPI = 1.7724538509055160f, TRPI = 2.f * RPI, TPI = 6.283185307179586f;
        const float C1 = TPI / 3.f, C3 = 0.75f / RPI * 0.375f, C7 = 0.09375f / RPI, RPI3by4 = RPI * 0.75f;
        for (int b = threadIdx.x; b < N; b += blockDim.x) {
            const float4 rb = pos32[b];
            const float4 xb = vec32[b];
            float a0 = xb.x, a1 = xb.y, a2 = xb.z;
            for (int j = 0; j < N; ++j) {
                if (j == b) continue;
                const float4 rj = pos32[j];
                const float4 xj = vec32[j];
                const float d0 = rj.x - rb.x, d1 = rj.y - rb.y, d2 = rj.z - rb.z;
                float sq = d0 * d0 + d1 * d1 + d2 * d2;
                sq = fmaxf(sq, 1e-12f);
                const float rinv = rsqrtf(sq);
                const float rs = sq * rinv;
                const float hsbyrs = hs * rinv, rsbyhs = rs / hs;
                const float h2 = hsbyrs * hsbyrs;
                float om1, om2;
                if (rsbyhs >= TRPI) {
                    om1 = RPI3by4 * hsbyrs * (1.f + C1 * h2);
                    om2 = RPI3by4 * hsbyrs * rinv * rinv * (1.f - TPI * h2);
                } else {
                    om1 = 1.f - C3 * rsbyhs;
                    om2 = C7 * rsbyhs * rinv * rinv;
                }
                const float dx = om2 * (d0 * xj.x + d1 * xj.y + d2 * xj.z);
                a0 += om1 * xj.x + dx * d0;
                a1 += om1 * xj.y + dx * d1;
                a2 += om1 * xj.z + dx * d2;
            }
            y[3 * b] = a0;
            y[3 * b + 1] = a1;
            y[3 * b + 2] = a2;
        }
    }

    // ---- RPY tensor (rpy_diffusion_matrix, src/hydrodynamics.cpp:12-54) --
    // Writes the dense D at ptr with leading dimension ld. For pair mu<nu the
    // value of element (3mu+i, 3nu+j) and its mirror is
    // om2*b_i*b_j + (i==j ? om1 : 0).
    __device__ void build_rpy(const double* R, double* Dp, int ld) {
        for (int idx = threadIdx.x; idx < 9 * N; idx += blockDim.x) {
            const int mu = idx / 9, i = (idx % 9) / 3, j = idx % 3;
            Dp[(int64_t)(3 * mu + i) * ld + 3 * mu + j] = (i == j) ? 1.0 : 0.0;
        }
        const int npairs = N * (N - 1) / 2;
        for (int pidx = threadIdx.x; pidx < npairs; pidx += blockDim.x) {
            int nu = (int)((1.0 + sqrt(1.0 + 8.0 * (double)pidx)) * 0.5);
            while (nu * (nu - 1) / 2 > pidx) --nu;
            while ((nu + 1) * nu / 2 <= pidx) ++nu;
            const int mu = pidx - nu * (nu - 1) / 2;
            double b[3];
            for (int d = 0; d < 3; ++d) b[d] = R[3 * nu + d] - R[3 * mu + d];
            const double sq = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
            double om1, om2;
            rpy_weights(ch.hstar, sq, om1, om2);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double val = om2 * b[i] * b[j] + (i == j ? om1 : 0.0);
                    Dp[(int64_t)(3 * mu + i) * ld + 3 * nu + j] = val;
                    Dp[(int64_t)(3 * nu + j) * ld + 3 * mu + i] = val;
                }
        }
    }

    // ---- Cholesky (cholesky_lower, src/linalg.cpp:91-107) ---------------
    // Right-looking on Lt = L^T (Lt[k*ldl + i] = L(i,k)). Element (i,j) receives
    // M(i,j) - L(i,0)L(j,0) - L(i,1)L(j,1) - ... in k order, then / L(j,j):
    // the reference's rounding sequence. Returns false on a pivot <= 0.
    // src: dense D at (Dp, ld) or, if src_in_lt, Lt already holds D's lower part.
    // From 3N = kBlockedCholMin the factorisation is blocked (cholesky_blocked);
    // vector slots kCholFirstSlot.. must then be free (the callers' are).
    __device__ bool cholesky(const double* Dp, int ld, bool src_in_lt) {
        double* L = Lt;
        if (!src_in_lt) {
            for (int j = threadIdx.x >> 5; j < n; j += blockDim.x >> 5)
                for (int i = j + (threadIdx.x & 31); i < n; i += 32) L[(int64_t)j * ldl + i] = Dp[(int64_t)i * ld + j];
        }
        __syncthreads();
        const int nb = chol_panel_width();
        if (nb > 0) return cholesky_blocked(nb);
        for (int k = 0; k < n; ++k) {
            if (threadIdx.x == 0) {
                const double s = L[(int64_t)k * ldl + k];
                if (!(s > 0.0)) ctl.brk = 1; else L[(int64_t)k * ldl + k] = sqrt(s);
            }
            __syncthreads();
            if (ctl.brk) return false;
            const double dk = L[(int64_t)k * ldl + k];
            for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) L[(int64_t)k * ldl + i] = L[(int64_t)k * ldl + i] / dk;
            __syncthreads();
            const double* colk = L + (int64_t)k * ldl;
            for (int j = k + 1 + (threadIdx.x >> 5); j < n; j += blockDim.x >> 5) {
                const double ljk = colk[j];
                for (int i = j + (threadIdx.x & 31); i < n; i += 32)
                    L[(int64_t)j * ldl + i] = L[(int64_t)j * ldl + i] - colk[i] * ljk;
            }
            __syncthreads();
        }
        return true;
    }

    // Column-block width of the blocked factorisation (0: unblocked): up to
    // kCholMaxBlock columns, a multiple of 8, such that two staged tiles of
    // panel rows fit the staging area.
    __device__ int chol_panel_width() const {
        if (n < kBlockedCholMin || stage == nullptr) return 0;
        int64_t nb = stage_cap / (2 * kCholTileStride);
        nb = nb > kCholMaxBlock ? kCholMaxBlock : nb;
        nb &= ~7;
        return nb >= 8 ? (int)nb : 0;
    }

    // Blocked right-looking Cholesky. For each column block [kb, ke) of up to
    // nb columns:
    // (1) the block is factored as sub-panels [p0, p1) of up to kCholMaxPanel
    //     columns: the sub-panel's columns (rows >= p0) first receive the
    //     products of the block's earlier columns k in [kb, p0) (trailing
    //     update restricted to columns [p0, p1)); then its diagonal block is
    //     factored in shared memory column by column (pivot, scale, update
    //     of the remaining columns) and each row below it is solved by one
    //     thread, its sub-panel entries in registers: L(i,j) = (A(i,j) -
    //     sum_{k<j} L(i,k) L(j,k)) / L(j,j) for j = p0, p0+1, ... in order;
    // (2) the trailing lower triangle [ke, n)^2 is updated by the block,
    //     C(i,j) -= sum_{k in [kb,ke)} L(i,k) L(j,k), tile by tile, with the
    //     tile's panel rows staged in shared memory.
    // Every element still receives its products in k order before its
    // division, so the plain form keeps the reference's rounding sequence
    // (trailing updates one rounded product and one rounded subtraction per
    // k); the mixed form's trailing updates run on the FP64 tensor cores
    // (mma.m8n8k4, products accumulated in the tensor core's own order).
    __device__ bool cholesky_blocked(int nb) {
        for (int kb = 0; kb < n; kb += nb) {
            const int ke = kb + nb < n ? kb + nb : n;
            for (int p0 = kb; p0 < ke; p0 += kCholMaxPanel) {
                const int p1 = p0 + kCholMaxPanel < ke ? p0 + kCholMaxPanel : ke;
                if (p0 > kb) chol_update(kb, p0, p0, p0, p1);
                if (ctl.brk) return false;  // a staging wait expired
                if (!chol_panel(p0, p1)) return false;
            }
            if (ke >= n) break;
            chol_update(kb, ke, ke, ke, n);
            if (ctl.brk) return false;
        }
        return true;
    }

    // C(i,j) -= sum_{k in [k0,k1)} L(i,k) L(j,k) (k in order) for columns j in
    // [c0, c1) and rows i in [r0, n), i >= j, in kCholTile^2 tiles.
    __device__ void chol_update(int k0, int k1, int r0, int c0, int c1) {
        double* L = Lt;
        const int kk = k1 - k0, kk4 = (kk + 3) & ~3;  // staged rows k >= kk are zero
        if constexpr (kMixed)
            if ((int64_t)kStageBufs * kk4 * kCholTileStride + 8 <= stage_cap && (r0 & 7) == 0 && (c0 & 7) == 0) {
                chol_update_bulk(k0, k1, r0, c0, c1);
                return;
            }
        if constexpr (!kMixed)
            if (blockDim.x == 512 && (int64_t)3 * kk4 * kCholTile <= stage_cap) {
                chol_update_pairs(k0, k1, r0, c0, c1);
                return;
            }
        double* As = stage;                                   // As[k*TS + r] = L(i0 + r, k0 + k)
        double* Bs = stage + (int64_t)kk4 * kCholTileStride;  // Bs[k*TS + c] = L(j0 + c, k0 + k)
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
        const int nti = (n - r0 + kCholTile - 1) / kCholTile, ntj = (c1 - c0 + kCholTile - 1) / kCholTile;
        // Staging loads are issued kStageBatch at a time before their shared
        // stores, so one memory latency covers a batch instead of each element.
        // The tiles go row by row; the mixed form stages As once per tile-row
        // (a_i0) and Bs only when its column block changes (b_j0), and a
        // diagonal tile (i0 == j0) multiplies As by itself (its B rows beyond c1
        // differ from the zeros Bs would hold, but they only reach C columns >=
        // c1, which are not stored). The plain form restages both for every
        // tile: the reuse measured 2.5% slower there (5% faster in the mixed form).
        constexpr int kStageBatch = 8;
        const int tot = kk4 * kCholTile, nt = nti * ntj;
        auto next_tile = [&](int t) {  // first tile >= t not wholly above the diagonal
            while (t < nt && r0 + (t / ntj) * kCholTile + kCholTile - 1 < c0 + (t % ntj) * kCholTile) ++t;
            return t;
        };
        int a_i0 = -1, b_j0 = -1;
        for (int t = next_tile(0); t < nt; t = next_tile(t + 1)) {
            const int i0 = r0 + (t / ntj) * kCholTile, j0 = c0 + (t % ntj) * kCholTile;
            const bool diag = kMixed && i0 == j0, stA = !kMixed || i0 != a_i0, stB = !kMixed || (!diag && j0 != b_j0);
            a_i0 = i0;
            if (stB) b_j0 = j0;
            if (stA || stB) {
                for (int e0 = threadIdx.x; e0 < tot; e0 += kStageBatch * blockDim.x) {
                    double va[kStageBatch], vb[kStageBatch];
#pragma unroll
                    for (int u = 0; u < kStageBatch; ++u) {
                        const int e = e0 + u * blockDim.x, k = e / kCholTile, r = e % kCholTile;
                        const bool kin = e < tot && k < kk;
                        va[u] = (stA && kin && i0 + r < n) ? L[(int64_t)(k0 + k) * ldl + i0 + r] : 0.0;
                        vb[u] = (stB && kin && j0 + r < c1) ? L[(int64_t)(k0 + k) * ldl + j0 + r] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < kStageBatch; ++u) {
                        const int e = e0 + u * blockDim.x, k = e / kCholTile, r = e % kCholTile;
                        if (e < tot) {
                            if (stA) As[k * kCholTileStride + r] = va[u];
                            if (stB) Bs[k * kCholTileStride + r] = vb[u];
                        }
                    }
                }
            }
            __syncthreads();
            {  // the next tile's new panel rows and its C tile into L2 while this one is multiplied
                const int tn = next_tile(t + 1);
                if (tn < nt) {
                    const int i1 = r0 + (tn / ntj) * kCholTile, j1 = c0 + (tn % ntj) * kCholTile;
                    prefetch_tile(k0, kk, i1, j1, c1, !kMixed || i1 != i0, !kMixed || (i1 != j1 && j1 != b_j0));
                }
            }
            const double* Bt = diag ? As : Bs;
            if constexpr (!kMixed) chol_tile_simt<kCholTileStride>(As, Bt, i0, j0, c1, kk, threadIdx.x, blockDim.x);
            else chol_tile_dmma(As, Bt, i0, j0, c1, kk4, warp, lane, nwarps);
            __syncthreads();
        }
    }

    // chol_update for the mixed form with its panel rows staged by bulk
    // copies (cp.async.bulk, global -> shared, completion on an mbarrier)
    // issued one tile ahead. The panel rows L(x + r, k0 + k), r < kCholTile,
    // k < kk, of the tile row or tile column starting at row x are the same
    // data whether a tile uses them as A (i0 = x) or as B (j0 = x), so
    // kStageBufs buffers form a pool tagged by x. Before tile t is multiplied,
    // the rows tile t + 1 needs and the pool lacks are requested into buffers
    // tile t does not use, and tile t + 1's C columns are prefetched into L2
    // (cp.async.bulk.prefetch.L2); a tile row ends with its diagonal tile,
    // which uses one buffer, so the next row's A and B both arrive ahead.
    // There is no block barrier between tiles: warp 0 issues the copies
    // (lane 0 posts the byte count on the buffer's "full" mbarrier), every
    // warp waits on "full" before reading a buffer and, after the last tile
    // that uses it, arrives on its "empty" mbarrier (one arrival per warp);
    // warp 0 waits on "empty" before refilling a buffer. Column k of L
    // starts at Lt + k*ldl (a multiple of 16 doubles) and x is a multiple of 8,
    // so each copy is min(kCholTile, ldl - x) doubles on 16-byte boundaries;
    // rows beyond n or c1 in a buffer (padding, stale data) reach only C rows
    // or columns that are not stored, and rows k in [kk, kk4) are zero. The
    // panel columns are not written during the update; the generic-proxy
    // writes that produced them are ordered before the copies by a barrier and
    // fence.proxy.async. Every wait is bounded: on expiry the block records
    // ctl.brk = 2, waits (bounded) for its copies in flight and returns.
    static constexpr int kStageBufs = 3;

    __device__ __forceinline__ static uint32_t smem_addr(const void* p) {
        return (uint32_t)__cvta_generic_to_shared(p);
    }

    // Warp 0: the copies of panel rows starting at x into buf, completing on
    // bar (lane 0 posts the byte count, then each lane issues every 32nd row).
    __device__ void bulk_stage(double* buf, uint64_t* bar, int k0, int kk, int x, int lane) const {
        const int cnt = ldl - x < kCholTile ? ldl - x : kCholTile;
        const uint32_t bytes = (uint32_t)cnt * 8u, mb = smem_addr(bar);
        if (lane == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes * (uint32_t)kk)
                         : "memory");
        __syncwarp();
        for (int k = lane; k < kk; k += 32) {
            const double* src = Lt + (int64_t)(k0 + k) * ldl + x;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             smem_addr(buf + k * kCholTileStride)),
                         "l"(src), "r"(bytes), "r"(mb)
                         : "memory");
        }
    }

    // Wait for phase `parity` of bar; false if the bounded wait expired.
    // (at most ~1 s of the global timer, and at most 2^24 polls)
    __device__ static bool bar_wait(uint64_t* bar, uint32_t parity) {
        const uint32_t mb = smem_addr(bar);
        uint64_t t0 = 0;
        for (int it = 0; it < (1 << 24); ++it) {
            uint32_t done;
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                : "=r"(done)
                : "r"(mb), "r"(parity)
                : "memory");
            if (done) return true;
            if ((it & 255) == 0) {
                const uint64_t now = global_ns();
                if (it == 0) t0 = now;
                else if (now - t0 > 1000000000ull) return false;
            }
        }
        return false;
    }

    __device__ void chol_update_bulk(int k0, int k1, int r0, int c0, int c1) {
        const int kk = k1 - k0, kk4 = (kk + 3) & ~3;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
        const int nti = (n - r0 + kCholTile - 1) / kCholTile, ntj = (c1 - c0 + kCholTile - 1) / kCholTile;
        const int nt = nti * ntj;
        const int64_t bstride = (int64_t)kk4 * kCholTileStride;
        uint64_t* full = reinterpret_cast<uint64_t*>(stage + stage_cap - 8);  // copies landed
        uint64_t* empty = full + kStageBufs;                                   // every warp done reading
        for (int e = threadIdx.x; e < kStageBufs * (kk4 - kk) * kCholTile; e += blockDim.x) {
            const int b = e / ((kk4 - kk) * kCholTile), rem = e % ((kk4 - kk) * kCholTile);
            stage[b * bstride + (kk + rem / kCholTile) * kCholTileStride + rem % kCholTile] = 0.0;
        }
        if (threadIdx.x == 0)
            for (int b = 0; b < kStageBufs; ++b) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(full + b)) : "memory");
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(empty + b)), "r"(nwarps)
                             : "memory");
            }
        if (warp == 0) {  // the issuing warp: barrier inits visible, panel writes ordered before the copies
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile("fence.proxy.async;" ::: "memory");
        }
        __syncthreads();
        // Pool state, the same in every warp: the row each buffer holds or is
        // receiving (-1: none), a fill not yet consumed, a release the issuing
        // warp has not yet waited for, and the two barriers' phase parities.
        // A buffer released after its last use gives up its row (it is
        // fetched again if needed), so each release pairs with the next fill.
        int tag[kStageBufs], pend[kStageBufs], rel[kStageBufs];
        uint32_t par[kStageBufs], epar[kStageBufs];
#pragma unroll
        for (int b = 0; b < kStageBufs; ++b) tag[b] = -1, pend[b] = 0, rel[b] = 0, par[b] = 0, epar[b] = 0;
        volatile int32_t* gave_up = &ctl.brk;
        auto next_tile = [&](int t) {  // first tile >= t not wholly above the diagonal
            while (t < nt && r0 + (t / ntj) * kCholTile + kCholTile - 1 < c0 + (t % ntj) * kCholTile) ++t;
            return t;
        };
        auto find = [&](int x) {
            int f = -1;
#pragma unroll
            for (int b = 0; b < kStageBufs; ++b)
                if (tag[b] == x) f = b;
            return f;
        };
        // request row x unless present, into a buffer whose row is none of
        // keep0..keep2 (-2: no row) (no buffer free: it is requested again
        // when its tile comes); the issuing warp first waits until every warp
        // has released the buffer's previous contents
        auto request = [&](int x, int keep0, int keep1, int keep2) {
            if (find(x) >= 0) return;
            int f = -1;
#pragma unroll
            for (int b = kStageBufs - 1; b >= 0; --b)
                if (tag[b] != keep0 && tag[b] != keep1 && tag[b] != keep2) f = b;
            if (f < 0) return;
#pragma unroll
            for (int b = 0; b < kStageBufs; ++b)
                if (b == f) {
                    if (warp == 0) {
                        const bool freed = !rel[b] || __all_sync(0xffffffffu, bar_wait(empty + b, epar[b]));
                        if (freed) bulk_stage(stage + b * bstride, full + b, k0, kk, x, lane);
                        else if (lane == 0) *gave_up = 2;
                    }
                    if (rel[b]) epar[b] ^= 1u, rel[b] = 0;
                    tag[b] = x, pend[b] = 1;
                }
        };
        for (int t = next_tile(0), tn; t < nt; t = tn) {
            if (*gave_up) break;
            const int i0 = r0 + (t / ntj) * kCholTile, j0 = c0 + (t % ntj) * kCholTile;
            request(i0, i0, j0, -2);  // (present after a prefetch; else fetched now)
            request(j0, i0, j0, -2);
            const int ba = find(i0), bb = find(j0);
            bool landed = true;
#pragma unroll
            for (int b = 0; b < kStageBufs; ++b)
                if (pend[b] && (b == ba || b == bb)) {
                    if (__all_sync(0xffffffffu, bar_wait(full + b, par[b])))
                        par[b] ^= 1u, pend[b] = 0;
                    else
                        landed = false;
                }
            if (!landed) {
                if (lane == 0) *gave_up = 2;
                break;
            }
            tn = next_tile(t + 1);
            const int i1 = tn < nt ? r0 + (tn / ntj) * kCholTile : -2, j1 = tn < nt ? c0 + (tn % ntj) * kCholTile : -2;
            if (tn < nt) {  // the next tile's rows into buffers this tile does not use
                request(i1, i0, j0, -2);
                request(j1, i0, j0, i1);
                // and its C columns into L2 (bulk prefetch, one per column segment)
                if (warp == 1 % nwarps) {
                    const int cnt = ldl - i1 < kCholTile ? ldl - i1 : kCholTile;
                    const int jn = c1 - j1 < kCholTile ? c1 - j1 : kCholTile;
                    for (int c = lane; c < jn; c += 32)
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Lt + (int64_t)(j1 + c) * ldl + i1),
                                     "r"((uint32_t)cnt * 8u)
                                     : "memory");
                }
            }
            chol_tile_dmma(stage + ba * bstride, stage + bb * bstride, i0, j0, c1, kk4, warp, lane, nwarps);
            // release this tile's buffers the next tile does not use (no block
            // barrier: warps run ahead until a fill they need has not landed)
            __syncwarp();
#pragma unroll
            for (int b = 0; b < kStageBufs; ++b)
                if ((b == ba || b == bb) && tag[b] != i1 && tag[b] != j1) {
                    if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(empty + b)) : "memory");
                    rel[b] = 1, tag[b] = -1;
                }
        }
        __syncthreads();
        // fills still in flight (after a wait gave up) complete before the buffers go
        int expired = 0;
#pragma unroll
        for (int b = 0; b < kStageBufs; ++b)
            if (pend[b] && !bar_wait(full + b, par[b])) expired = 1;
        expired = __syncthreads_or(expired);
        if (threadIdx.x == 0) {
            for (int b = 0; b < 2 * kStageBufs; ++b)
                asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(full + b)) : "memory");
            if (expired) ctl.brk = 2;
        }
        __syncthreads();
    }

    // chol_update for the plain form with 512 threads: a 4x4 micro-tile per
    // thread covers 256 threads of a tile, so each pass takes two tiles of a
    // tile-row, (i0, j0) for threads 0-255 and (i0, j0 + 64) for 256-511,
    // against one staged As and two Bs. The three buffers are unpadded
    // (every access to them runs along a row). Each element still receives
    // its products in k order: the arithmetic is the single-tile path's.
    __device__ void chol_update_pairs(int k0, int k1, int r0, int c0, int c1) {
        const double* L = Lt;
        constexpr int TS = kCholTile;
        const int kk = k1 - k0, kk4 = (kk + 3) & ~3, tot = kk4 * kCholTile;
        double* As = stage;
        double* B0 = stage + (int64_t)kk4 * TS;
        double* B1 = B0 + (int64_t)kk4 * TS;
        const int nti = (n - r0 + kCholTile - 1) / kCholTile, ntj = (c1 - c0 + kCholTile - 1) / kCholTile;
        const int half = threadIdx.x >> 8, hl = threadIdx.x & 255;
        constexpr int kB = 4;  // staged elements per thread per array between loads and stores
        for (int ti = 0; ti < nti; ++ti) {
            const int i0 = r0 + ti * kCholTile;
            // tiles (ti, tj) with tj < tjn reach the diagonal (r0 == c0 in both callers, so i0 >= c0)
            const int tjn = min(ntj, (i0 + kCholTile - 1 - c0) / kCholTile + 1);
            for (int tj = 0; tj < tjn; tj += 2) {
                const int j0 = c0 + tj * kCholTile, j1 = j0 + kCholTile;
                const bool two = tj + 1 < tjn;
                for (int e0 = threadIdx.x; e0 < tot; e0 += kB * blockDim.x) {
                    double va[kB], v0[kB], v1[kB];
#pragma unroll
                    for (int u = 0; u < kB; ++u) {
                        const int e = e0 + u * blockDim.x, k = e / kCholTile, r = e % kCholTile;
                        const bool kin = e < tot && k < kk;
                        const double* col = L + (int64_t)(k0 + k) * ldl;
                        va[u] = (kin && i0 + r < n) ? col[i0 + r] : 0.0;
                        v0[u] = (kin && j0 + r < c1) ? col[j0 + r] : 0.0;
                        v1[u] = (two && kin && j1 + r < c1) ? col[j1 + r] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < kB; ++u) {
                        const int e = e0 + u * blockDim.x, k = e / kCholTile, r = e % kCholTile;
                        if (e < tot) {
                            As[k * TS + r] = va[u];
                            B0[k * TS + r] = v0[u];
                            if (two) B1[k * TS + r] = v1[u];
                        }
                    }
                }
                __syncthreads();
                {  // the next pass's panel rows and C tiles into L2 while this one is multiplied
                    int ti1 = ti, tj1 = tj + 2;
                    if (tj1 >= tjn) ti1 = ti + 1, tj1 = 0;
                    if (ti1 < nti) {
                        const int i1 = r0 + ti1 * kCholTile, n1 = min(ntj, (i1 + kCholTile - 1 - c0) / kCholTile + 1);
                        prefetch_tile(k0, kk, i1, c0 + tj1 * kCholTile, c1, true, true);
                        if (tj1 + 1 < n1) prefetch_tile(k0, kk, i1, c0 + (tj1 + 1) * kCholTile, c1, false, true);
                    }
                }
                if (half == 0) chol_tile_simt<TS>(As, B0, i0, j0, c1, kk, hl, 256);
                else if (two) chol_tile_simt<TS>(As, B1, i0, j1, c1, kk, hl, 256);
                __syncthreads();
            }
        }
    }

    // L2 prefetch hints for the tile at (i0, j0) of chol_update: its staged
    // panel segments L(i0.., k0 + k) (if wantA) and L(j0.., k0 + k) (if
    // wantB), k < kk, and its C columns L(i0.., j), j in [j0, min(j0 +
    // kCholTile, c1)). Each 64-element column segment spans at most five
    // 128-byte lines; one hint goes to elements 0, 16, 32, 48 and 63 of it
    // (clamped to the matrix).
    __device__ void prefetch_tile(int k0, int kk, int i0, int j0, int c1, bool wantA, bool wantB) const {
        const double* L = Lt;
        const int na = wantA ? kk : 0, nb = wantB ? kk : 0;
        const int ncc = c1 - j0 < kCholTile ? c1 - j0 : kCholTile;
        const int work = (na + nb + ncc) * 5;
        for (int w = threadIdx.x; w < work; w += blockDim.x) {
            const int seg = w / 5, p = w % 5, r = p == 4 ? kCholTile - 1 : p * 16;
            int col, row;
            if (seg < na) col = k0 + seg, row = min(i0 + r, n - 1);
            else if (seg < na + nb) col = k0 + seg - na, row = min(j0 + r, c1 - 1);
            else col = j0 + seg - na - nb, row = min(i0 + r, n - 1);
            asm volatile("prefetch.L2 [%0];" ::"l"(L + (int64_t)col * ldl + row));
        }
    }

    // Panel [kb, ke) of the blocked factorisation (step 1 above). The
    // diagonal block is staged column-major in shared memory (stage);
    // returns false on a pivot <= 0.
    __device__ bool chol_panel(int kb, int ke) {
        double* L = Lt;
        const int kk = ke - kb;
        double* D11 = stage;  // D11[c * kk + r] = L(kb + r, kb + c), r >= c
        for (int e = threadIdx.x; e < kk * kk; e += blockDim.x) {
            const int r = e % kk, c = e / kk;
            D11[e] = r >= c ? L[(int64_t)(kb + c) * ldl + kb + r] : 0.0;
        }
        __syncthreads();
        for (int k = 0; k < kk; ++k) {
            if (threadIdx.x == 0) {
                const double s = D11[k * kk + k];
                if (!(s > 0.0)) ctl.brk = 1; else D11[k * kk + k] = sqrt(s);
            }
            __syncthreads();
            if (ctl.brk) return false;
            const double dk = D11[k * kk + k];
            for (int r = k + 1 + threadIdx.x; r < kk; r += blockDim.x) D11[k * kk + r] = D11[k * kk + r] / dk;
            __syncthreads();
            for (int e = threadIdx.x; e < kk * kk; e += blockDim.x) {
                const int r = e % kk, j = e / kk;
                if (j > k && r >= j) D11[j * kk + r] = D11[j * kk + r] - D11[k * kk + r] * D11[k * kk + j];
            }
            __syncthreads();
        }
        for (int e = threadIdx.x; e < kk * kk; e += blockDim.x) {
            const int r = e % kk, c = e / kk;
            if (r >= c) L[(int64_t)(kb + c) * ldl + kb + r] = D11[e];
        }
        // rows below the block, one per thread
        for (int i = ke + threadIdx.x; i < n; i += blockDim.x) {
            double a[kCholMaxPanel];
#pragma unroll
            for (int k = 0; k < kCholMaxPanel; ++k) a[k] = k < kk ? L[(int64_t)(kb + k) * ldl + i] : 0.0;
#pragma unroll
            for (int j = 0; j < kCholMaxPanel; ++j) {
                if (j < kk) {
                    double s = a[j];
#pragma unroll
                    for (int k = 0; k < j; ++k) s = s - a[k] * D11[k * kk + j];
                    a[j] = s / D11[j * kk + j];
                }
            }
#pragma unroll
            for (int k = 0; k < kCholMaxPanel; ++k)
                if (k < kk) L[(int64_t)(kb + k) * ldl + i] = a[k];
        }
        __syncthreads();
        return true;
    }

    // Trailing-update tile, FP64 CUDA cores: 4x4 elements per thread, each
    // element c = c - a_k * b_k for k = 0, 1, ... (no contraction: the plain
    // form is compiled without FMA).
    // Threads take micro-tiles first, first + step, ...; As / Bs rows are TS
    // doubles apart.
    template <int TS>
    __device__ void chol_tile_simt(const double* As, const double* Bs, int i0, int j0, int jend, int kk, int first,
                                   int step) {
        double* L = Lt;
        constexpr int Q = kCholTile / 4;
        for (int mtl = first; mtl < Q * Q; mtl += step) {
            const int r0 = (mtl % Q) * 4, c0 = (mtl / Q) * 4;
            if (i0 + r0 + 3 < j0 + c0) continue;  // all above the diagonal
            double c[4][4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int i = i0 + r0 + u, j = j0 + c0 + v;
                    c[u][v] = (i < n && j < jend && i >= j) ? L[(int64_t)j * ldl + i] : 0.0;
                }
            for (int k = 0; k < kk; ++k) {
                const double2 a01 = *reinterpret_cast<const double2*>(As + k * TS + r0);
                const double2 a23 = *reinterpret_cast<const double2*>(As + k * TS + r0 + 2);
                const double2 b01 = *reinterpret_cast<const double2*>(Bs + k * TS + c0);
                const double2 b23 = *reinterpret_cast<const double2*>(Bs + k * TS + c0 + 2);
                const double av[4] = {a01.x, a01.y, a23.x, a23.y}, bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 4; ++v) c[u][v] = c[u][v] - av[u] * bv[v];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int i = i0 + r0 + u, j = j0 + c0 + v;
                    if (i < n && j < jend && i >= j) L[(int64_t)j * ldl + i] = c[u][v];
                }
        }
    }

    // Trailing-update tile on the FP64 tensor cores. The 64x64 tile is 8x8
    // blocks of 8x8, grouped in 16 strips of one block-row by four
    // block-columns (strip s: rows 8 (s % 8), columns 32 (s / 8) + 8u, u < 4);
    // warp w takes strips w, w + nwarps, ... Per k step of 4 the strip's A
    // fragment is read once and multiplied into its four C fragments with
    // mma.sync.m8n8k4.f64, C += (-A) B (A 8x4 row: lane holds
    // A[lane/4][lane%4]; B 4x8 col: lane holds B[lane%4][lane/4]; C 8x8: lane
    // holds C[lane/4][2(lane%4)], C[lane/4][2(lane%4)+1]). (Loading the first
    // strip's C fragments before the staging barrier instead made the kernel
    // spill at its 128-register cap and measured 3% slower.) jend: columns
    // from jend on are left alone. kk4: the panel width rounded up to 4 (the
    // staged rows are zero beyond).
    static constexpr int kStrips = (kCholTile / 8) * (kCholTile / 32);

    // C fragments of strip s of the tile at (i0, j0) (zero outside the lower
    // triangle and the matrix).
    __device__ void dmma_load_c(int s, int i0, int j0, int jend, int lane, double (&c)[4][2]) const {
        const double* L = Lt;
        const int g = lane >> 2, q = lane & 3, tr = (s % 8) * 8, tcs = (s / 8) * 32;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int tc = tcs + 8 * u;
            const bool act = !(i0 + tr + 7 < j0 + tc);
            const int i = i0 + tr + g, ja = j0 + tc + 2 * q, jb = ja + 1;
            c[u][0] = (act && i < n && ja < jend && i >= ja) ? L[(int64_t)ja * ldl + i] : 0.0;
            c[u][1] = (act && i < n && jb < jend && i >= jb) ? L[(int64_t)jb * ldl + i] : 0.0;
        }
    }

    __device__ void chol_tile_dmma(const double* As, const double* Bs, int i0, int j0, int jend, int kk4, int warp,
                                   int lane, int nwarps) {
        for (int s = warp; s < kStrips; s += nwarps) {
            const int tr = (s % 8) * 8, tcs = (s / 8) * 32;
            if (i0 + tr + 7 < j0 + tcs) continue;  // the whole strip above the diagonal (warp-uniform)
            double c[4][2];
            dmma_load_c(s, i0, j0, jend, lane, c);
            dmma_strip<4>(s, c, As, Bs, i0, j0, jend, kk4, lane);
        }
    }

    // Strip s of the tile at (i0, j0): C (loaded into c) -= A B over kk4 staged
    // k rows, stored back. kDmmaChains accumulation chains per fragment (k
    // steps rotate over c and cx, summed at the end) cut the dependent-DMMA
    // wait; the mixed form's tolerance admits the reassociation.
    template <int kDmmaChains>
    __device__ void dmma_strip(int s, double (&c)[4][2], const double* As, const double* Bs, int i0, int j0, int jend,
                               int kk4, int lane) {
        double* L = Lt;
        const int g = lane >> 2, q = lane & 3;
        const int tr = (s % 8) * 8, tcs = (s / 8) * 32;
        {
            // blocks u < nact are active: the columns grow with u (warp-uniform)
            const int d = i0 + tr + 7 - j0 - tcs, nact = d >= 24 ? 4 : d / 8 + 1;
            double cx[kDmmaChains - 1][4][2];
#pragma unroll
            for (int h = 0; h < kDmmaChains - 1; ++h)
#pragma unroll
                for (int u = 0; u < 4; ++u) cx[h][u][0] = cx[h][u][1] = 0.0;
            int k = 0;
            for (; k + 4 * kDmmaChains <= kk4; k += 4 * kDmmaChains) {
#pragma unroll
                for (int h = 0; h < kDmmaChains; ++h) {
                    const double av = -As[(k + 4 * h + q) * kCholTileStride + tr + g];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        if (u < nact) {
                            const double bv = Bs[(k + 4 * h + q) * kCholTileStride + tcs + 8 * u + g];
                            double& d0 = h == 0 ? c[u][0] : cx[h > 0 ? h - 1 : 0][u][0];
                            double& d1 = h == 0 ? c[u][1] : cx[h > 0 ? h - 1 : 0][u][1];
                            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                                         : "+d"(d0), "+d"(d1)
                                         : "d"(av), "d"(bv));
                        }
                    }
                }
            }
            for (; k < kk4; k += 4) {  // kk4 is a multiple of 4
                const double av = -As[(k + q) * kCholTileStride + tr + g];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (u < nact) {
                        const double bv = Bs[(k + q) * kCholTileStride + tcs + 8 * u + g];
                        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                                     : "+d"(c[u][0]), "+d"(c[u][1])
                                     : "d"(av), "d"(bv));
                    }
                }
            }
#pragma unroll
            for (int h = 0; h < kDmmaChains - 1; ++h)
#pragma unroll
                for (int u = 0; u < 4; ++u) c[u][0] += cx[h][u][0], c[u][1] += cx[h][u][1];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = i0 + tr + g, ja = j0 + tcs + 8 * u + 2 * q, jb = ja + 1;
                if (u < nact && i < n && ja < jend && i >= ja) L[(int64_t)ja * ldl + i] = c[u][0];
                if (u < nact && i < n && jb < jend && i >= jb) L[(int64_t)jb * ldl + i] = c[u][1];
            }
        }
    }

    // y = L x (lower_matvec, src/linalg.cpp:109-117), row sums in j order.
    __device__ void lower_matvec(const double* x, double* y) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double s = 0.0;
            for (int j = 0; j <= i; ++j) s += Lt[(int64_t)j * ldl + i] * x[j];
            y[i] = s;
        }
    }

    // ---- forces ---------------------------------------------------------

    // Bonds (N-1 x 3) and clamped lengths of R (chain_geometry, src/config.cpp:15-25).
    __device__ void geometry(const double* R, double* bond, double* len) {
        for (int b = threadIdx.x; b < N - 1; b += blockDim.x) {
            const double b0 = R[3 * b + 3] - R[3 * b], b1 = R[3 * b + 4] - R[3 * b + 1],
                         b2 = R[3 * b + 5] - R[3 * b + 2];
            bond[3 * b] = b0;
            bond[3 * b + 1] = b1;
            bond[3 * b + 2] = b2;
            len[b] = clamped_len(b0, b1, b2);
        }
    }

    // Spring bead forces from bonds (connector_forces + bead_forces_from_connectors,
    // src/spring.cpp:183-207). Fc: scratch for the bond forces.
    __device__ void spring_from_geometry(const double* bond, const double* len, double* Fc, double* F) {
        for (int b = threadIdx.x; b < N - 1; b += blockDim.x) {
            const double f = connector_factor(ch, len[b]);
            Fc[3 * b] = f * bond[3 * b];
            Fc[3 * b + 1] = f * bond[3 * b + 1];
            Fc[3 * b + 2] = f * bond[3 * b + 2];
        }
        __syncthreads();
        bead_forces(Fc, F);
    }

    __device__ void bead_forces(const double* Fc, double* F) {
        for (int i = threadIdx.x; i < N; i += blockDim.x)
            for (int d = 0; d < 3; ++d) {
                double v;
                if (i == 0) v = Fc[d];
                else if (i == N - 1) v = (-1.0) * Fc[3 * (N - 2) + d];
                else v = Fc[3 * i + d] - Fc[3 * (i - 1) + d];
                F[3 * i + d] = v;
            }
    }

    // Excluded-volume force on bead b (ExcludedVolume::force,
    // src/excluded_volume.cpp:60-89): bead b receives -f(j,b) for j<b, then
    // +f(b,j) for j>b, in ascending j -- the reference loop's order.
    __device__ void ev_on_bead(const double* R, int b, double f[3]) {
        f[0] = f[1] = f[2] = 0.0;
        if (ch.ev_type == BDCU_EV_NONE) return;
        const double* phi = (ch.ev_type == BDCU_EV_SDK && ch.phi_off >= 0) ? a.arena + ch.phi_off : nullptr;
        if constexpr (!kMixed) {
            for (int j = 0; j < N; ++j) {
                if (j == b) continue;
                const int mu = j < b ? j : b, nu = j < b ? b : j;
                if ((nu - mu) < ch.cd) continue;
                const double q0 = R[3 * nu] - R[3 * mu], q1 = R[3 * nu + 1] - R[3 * mu + 1],
                             q2 = R[3 * nu + 2] - R[3 * mu + 2];
                double sq = q0 * q0 + q1 * q1 + q2 * q2;
                if (sq < 1.0e-12) sq = 1.0e-12;
                const double r = sqrt(sq);
                const double fac = ev_factor(ch, r, phi ? phi[mu * N + nu] : 0.0);
                const double g0 = (-fac) * q0, g1 = (-fac) * q1, g2 = (-fac) * q2;
                if (b == mu) {
                    f[0] = f[0] + g0; f[1] = f[1] + g1; f[2] = f[2] + g2;
                } else {
                    f[0] = f[0] - g0; f[1] = f[1] - g1; f[2] = f[2] - g2;
                }
            }
        } else {
            // FP32 pair sums from the staged FP32 coordinates.
            const float4 rb = pos32[b];
            float f0 = 0.f, f1 = 0.f, f2 = 0.f;
            const float zs = (float)ch.zsbyds5, p5 = (float)ch.pt5bydssq;
            for (int j = 0; j < N; ++j) {
                if (j == b) continue;
                const int mu = j < b ? j : b, nu = j < b ? b : j;
                if ((nu - mu) < ch.cd) continue;
                const float4 rj = pos32[j];
                // q = R_nu - R_mu; the force on b is -fac*q if b == mu, +fac*q if b == nu
                const float s = (b == mu) ? 1.f : -1.f;
                const float q0 = s * (rj.x - rb.x), q1 = s * (rj.y - rb.y), q2 = s * (rj.z - rb.z);
                float sq = fmaxf(q0 * q0 + q1 * q1 + q2 * q2, 1e-12f);
                const float r = sqrtf(sq);
                float fac;
                if (ch.ev_type == BDCU_EV_GAUSS) {
                    fac = zs * __expf(-sq * p5);
                } else {
                    fac = (float)ev_factor(ch, (double)r, phi ? phi[mu * N + nu] : 0.0);
                }
                const float g = (b == mu) ? -fac : fac;
                f0 += g * q0;
                f1 += g * q1;
                f2 += g * q2;
            }
            f[0] = f0;
            f[1] = f1;
            f[2] = f2;
        }
    }

    // Explicit force Fe = (EV + bending)(R) + external(t) (src/model.hpp:56-64,
    // src/integrator.cpp:75-76). bond/len: geometry of R (already computed);
    // u, cs: scratch.
    __device__ void explicit_force(const double* R, double t, const double* bond, const double* len, double* u,
                                   double* cs, double* out, bool with_external = true) {
        const bool bend = (ch.bend_type != BDCU_BEND_NONE) && N > 2;
        if (bend) {
            for (int b = threadIdx.x; b < N - 1; b += blockDim.x)
                for (int d = 0; d < 3; ++d) u[3 * b + d] = (1.0 / len[b]) * bond[3 * b + d];
            __syncthreads();
            for (int b = threadIdx.x; b < N - 2; b += blockDim.x)
                cs[b] = u[3 * (b + 1)] * u[3 * b] + u[3 * (b + 1) + 1] * u[3 * b + 1] + u[3 * (b + 1) + 2] * u[3 * b + 2];
            __syncthreads();
        }
        for (int m = threadIdx.x; m < N; m += blockDim.x) {
            double fe[3], fb[3] = {0.0, 0.0, 0.0}, fx[3] = {0.0, 0.0, 0.0};
            ev_on_bead(R, m, fe);
            if (bend) bending_on_bead(ch, m, u, cs, len, fb);
            if (!with_external) {
                for (int d = 0; d < 3; ++d) out[3 * m + d] = fe[d] + fb[d];
                continue;
            }
            if (ch.ext_n > 0) external_on_bead(ch, a.arena, m, t, fx);
            for (int d = 0; d < 3; ++d) out[3 * m + d] = (fe[d] + fb[d]) + fx[d];
        }
    }

    // ---- Lanczos bounds --------------------------------------------------

    __device__ double* Vvec(int j, int m) { return (m <= a.v_cap ? Vs : Vg) + (int64_t)j * ldv; }

    // lanczos_extremes (src/hydrodynamics.cpp:146-221). Writes alpha/beta,
    // ctl.rmin/rmax, ctl.lz_steps, and the Ritz vectors into vmin/vmax.
    // The first product D v0 is formed together with `nex` other products of
    // the step (ex[r] -> ey[r]), against the same D.
    __device__ void lanczos(int m, bool warm, const double* cache, double* w, double* vmin, double* vmax,
                            int nex = 0, const double* const* ex = nullptr, double* const* ey = nullptr) {
        if (n < m) m = n;
        double* V0 = Vvec(0, m);
        if (warm) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) V0[i] = cache[i];
            __syncthreads();
            double nv = sqrt(block_dot(V0, V0, n, red));
            if (!(nv > 0.0)) {
                for (int i = threadIdx.x; i < n; i += blockDim.x) V0[i] = a.seed_table[i];
                nv = ch.seed_norm;
            }
            __syncthreads();
            for (int i = threadIdx.x; i < n; i += blockDim.x) V0[i] = V0[i] / nv;
        } else {
            const double nv = ch.seed_norm;
            for (int i = threadIdx.x; i < n; i += blockDim.x) V0[i] = a.seed_table[i] / nv;
        }
        __syncthreads();
        int k = 0;
        double b = 0.0;
        for (int j = 0; j < m; ++j) {
            double* v = Vvec(j, m);
            const double* vprev = (j > 0) ? Vvec(j - 1, m) : nullptr;
            if (j == 0 && nex > 0) {
                const double* xs[4] = {v, ex[0], nex > 1 ? ex[1] : nullptr, nex > 2 ? ex[2] : nullptr};
                double* ys[4] = {w, ey[0], nex > 1 ? ey[1] : nullptr, nex > 2 ? ey[2] : nullptr};
                apply_D_n(1 + nex, xs, ys);
            } else {
                apply_D(v, w);
            }
            __syncthreads();
            const double al = block_dot(v, w, n, red);
            if (threadIdx.x == 0) alpha[k] = al;
            ++k;
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const double vp = vprev ? vprev[i] : 0.0;
                w[i] -= al * v[i] + b * vp;
            }
            __syncthreads();
            for (int u = 0; u <= j; ++u) {
                const double* uu = Vvec(u, m);
                const double dd = block_dot(w, uu, n, red);
                for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] -= dd * uu[i];
                __syncthreads();
            }
            b = sqrt(block_dot(w, w, n, red));
            if (b < 1.0e-10) break;
            if (j + 1 < m) {
                double* vn = Vvec(j + 1, m);
                for (int i = threadIdx.x; i < n; i += blockDim.x) vn[i] = w[i] / b;
            }
            if (threadIdx.x == 0) beta[j] = b;
            __syncthreads();
        }
        __syncthreads();
        if (k == 1) {
            if (threadIdx.x == 0) {
                ctl.rmin = alpha[0];
                ctl.rmax = alpha[0];
                ctl.lz_steps = 1;
            }
            for (int i = threadIdx.x; i < n; i += blockDim.x) vmin[i] = vmax[i] = V0[i];
            __syncthreads();
            return;
        }
        // Gershgorin bracket (src/hydrodynamics.cpp:187-194)
        if (threadIdx.x == 0) {
            double lo = alpha[0], hi = alpha[0];
            for (int i = 0; i < k; ++i) {
                const double rad = (i > 0 ? fabs(beta[i - 1]) : 0.0) + (i < k - 1 ? fabs(beta[i]) : 0.0);
                lo = dmin_(lo, alpha[i] - rad);
                hi = dmax_(hi, alpha[i] + rad);
            }
            ctl.glo = lo;
            ctl.ghi = hi;
            ctl.lz_steps = k;
        }
        __syncthreads();
        const int warp = threadIdx.x >> 5;
        if (warp < 2) {
            double lo = ctl.glo, hi = ctl.ghi;
            warp_bisect(alpha, beta, k, warp == 0 ? 1 : k, lo, hi);
            if ((threadIdx.x & 31) == 0) {
                const double r = 0.5 * (lo + hi);
                if (warp == 0) ctl.rmin = r; else ctl.rmax = r;
                tridiag_eigenvector(alpha, beta, k, r, warp == 0 ? ymin : ymax);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double s1 = 0.0, s2 = 0.0;
            for (int j = 0; j < k; ++j) {
                const double vji = Vvec(j, m)[i];
                s1 += ymin[j] * vji;
                s2 += ymax[j] * vji;
            }
            vmin[i] = s1;
            vmax[i] = s2;
        }
        __syncthreads();
    }

    // spectral_bounds (src/hydrodynamics.cpp:224-264). Updates the chain's
    // warm-start vector in `cache` and ctl.lmin/lmax.
    // The first Lanczos product is fused with `nex` (<= 3) further products
    // of the step (ex[r] -> ey[r]).
    __device__ void spectral_bounds(double* cache, double* w, double* vmin, double* vmax, double* s, int nex = 0,
                                    const double* const* ex = nullptr, double* const* ey = nullptr) {
        const bool can_warm = ctl.cache_valid != 0;
        lanczos(can_warm ? kLanczosWarm : kLanczosCold, can_warm, cache, w, vmin, vmax, nex, ex, ey);
        if (can_warm && ctl.lz_steps < 4) {
            lanczos(kLanczosCold, false, cache, w, vmin, vmax);
            count(C_LZCOLD, 1);
        } else {
            count(can_warm ? C_LZWARM : C_LZCOLD, 1);
        }
        const double un = ch.seed_norm;
        for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = vmin[i] + vmax[i] + 0.01 * a.seed_table[i] / un;
        __syncthreads();
        const double sn = sqrt(block_dot(s, s, n, red));
        if (sn > 0.0 && isfinite(sn)) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) cache[i] = s[i] / sn;
        }
        if (threadIdx.x == 0) {
            ctl.cache_valid = (sn > 0.0 && isfinite(sn)) ? 1 : 0;
            double lmin = 0.5 * ctl.rmin;
            const double lmax = 1.02 * ctl.rmax;
            if (lmin < 1.0e-12) lmin = 1.0e-12;
            if (lmin >= lmax) lmin = lmax * 1.0e-6;
            ctl.lmin = lmin;
            ctl.lmax = lmax;
        }
        __syncthreads();
    }

    // ---- Chebyshev square root (src/hydrodynamics.cpp:267-337) ----------
    // out = D^{1/2} x0 approximation; returns with ctl.fd_err, ctl.L set.
    // Scratch: Dx0, t1, t2, t3, Dv.
    // dx0_ready: Dx0 already holds D x0 (formed with the step's other products).
    __device__ void chebyshev(const double* x0, double* out, double* Dx0, double* t1, double* t2, double* t3,
                              double* Dv, bool dx0_ready = false) {
        if (!dx0_ready) apply_D(x0, Dx0);
        __syncthreads();
        const double x0Dx0 = block_dot(x0, Dx0, n, red);
        const double lmin = ctl.lmin, lmax = ctl.lmax;
        double Lr = sqrt(lmax / lmin) * ch.mult + 0.5;
        int L;
        if (!(Lr < 2.0e9)) L = kMaxCheb;  // guards the int conversion (NaN/huge)
        else L = (int)Lr + 1;
        L = L > kMaxCheb ? kMaxCheb : L;
        L = L < 2 ? 2 : L;
        const double da = 2.0 / (lmax - lmin);
        const double db = -(lmax + lmin) / (lmax - lmin);
        for (;;) {
            // sqrt_chebyshev_coefficients (src/hydrodynamics.cpp:267-280)
            for (int k = threadIdx.x; k <= L; k += blockDim.x)
                sqx[k] = sqrt(cos(kPi * (k + 0.5) / (L + 1)) / da - db / da);
            __syncthreads();
            for (int j = threadIdx.x; j <= L; j += blockDim.x) {
                double s = 0.0;
                for (int k = 0; k <= L; ++k) s += sqx[k] * cos(j * (k + 0.5) * kPi / (L + 1));
                s *= 2.0 / (L + 1);
                if (j == 0) s /= 2.0;
                coef[j] = s;
            }
            __syncthreads();
            // chebyshev_series (src/hydrodynamics.cpp:284-312). T1 = da*D x0 + db*x0
            // reuses D x0 from above (the same product, bit for bit).
            const double c0 = coef[0], c1 = coef[1];
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const double tc = da * Dx0[i] + db * x0[i];
                t1[i] = tc;
                out[i] = c0 * x0[i];
                out[i] += c1 * tc;
            }
            __syncthreads();
            // three rotating buffers: T_{l-2} (x0 at first), T_{l-1}, T_l
            double* T[3] = {t1, t2, t3};
            const double* tp = x0;
            int ic = 0, in = 1;
            for (int l = 2; l <= L; ++l) {
                const double* tc = T[ic];
                double* tn = T[in];
                apply_D(tc, Dv);
                __syncthreads();
                const double cl = coef[l];
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    double v = da * Dv[i] + db * tc[i];
                    v = 2.0 * v - tp[i];
                    tn[i] = v;
                    out[i] += cl * v;
                }
                __syncthreads();
                tp = tc;
                const int nx = 3 - ic - in;
                ic = in;
                in = nx;
            }
            count(C_CHEB, L);
            const double rr = block_dot(out, out, n, red);
            const double fd = fabs(rr - x0Dx0) / x0Dx0;
            if (fd <= ch.fd_tol || L >= kMaxCheb) {
                if (threadIdx.x == 0) {
                    ctl.fd_err = fd;
                    ctl.L = L;
                }
                __syncthreads();
                return;
            }
            const int grow = L / 4 > 1 ? L / 4 : 1;
            L = (L + grow) > kMaxCheb ? kMaxCheb : L + grow;
            __syncthreads();
        }
    }
};

// ------------------------------------------------------------ the kernel

template <int FORM>
__global__ void __launch_bounds__(512, 1) integrate_kernel(const RunArgs a) {
    extern __shared__ __align__(16) double sm[];
    constexpr bool kMixed = (FORM == BDCU_FORM_MIXED_FP32);
    const SmemLayout lay = smem_layout(a.n_max, a.d_in_smem, a.v_cap, kMixed);
    const ScratchLayout scl = scratch_layout(a.n_max, a.d_in_smem, a.v_cap, a.need_chol, kMixed, a.need_d, a.need_lz);
    Ctl& ctl = *reinterpret_cast<Ctl*>(sm + lay.ctl);
    DevChain& ch = *reinterpret_cast<DevChain*>(sm + lay.chain);
    double* scr = a.scratch + (int64_t)blockIdx.x * a.scratch_stride;

    Block<FORM> B(a, ctl, ch);
    B.red = sm + lay.red;
    B.alpha = sm + lay.alpha;
    B.beta = sm + lay.beta;
    B.ymin = sm + lay.ymin;
    B.ymax = sm + lay.ymax;
    B.coef = sm + lay.coef;
    B.sqx = sm + lay.sqx;
    const int nvs = (int)round_up8(a.n_max);
    for (int k = 0; k < kSlots; ++k) B.slot[k] = sm + lay.slots + (int64_t)k * nvs;
    B.Vs = sm + lay.V;
    B.Vg = scr + scl.V;
    B.ldv = nvs;
    B.Lt = scr + scl.Lt;
    B.stage = B.slot[kCholFirstSlot];
    B.stage_cap = (int64_t)(kSlots - kCholFirstSlot) * nvs;
    B.pos32 = reinterpret_cast<float4*>(sm + lay.f32);
    B.vec32 = reinterpret_cast<float4*>(sm + lay.f32 + nvs);

    const int tid = threadIdx.x;
    const uint64_t t_launch = global_ns();
    for (;;) {
        if (tid == 0) {
            const int item = atomicAdd(a.work_counter, 1);
            ctl.chain = item >= a.n_work ? -1 : (a.order ? a.order[item] : item);
        }
        __syncthreads();
        const int c = ctl.chain;
        if (c < 0) break;
        {
            const int nw = (int)(sizeof(DevChain) / 8);
            const double* src = reinterpret_cast<const double*>(a.chains + c);
            double* dst = reinterpret_cast<double*>(&ch);
            for (int i = tid; i < nw; i += blockDim.x) dst[i] = src[i];
        }
        if (tid == 0) {
            ctl.status = a.status[c];
            ctl.cache_valid = (a.cache_mode == BDCU_CACHE_PERSIST) ? a.cache_valid[c] : 0;
            for (int k = 0; k < 8; ++k) ctl.cnt[k] = 0;
            ctl.brk = 0;
        }
        __syncthreads();
        if (ctl.status & BDCU_ST_FATAL_MASK) {
            __syncthreads();
            continue;
        }
        if (ch.bad_param) {
            if (tid == 0) a.status[c] = ctl.status | BDCU_ST_BAD_PARAM;
            __syncthreads();
            continue;
        }
        const int N = ch.N, n = 3 * N;
        B.N = N;
        B.n = n;
        B.ldl = chol_ld(n);
        B.hi = ch.hstar > 0.0;
        if constexpr (!kMixed) {
            B.D = a.d_in_smem ? (sm + lay.D) : (scr + scl.D);
            B.ldd = a.d_in_smem ? n : a.n_max;
        } else {
            B.D = nullptr;
            B.ldd = 0;
        }
        double* R = B.slot[0];
        double* Fs = B.slot[1];
        double* Fe = B.slot[2];
        double* dW = B.slot[3];
        double* X0 = B.slot[4];
        double* Rp = B.slot[5];
        double* A = B.slot[6];
        double* Bv = B.slot[7];
        double* Cv = B.slot[8];
        double* E = B.slot[9];
        double* F = B.slot[10];
        double* G = B.slot[11];
        double* H = B.slot[12];
        double* I = B.slot[13];
        double* J = B.slot[14];
        double* K = B.slot[15];
        double* gR = a.R + 3 * ch.bead_off;
        double* gcache = a.cache + 3 * ch.bead_off;
        for (int i = tid; i < n; i += blockDim.x) R[i] = gR[i];
        int32_t ix = 0, iy = 0, iseed = 0;
        if (tid == 0) {
            ix = a.rng[3 * c];
            iy = a.rng[3 * c + 1];
            iseed = a.rng[3 * c + 2];
        }
        const int nsteps = a.n_steps[c];
        double t = a.t_start[c];
        const double dt = ch.dt;
        const double sqrt2inv = 1.0 / sqrt(2.0);
        const double sqrt_dt = sqrt(dt);
        __syncthreads();

        int step = 0;
        for (; step < nsteps; ++step) {
            if (a.budget_ns > 0) {  // time slice: no new step past the budget
                if (tid == 0) ctl.stop = (int64_t)(global_ns() - t_launch) >= a.budget_ns;
                __syncthreads();
                if (ctl.stop) break;
            }
            bool pre = false;        // J, K hold D (Fs + Fe) and D Fs from the bounds' first pass
            bool chol_used = false;  // this step factored D into Lt
            // recenter (src/integrator.cpp:88-93)
            if (ch.update_com) {
                if (tid < 3) {
                    double s = 0.0;
                    for (int i = 0; i < N; ++i) s = s + R[3 * i + tid];
                    ctl.com[tid] = (1.0 / N) * s;
                }
                __syncthreads();
                for (int i = tid; i < n; i += blockDim.x) R[i] = R[i] - ctl.com[i % 3];
                __syncthreads();
            }
            if constexpr (kMixed) {
                for (int b = tid; b < N; b += blockDim.x)
                    B.pos32[b] = make_float4((float)R[3 * b], (float)R[3 * b + 1], (float)R[3 * b + 2], 0.f);
            }
            // Fs, Fe at R (src/integrator.cpp:70-76)
            B.geometry(R, Cv, E);
            __syncthreads();
            B.spring_from_geometry(Cv, E, F, Fs);
            __syncthreads();
            B.explicit_force(R, t, Cv, E, F, G, Fe);
            // The raw noise (src/mobility.cpp:18-29) and D at R (src/mobility.cpp:39-51):
            // thread 0 draws the 3N uniforms, then joins the other threads, which
            // have started assembling D.
            if (tid == 0) {
                if (iseed <= 0 || iy < 0) {
                    const int32_t s = iseed < 0 ? -iseed : iseed;
                    iy = (888889999 ^ s) | 1;
                    ix = 777755555 ^ s;
                    iseed = s + 1;
                }
                const float am = __fdiv_rn(__int_as_float(0x3f7fffff), 2147483648.0f);
                uint32_t ux = (uint32_t)ix;
                for (int k = 0; k < n; ++k) {
                    ux ^= (ux << 13);
                    ux ^= (ux >> 17);
                    ux ^= (ux << 5);
                    const int32_t kk = iy / 127773;
                    iy = 16807 * (iy - kk * 127773) - 2836 * kk;
                    if (iy < 0) iy += 2147483647;
                    const uint32_t mixed = ux ^ (uint32_t)iy;
                    const int32_t res = (int32_t)((mixed & 0x7fffffffu) | 1u);
                    X0[k] = (double)__fmul_rn(am, __int2float_rn(res));
                }
                ix = (int32_t)ux;
            }
            if (B.hi) {
                if constexpr (!kMixed) {
                    B.build_rpy(R, B.D, B.ldd);
                } else {
                    if (ch.hi_method == BDCU_HI_CHOLESKY) {
                        // dense FP64 D straight into the factor's storage (lower part)
                        B.build_rpy(R, B.Lt, B.ldl);
                    }
                }
            }
            __syncthreads();
            for (int i = tid; i < n; i += blockDim.x) {
                const double y = X0[i] - 0.5;
                X0[i] = (14.14855378 * y * y + 1.21569221) * y;
            }
            __syncthreads();
            // brownian_step (src/mobility.cpp:58-88)
            if (!B.hi) {
                for (int i = tid; i < n; i += blockDim.x) dW[i] = sqrt_dt * X0[i];
            } else if (ch.hi_method == BDCU_HI_CHOLESKY) {
                chol_used = true;
                bool ok;
                if constexpr (!kMixed) ok = B.cholesky(B.D, B.ldd, false);
                else ok = B.cholesky(nullptr, 0, true);
                if (!ok) {
                    if (tid == 0) ctl.status |= ctl.brk == 2 ? BDCU_ST_TIMEOUT : BDCU_ST_NOT_PD;
                    __syncthreads();
                    break;
                }
                B.lower_matvec(X0, A);
                __syncthreads();
                for (int i = tid; i < n; i += blockDim.x) dW[i] = sqrt_dt * A[i];
            } else {
                // the step's products that do not depend on one another go with
                // the Lanczos start vector's: D x0 (Chebyshev) -> H, D (Fs + Fe)
                // (predictor) -> J, D Fs (upsilon) -> K, with Fs + Fe in I
                for (int i = tid; i < n; i += blockDim.x) I[i] = Fs[i] + Fe[i];
                __syncthreads();
                const double* ex[3] = {X0, I, Fs};
                double* ey[3] = {H, J, K};
                B.spectral_bounds(gcache, A, Bv, Cv, E, 3, ex, ey);
                B.chebyshev(X0, F, H, Bv, Cv, E, G, true);
                pre = true;
                if (!(ctl.fd_err <= ch.fd_tol)) {
                    // Cholesky fallback (src/mobility.cpp:69-81)
                    if (tid == 0) {
                        ctl.status |= BDCU_ST_CHEB_FALLBACK;
                        ctl.cnt[C_FALLBACK] += 1;
                    }
                    chol_used = true;
                    bool ok;
                    if constexpr (!kMixed) {
                        ok = B.cholesky(B.D, B.ldd, false);
                    } else {
                        B.build_rpy(R, B.Lt, B.ldl);
                        ok = B.cholesky(nullptr, 0, true);
                    }
                    if (!ok) {
                        if (tid == 0) ctl.status |= ctl.brk == 2 ? BDCU_ST_TIMEOUT : BDCU_ST_NOT_PD;
                        __syncthreads();
                        break;
                    }
                    B.lower_matvec(X0, F);
                    __syncthreads();
                    pre = false;  // the blocked factorisation stages tiles in slots I..K
                }
                for (int i = tid; i < n; i += blockDim.x) dW[i] = sqrt_dt * F[i];
            }
            __syncthreads();
            // predictor (src/integrator.cpp:96-101)
            double K1[9], K2[9];
            kappa_at(ch, a.arena, t, K1);
            kappa_at(ch, a.arena, t + dt, K2);
            if (!pre) {
                // D (Fs + Fe) -> J for the predictor and D Fs -> K for upsilon, in one pass
                for (int i = tid; i < n; i += blockDim.x) I[i] = Fs[i] + Fe[i];
                __syncthreads();
                const double* xs[2] = {I, Fs};
                double* ys[2] = {J, K};
                B.template apply_D_multi<2>(xs, ys);
            }
            __syncthreads();
            for (int i = tid; i < n; i += blockDim.x) {
                const int r = i % 3, b3 = i - r;
                const double fl1 = K1[3 * r] * R[b3] + K1[3 * r + 1] * R[b3 + 1] + K1[3 * r + 2] * R[b3 + 2];
                Rp[i] = R[i] + dt * (fl1 + 0.25 * J[i]) + sqrt2inv * dW[i];
            }
            __syncthreads();
            if constexpr (kMixed) {
                // FP32 coordinates of R~ for the EV force at the predictor point
                for (int b = tid; b < N; b += blockDim.x)
                    B.pos32[b] = make_float4((float)Rp[3 * b], (float)Rp[3 * b + 1], (float)Rp[3 * b + 2], 0.f);
            }
            // upsilon (src/integrator.cpp:107-119)
            B.geometry(Rp, E, F);
            __syncthreads();
            B.explicit_force(Rp, t + dt, E, F, G, H, Cv);
            __syncthreads();
            if constexpr (kMixed) {
                // D stays the tensor at R (built once per step, src/integrator.cpp:78)
                for (int b = tid; b < N; b += blockDim.x)
                    B.pos32[b] = make_float4((float)R[3 * b], (float)R[3 * b + 1], (float)R[3 * b + 2], 0.f);
                __syncthreads();
            }
            // solve_connectors (src/integrator.cpp:125-165): its first
            // iteration's bonds are those of R~, so its first product D Fb is
            // formed here together with upsilon's D (Fe + Fe~)
            double* ups = Bv;
            double* dups = Cv;
            double* bond = E;
            double* Rprev = G;
            double* Fc = H;
            double* Fb = I;
            double* DFs = J;
            double* Rc = K;
            double* d2 = F;
            for (int b = tid; b < N - 1; b += blockDim.x)
                for (int d = 0; d < 3; ++d) bond[3 * b + d] = Rp[3 * (b + 1) + d] - Rp[3 * b + d];
            __syncthreads();
            for (int b = tid; b < N - 1; b += blockDim.x) {
                const double l = clamped_len(bond[3 * b], bond[3 * b + 1], bond[3 * b + 2]);
                const double f = connector_factor(ch, l);
                Fc[3 * b] = f * bond[3 * b];
                Fc[3 * b + 1] = f * bond[3 * b + 1];
                Fc[3 * b + 2] = f * bond[3 * b + 2];
            }
            __syncthreads();
            B.bead_forces(Fc, Fb);
            for (int i = tid; i < n; i += blockDim.x) G[i] = Fe[i] + Cv[i];
            __syncthreads();
            {
                const double* xs[2] = {G, Fb};
                double* ys[2] = {F, DFs};
                B.template apply_D_multi<2>(xs, ys);
            }
            __syncthreads();
            for (int i = tid; i < n; i += blockDim.x) {
                const int r = i % 3, b3 = i - r;
                const double fl1 = K1[3 * r] * R[b3] + K1[3 * r + 1] * R[b3 + 1] + K1[3 * r + 2] * R[b3 + 2];
                const double fl2 = K2[3 * r] * Rp[b3] + K2[3 * r + 1] * Rp[b3 + 1] + K2[3 * r + 2] * Rp[b3 + 2];
                const double flow = 0.5 * (fl1 + fl2);
                Bv[i] = R[i] + dt * (flow + 0.125 * K[i] + 0.125 * F[i]) + sqrt2inv * dW[i];
            }
            __syncthreads();
            for (int b = tid; b < N - 1; b += blockDim.x)
                for (int d = 0; d < 3; ++d) dups[3 * b + d] = ups[3 * (b + 1) + d] - ups[3 * b + d];
            for (int i = tid; i < n; i += blockDim.x) Rprev[i] = Rp[i];
            __syncthreads();
            const int max_iter = 100 * N;
            int lstat = 0;
            for (int iter = 0;; ++iter) {
                if (iter > 0) {  // (the first iteration's Fc, Fb and D Fb are formed above)
                    for (int b = tid; b < N - 1; b += blockDim.x) {
                        const double l = clamped_len(bond[3 * b], bond[3 * b + 1], bond[3 * b + 2]);
                        const double f = connector_factor(ch, l);
                        Fc[3 * b] = f * bond[3 * b];
                        Fc[3 * b + 1] = f * bond[3 * b + 1];
                        Fc[3 * b + 2] = f * bond[3 * b + 2];
                    }
                    __syncthreads();
                    B.bead_forces(Fc, Fb);
                    __syncthreads();
                    if (B.hi) {
                        B.apply_D(Fb, DFs);
                        __syncthreads();
                    }
                }
                const double* DF = B.hi ? DFs : Fb;
                const double c8 = 0.125 * dt, c4 = 0.25 * dt;
                for (int b = tid; b < N - 1; b += blockDim.x) {
                    double g[3], q[3];
                    for (int d = 0; d < 3; ++d)
                        g[d] = dups[3 * b + d] + c8 * (DF[3 * (b + 1) + d] - DF[3 * b + d]) + c4 * Fc[3 * b + d];
                    solve_connector(g, dt, ch, q, lstat);
                    bond[3 * b] = q[0];
                    bond[3 * b + 1] = q[1];
                    bond[3 * b + 2] = q[2];
                }
                __syncthreads();
                if (tid < 3) {
                    double acc = Rp[tid];
                    Rc[tid] = acc;
                    for (int b = 0; b < N - 1; ++b) {
                        acc = acc + bond[3 * b + tid];
                        Rc[3 * (b + 1) + tid] = acc;
                    }
                }
                __syncthreads();
                for (int i = tid; i < N; i += blockDim.x) {
                    const double e0 = Rc[3 * i] - Rprev[3 * i], e1 = Rc[3 * i + 1] - Rprev[3 * i + 1],
                                 e2 = Rc[3 * i + 2] - Rprev[3 * i + 2];
                    d2[i] = e0 * e0 + e1 * e1 + e2 * e2;
                }
                __syncthreads();
                if (tid == 0) {
                    double s = 0.0;
                    for (int i = 0; i < N; ++i) s += d2[i];
                    ctl.incr = sqrt(s) / N;
                    ctl.cnt[C_CORR] += 1;
                    int verdict = 0;  // 0 continue, 1 converged, 2 cap reached, 3 non-finite
                    if (ctl.incr < ch.tol) verdict = 1;
                    else if (!(ctl.incr == ctl.incr) || isinf(ctl.incr)) verdict = 3;
                    else if (iter >= max_iter) verdict = 2;
                    ctl.brk = verdict;
                }
                __syncthreads();
                const int verdict = ctl.brk;
                if (verdict != 0) {
                    __syncthreads();
                    if (tid == 0) {
                        ctl.brk = 0;
                        if (verdict == 2) {
                            ctl.status |= BDCU_ST_NONCONVERGED;
                            ctl.cnt[C_NONCONV] += 1;
                        }
                        if (verdict == 3) ctl.status |= BDCU_ST_NONFINITE;
                    }
                    __syncthreads();
                    break;
                }
                for (int i = tid; i < n; i += blockDim.x) Rprev[i] = Rc[i];
                __syncthreads();
            }
            if (lstat) atomicOr(&ctl.status, lstat);
            __syncthreads();
            if (ctl.status & BDCU_ST_FATAL_MASK) break;
            for (int i = tid; i < n; i += blockDim.x) R[i] = Rc[i];
            if (tid == 0) ctl.cnt[C_STEPS] += 1;
            t += dt;
            __syncthreads();
            if constexpr (!kMixed) {
                // D (and a factor made this step) are dead until the next
                // step rebuilds them: drop their L2 lines unwritten
                if (B.hi && !a.d_in_smem) discard_l2(B.D, (int64_t)n * B.ldd);
                if (chol_used) discard_l2(B.Lt, (int64_t)n * B.ldl);
                __syncthreads();
            }
        }
        __syncthreads();
        // write back: positions (unless the chain failed), RNG, cache flag, status, counters
        if (!(ctl.status & BDCU_ST_FATAL_MASK))
            for (int i = tid; i < n; i += blockDim.x) gR[i] = R[i];
        if (tid == 0) {
            a.rng[3 * c] = ix;
            a.rng[3 * c + 1] = iy;
            a.rng[3 * c + 2] = iseed;
            a.cache_valid[c] = ctl.cache_valid;
            a.status[c] = ctl.status;
            int64_t* cc = reinterpret_cast<int64_t*>(a.counters + c);
            for (int k = 0; k < 8; ++k) cc[k] += ctl.cnt[k];
            if (a.steps_done) a.steps_done[c] = step;
            if (a.t_end) a.t_end[c] = t;
        }
        __syncthreads();
    }
}

}  // namespace bdcu
