// team_layout.h -- sizes of the team kernel's shared and global scratch
// (integrator_team.cuh), shared by the host launch code and the kernel.
//
// A team is T warps (T = 1, 2, 4, 8) that integrate one chain of up to 32*T*Q
// beads: every thread holds Q (1 or 2) beads in registers, thread u beads u
// and u + 32T. A thread block holds kTeamsPerCta teams, each with its own
// shared-memory area and (T > 1) its own named barrier. The pair (T, Q) is the
// team shape; a bucket of chains runs one shape, chosen by bdcu_autotune or
// by default Q = 2 with the narrowest T that holds the bucket.
#pragma once

#include "integrator.cuh"

namespace bdcu {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kTeamMaxWarps = 8;
constexpr int kTeamMaxN = 64 * kTeamMaxWarps;

template <int T, int Q>
struct TeamCfg {
    static_assert(Q == 1 || Q == 2, "one or two beads per thread");
    static constexpr int kThreads = 32 * T;
    static constexpr int kMaxN = 32 * T * Q;
    static constexpr int kMaxn = 3 * kMaxN;
    static constexpr int kTeamsPerCta = T == 1 ? 4 : (T == 2 ? 2 : 1);
    static constexpr int kCtaThreads = kThreads * kTeamsPerCta;
    // blocks per SM the register allocation is sized for: two per SM (255
    // registers per thread) for every shape narrower than 8 warps. One bead
    // per thread would fit three blocks at 168 registers, but spills; two
    // blocks without spills measured 6.5% faster for (2,1) at N = 50
    static constexpr int kMinBlocks = T == 8 ? 1 : 2;
};

// Per-team shared memory (fixed part). The warm Lanczos basis
// (kLanczosWarm x nv doubles) follows it; the Chebyshev node and coefficient
// tables (2 x kCoefCap floats) share that area, as the basis is dead once the
// spectral bounds are known.
template <int T, int Q>
struct TeamShared {
    float4 pos[32 * T * Q];   // FP32 bead coordinates of the tensor's configuration
    float ps[3][32 * T * Q];  // the same coordinates by component (x, y, z rows), for the D.x pass
    float xk[3][3][32 * T * Q];  // staged D.x inputs: product r, component d, bead
    double s0[96 * T * Q];    // FP64 neighbour-exchange buffers
    double s1[96 * T * Q];
    double s2[96 * T * Q];
    // s3 / s4 also hold the cold runs' inverse-iteration scratch (2 x 32 each)
    double s3[32 * T * Q > 64 ? 32 * T * Q : 64];
    double s4[32 * T * Q > 64 ? 32 * T * Q : 64];
    double alpha[32], beta[32], ymin[32], ymax[32];
    double red[8 * T];    // per-warp partial sums (up to 8 reduced together)
    double tot[6 * T];    // per-warp scan totals (2 bead slots x 3 components)
    double rr[2];         // extreme Ritz values
    uint32_t bu;          // RNG state handed from the last drawing thread
    int32_t bi;
    int32_t item;         // claimed chain
    int32_t flag[T];      // per-warp status bits
    DevChain ch;
};

template <int T, int Q>
__host__ __device__ inline int64_t team_area_stride(int n_max) {
    const int64_t nv = round_up8(n_max);
    int64_t area = (int64_t)kLanczosWarm * nv * 8;
    if (area < (int64_t)2 * kCoefCap * 4) area = (int64_t)2 * kCoefCap * 4;
    return (int64_t)((sizeof(TeamShared<T, Q>) + 15) / 16 * 16) + area;
}
template <int T, int Q>
__host__ __device__ inline int64_t team_smem_bytes(int n_max) {
    return team_area_stride<T, Q>(n_max) * TeamCfg<T, Q>::kTeamsPerCta;
}

// Per-team global scratch (doubles): cold Lanczos basis, Cholesky factor.
__host__ __device__ inline int64_t team_scratch_doubles(int n_max) {
    return (int64_t)kLanczosCold * round_up8(n_max) + (int64_t)n_max * n_max;
}

// Team width with two beads per thread for a chain of N beads, which names
// its team bucket (0: beyond the team kernel).
__host__ __device__ inline int team_warps_for(int N) {
    return N <= 64 ? 1 : N <= 128 ? 2 : N <= 256 ? 4 : N <= 512 ? 8 : 0;
}

// The team shape (warps, beads per thread) of team buckets 0..3 (N <= 64,
// 128, 256, 512) when none is tuned or pinned: one bead per thread on 2 and 4
// warps up to N = 128 (at N = 50, (2,1) ran 7.30 M chain-steps/s against 6.5 M
// for (1,2); at N = 100, (4,1) 1.78 M against 1.53 M for (2,2)), two beads per
// thread above.
constexpr int kDefaultTeamShape[4][2] = {{2, 1}, {4, 1}, {4, 2}, {8, 2}};

// The team shapes compiled into the library: (warps, beads per thread).
constexpr int kNumTeamShapes = 7;
constexpr int kTeamShapes[kNumTeamShapes][2] = {{1, 2}, {2, 1}, {2, 2}, {4, 1}, {4, 2}, {8, 1}, {8, 2}};

}  // namespace bdcu
