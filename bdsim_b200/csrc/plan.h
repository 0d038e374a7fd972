// plan.h -- which kernel and launch shape a chain gets: shared by bdcu_run's
// launch plans (api.cu) and the static-scratch entry point (static_scratch.cu),
// so that both run every chain on the same kernel.
#pragma once

#include <algorithm>

#include "ctx.h"
#include "team_layout.h"

namespace bdcu {

// Bucket of a chain for `form` (bucket ids as in ctx.h).
inline int bucket_of(const DevChain& c, int form) {
    const bool chol = c.hstar > 0.0 && c.hi_method == BDCU_HI_CHOLESKY;
    if (form == BDCU_FORM_MIXED_FP32 && !chol && c.N <= kTeamMaxN) {
        const int T = team_warps_for(c.N);
        return T == 1 ? 0 : T == 2 ? 1 : T == 4 ? 2 : 3;
    }
    for (int b = kFirstBlockBucket; b < kMaxBuckets - 1; ++b)
        if (c.N <= kBucketBeads[b]) return b;
    return kMaxBuckets - 1;
}

#define BDCU_TEAM_SHAPE_SWITCH(T, Q, EXPR, FALLBACK)            \
    (T == 1 && Q == 2)   ? EXPR(1, 2)                            \
    : (T == 2 && Q == 1) ? EXPR(2, 1)                            \
    : (T == 2 && Q == 2) ? EXPR(2, 2)                            \
    : (T == 4 && Q == 1) ? EXPR(4, 1)                            \
    : (T == 4 && Q == 2) ? EXPR(4, 2)                            \
    : (T == 8 && Q == 1) ? EXPR(8, 1)                            \
    : (T == 8 && Q == 2) ? EXPR(8, 2)                            \
                         : FALLBACK

// Shared memory of a team-kernel block of shape (T, Q) for chains of up to
// n_max/3 beads (-1: no such shape).
inline int64_t team_smem(int T, int Q, int n_max) {
#define BDCU_SMEM(t, q) team_smem_bytes<t, q>(n_max)
    return BDCU_TEAM_SHAPE_SWITCH(T, Q, BDCU_SMEM, (int64_t)-1);
#undef BDCU_SMEM
}

inline int teams_per_cta(int T, int Q) {
#define BDCU_TPC(t, q) TeamCfg<t, q>::kTeamsPerCta
    return BDCU_TEAM_SHAPE_SWITCH(T, Q, BDCU_TPC, 1);
#undef BDCU_TPC
}

// Whether (T, Q) is a compiled team shape that holds chains of `beads`.
inline bool team_shape_fits(int T, int Q, int beads) {
    for (int i = 0; i < kNumTeamShapes; ++i)
        if (kTeamShapes[i][0] == T && kTeamShapes[i][1] == Q) return beads <= 32 * T * Q;
    return false;
}

// Threads per block of the block kernel's heuristic shape: one thread per row
// of D up to 512.
inline int widest_block(int n_max) {
    int b = ((std::min(n_max, 512) + 31) / 32) * 32;
    return b < 64 ? 64 : b;
}

}  // namespace bdcu
