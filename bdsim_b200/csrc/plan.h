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

inline int64_t team_smem(int T, int n_max) {
    switch (T) {
        case 1: return team_smem_bytes<1>(n_max);
        case 2: return team_smem_bytes<2>(n_max);
        case 4: return team_smem_bytes<4>(n_max);
        default: return team_smem_bytes<8>(n_max);
    }
}

inline int teams_per_cta(int T) {
    return T == 1 ? TeamCfg<1>::kTeamsPerCta : T == 2 ? TeamCfg<2>::kTeamsPerCta
         : T == 4 ? TeamCfg<4>::kTeamsPerCta : TeamCfg<8>::kTeamsPerCta;
}

// Threads per block of the block kernel's heuristic shape: one thread per row
// of D up to 512.
inline int widest_block(int n_max) {
    int b = ((std::min(n_max, 512) + 31) / 32) * 32;
    return b < 64 ? 64 : b;
}

}  // namespace bdcu
