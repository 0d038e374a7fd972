// ctx.h -- the bdcu_ctx record behind the opaque handle of bdsim_cuda.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "bdcu_internal.h"

using bdcu::DevChain;

struct bdcu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int n_chains = 0;
    int n_max = 0;  // largest 3N
    int64_t total_beads = 0;
    int any_hi = 0, any_cheb = 0, need_chol = 0, any_chol_method = 0;
    uint32_t* xs_pow_d = nullptr;  // RNG jump-ahead tables (uploaded once)
    uint32_t* a_pow_d = nullptr;
    std::vector<DevChain> chains_h;
    std::vector<bdcu_sim> sims_h;
    DevChain* chains_d = nullptr;
    double* arena_d = nullptr;
    double* seed_d = nullptr;
    int seed_len = 0;
    int32_t* work_d = nullptr;
    double* scratch_d = nullptr;
    size_t scratch_bytes = 0;
    int sm_count = 148;
    size_t max_smem = 0;
    // buffers of bdcu_integrate_host
    double* hR = nullptr;
    int32_t* hrng = nullptr;
    double* hcache = nullptr;
    int32_t* hvalid = nullptr;
    double* ht0 = nullptr;
    int32_t* hsteps = nullptr;
    int32_t* hstatus = nullptr;
    bdcu_counters* hcnt = nullptr;
    int64_t hcap_beads = 0;
    int hcap_chains = 0;
};
