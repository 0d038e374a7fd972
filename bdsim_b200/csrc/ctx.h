// ctx.h -- the bdcu_ctx record behind the opaque handle of bdsim_cuda.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <deque>
#include <string>
#include <utility>
#include <vector>

#include "bdcu_internal.h"

using bdcu::DevChain;

namespace bdcu {

// Buckets of a launch plan. Buckets 0..3 run the team kernel (FP32-mixed
// form, no Cholesky method) with 1, 2, 4 and 8 warps per chain for N <= 64,
// 128, 256 and 512; buckets 4..7 run one chain per block and split the rest by
// bead count at 64, 128 and 256.
constexpr int kMaxBuckets = 8;
constexpr int kFirstBlockBucket = 4;
constexpr int kBucketBeads[kMaxBuckets] = {64, 128, 256, 512, 64, 128, 256, kMaxBeads};

// A launch shape chosen by bdcu_autotune. Block kernel: threads per block,
// Lanczos vectors in shared memory, dense D in shared memory. Team kernel:
// warps per team and beads per thread.
struct Shape {
    int block = 0;  // 0: not tuned
    int v_cap = -1;
    int d_in_smem = -1;
    int team_warps = 0;
    int team_q = 0;
};

struct Bucket {
    int id = 0;
    int kernel = BDCU_KERNEL_BLOCK;
    int team_warps = 0;  // team kernel: warps per chain
    int team_q = 0;      // team kernel: beads per thread
    int count = 0, min_beads = 0, max_beads = 0;
    int n_max = 0;  // 3 * max_beads
    int need_chol = 0, need_d = 0, need_lz = 0;
    int64_t order_off = 0;  // first entry of this bucket's work list in order_d
    int block = 0, grid = 0, v_cap = 0, d_in_smem = 0, tuned = 0;
    size_t smem = 0;
    int64_t scratch_stride = 1;  // doubles per block (per warp)
};

// A ring of pinned host memory for asynchronous uploads. Each upload takes the
// next free region and records an event after its copy; a region is reused
// only once its event has completed, so the stream never reads memory the host
// is rewriting and the host waits only when the ring is full.
struct Staging {
    unsigned char* p = nullptr;
    size_t bytes = 0;
    size_t head = 0;
    std::deque<std::pair<std::pair<size_t, size_t>, cudaEvent_t>> inflight;  // (start, end), event
    std::vector<cudaEvent_t> spare;
};

}  // namespace bdcu

struct bdcu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int n_chains = 0;  // records (chains, or slots of a pool)
    int n_max = 0;     // largest 3N among the records
    int64_t total_beads = 0;
    int any_hi = 0, any_cheb = 0, need_chol = 0, any_chol_method = 0;
    // pool mode (bdcu_reserve): records change between runs, bead offsets are given
    int pool = 0;
    int64_t bead_capacity = 0;
    int64_t arena_len = 0;
    std::vector<double> arena_h;  // host mirror of the arena (validation)
    uint32_t* xs_pow_d = nullptr;  // RNG jump-ahead tables (uploaded once)
    uint32_t* a_pow_d = nullptr;
    std::vector<DevChain> chains_h;
    std::vector<bdcu_sim> sims_h;
    std::vector<double> seed_norm_h;  // seed_norm_h[n] = |default_seed(n)|, summed in order
    DevChain* chains_d = nullptr;
    double* arena_d = nullptr;
    double* seed_d = nullptr;
    int seed_len = 0;
    int32_t* work_d = nullptr;  // one queue counter per bucket
    int sm_count = 148;
    int bounds_every = 1;  // bdcu_set_bounds_refresh
    int single_launch = 0; // bdcu_set_single_launch: every team-kernel chain in one launch
    size_t max_smem = 0;
    // the chains bdcu_run advances: all records (sel_all) or a list (bdcu_select)
    int sel_all = 1;
    std::vector<int32_t> sel;
    // the cached launch plan for plan_form
    int plan_form = -1;
    int plan_dirty = 1;
    std::vector<bdcu::Bucket> plan;
    std::vector<int32_t> order_h;
    bdcu::Staging order_stage, rec_stage, arena_stage;
    void* rec_dev = nullptr;  // device copies of staged records and slot ids
    size_t rec_dev_bytes = 0;
    int32_t* order_d = nullptr;
    size_t order_bytes = 0;
    double* bscratch[bdcu::kMaxBuckets] = {};
    size_t bscratch_bytes[bdcu::kMaxBuckets] = {};
    cudaStream_t aux[bdcu::kMaxBuckets] = {};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[bdcu::kMaxBuckets] = {};
    bdcu::Shape tuned[2][bdcu::kMaxBuckets];
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
