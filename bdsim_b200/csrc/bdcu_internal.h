// bdcu_internal.h -- records shared by the host API and the device kernels.
#pragma once

#include <stdint.h>

#include "../../include/bdsim_cuda.h"

namespace bdcu {

constexpr int kMaxCheb = 500;      // MAXCHEB (src/types.hpp:20)
constexpr int kLanczosCold = 30;   // src/hydrodynamics.cpp:79
constexpr int kLanczosWarm = 8;    // src/hydrodynamics.cpp:80
constexpr int kMaxBeads = 4096;    // largest chain a launch accepts

// Per-chain record derived on the host from bdcu_phys/bdcu_sim. Constants the
// reference computes with pow() in its constructors are computed here with
// the host libm, so the device sees the reference's exact values.
struct alignas(16) DevChain {
    int64_t bead_off;      // first bead of this chain in R
    int32_t N;             // beads
    int32_t spring_type;
    double sqrtb;
    double q0;             // natural_length / sqrtb (SpringParams::reduced_natural_length)
    int32_t ev_type;
    int32_t cd;            // contour_dist_for_EV
    int32_t equil;
    int32_t bend_type;
    double C;              // bending stiffness
    double zsbyds5, pt5bydssq, LJa, LJb, SDKa, SDKb;
    double Rmin, Rcutp, RcutpSDK, Rcutg;
    double lj_rmin_fac;    // LJa/pow(Rmin,14) - LJb/pow(Rmin,8)
    double sdk_rmin_fac;   // SDKa/pow(Rmin,14) - SDKb/pow(Rmin,8)
    int64_t phi_off;       // -1 => zeros
    double hstar;
    int32_t hi_method;
    int32_t flow_n;
    double mult;           // ncheb_multiplier
    double fd_tol;         // fd_err_max
    double K0[9];
    int64_t flow_off;
    int32_t ext_n;
    int32_t update_com;
    int64_t ext_off;
    double dt;
    double tol;            // implicit_loop_tol
    double seed_norm;      // sqrt(sum_i default_seed_i^2), summed in order on the host
    int32_t bad_param;     // WLCbounded sigma>1 or ExactSqrt under HI
    int32_t reserved;
};

// Everything a launch of the integrator kernel reads.
struct RunArgs {
    const DevChain* chains;
    int32_t n_chains;
    int32_t n_max;          // largest 3N in the batch
    const double* arena;
    const double* seed_table;  // default_seed(n) values, n >= n_max
    double* R;
    int32_t* rng;
    double* cache;
    int32_t* cache_valid;
    const double* t_start;
    const int32_t* n_steps;
    int32_t* status;
    bdcu_counters* counters;
    int32_t cache_mode;
    int32_t d_in_smem;      // dense D (plain form) lives in shared memory
    int32_t v_cap;          // Lanczos basis vectors that fit in shared memory
    int32_t need_chol;      // some chain may factor D (Cholesky or fallback)
    int32_t need_d;         // some chain has HI (dense D in the plain form)
    int32_t need_lz;        // some chain uses the Chebyshev method (Lanczos)
    int32_t* work_counter;  // persistent-grid chain queue (zeroed before launch)
    const int32_t* order;   // the launch's work list: chain indices, largest first (null: 0..n_work-1)
    int32_t n_work;         // entries of the work list
    double* scratch;        // per-CTA (per-team for the team kernel) global scratch
    int64_t scratch_stride; // doubles per CTA (per team)
    const uint32_t* xs_pow; // xorshift step matrix powers: columns of M^k, 32 words per k
    const uint32_t* a_pow;  // 16807^k mod (2^31 - 1)
    // time slice (bdcu_run_slice): a chain starts no new step once budget_ns
    // have passed since its thread block started (0: no budget); steps_done[c]
    // and t_end[c] (nullable) receive the steps it completed and its time.
    int64_t budget_ns;
    int32_t* steps_done;
    double* t_end;
    // FP32-mixed team kernel: spectral bounds recomputed every bounds_every
    // steps (1: every step, the reference) and whenever a step's Chebyshev
    // check fails on the kept ones
    int32_t bounds_every;
};

// Nanoseconds of the GPU's global timer.
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t v;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
    return v;
}

static_assert(sizeof(DevChain) % 8 == 0, "records are copied as doubles");

constexpr int kMaxDraws = 3 * kMaxBeads;  // jump-ahead tables cover k = 0..kMaxDraws

}  // namespace bdcu
