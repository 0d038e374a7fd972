// api.cu -- host side of the C ABI (include/bdsim_cuda.h): contexts, the
// per-chain parameter derivation, launch configuration and the
// reference-facing host-buffer integrate.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "bdcu_internal.h"
#include "integrator.cuh"
#include "warp_layout.h"

namespace bdcu {
cudaError_t launch_plain(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s);
cudaError_t launch_mixed(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s);
cudaError_t occupancy_plain(int block, size_t smem, int* per_sm);
cudaError_t occupancy_mixed(int block, size_t smem, int* per_sm);
cudaError_t launch_mixed_warp(const RunArgs& a, int grid, size_t smem, cudaStream_t s);
cudaError_t occupancy_mixed_warp(size_t smem, int* per_sm);
cudaError_t launch_forces(const DevChain* chains, int n_chains, int n_max, const double* arena, const double* R,
                          double t, int which, double* F, cudaStream_t s);
cudaError_t launch_ran1(int n_chains, int32_t* rng, int n_per, double* out, cudaStream_t s);
}  // namespace bdcu

using namespace bdcu;

#include "ctx.h"

namespace {

int fail(bdcu_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(bdcu_ctx* c, cudaError_t e, const char* where) {
    return fail(c, BDCU_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

// The constants of ExcludedVolume's constructor (src/excluded_volume.cpp:14-34),
// the spring's reduced natural length (src/spring.hpp:18), and the norm of
// default_seed(3N) (src/hydrodynamics.cpp:83-87), all with the host libm in the
// reference's operation order.
DevChain derive(const bdcu_phys& p, const bdcu_sim& s, int64_t bead_off) {
    DevChain c;
    memset(&c, 0, sizeof(c));
    c.bead_off = bead_off;
    c.N = p.n_beads;
    c.spring_type = p.spring_type;
    c.sqrtb = p.sqrtb;
    c.q0 = p.natural_length / p.sqrtb;
    c.ev_type = p.ev_type;
    c.cd = p.contour_dist_for_ev;
    c.equil = p.equilibration ? 1 : 0;
    c.bend_type = p.bend_type;
    c.C = p.bend_stiffness;
    const double z = p.zstar, d = p.dstar;
    c.zsbyds5 = z / pow(d, 5.0);
    c.pt5bydssq = 0.5 / (d * d);
    c.LJa = 12.0 * 4.0 * z * pow(d, 12.0);
    c.LJb = 6.0 * 4.0 * z * pow(d, 6.0);
    c.SDKa = 12.0 * 4.0 * pow(d, 12.0);
    c.SDKb = 6.0 * 4.0 * pow(d, 6.0);
    c.Rmin = p.min_cutoff;
    c.Rcutp = p.max_cutoff;
    c.RcutpSDK = p.max_cutoff;
    c.Rcutg = d * pow(2.0, 1.0 / 6.0);
    c.lj_rmin_fac = c.LJa / pow(c.Rmin, 14.0) - c.LJb / pow(c.Rmin, 8.0);
    c.sdk_rmin_fac = c.SDKa / pow(c.Rmin, 14.0) - c.SDKb / pow(c.Rmin, 8.0);
    c.phi_off = p.phi_offset;
    c.hstar = p.hstar;
    c.hi_method = p.hi_method;
    c.flow_n = p.flow_n_times;
    c.mult = p.ncheb_multiplier;
    c.fd_tol = p.fd_err_max;
    for (int k = 0; k < 9; ++k) c.K0[k] = p.flow_kappa[k];
    c.flow_off = p.flow_offset;
    c.ext_n = p.ext_n_entries;
    c.ext_off = p.ext_offset;
    c.update_com = s.update_center_of_mass ? 1 : 0;
    c.dt = s.dt;
    c.tol = s.implicit_loop_tol;
    double ss = 0.0;
    for (int i = 0; i < 3 * p.n_beads; ++i) {
        const double v = sin(0.7654321 * (i + 1)) + 0.5;
        ss += v * v;
    }
    c.seed_norm = sqrt(ss);
    c.bad_param = 0;
    if (p.hstar > 0.0 && p.hi_method == BDCU_HI_EXACT_SQRT) c.bad_param = 1;
    if (p.spring_type == BDCU_SPRING_WLC_BOUNDED && c.q0 > 1.0) c.bad_param = 1;
    return c;
}

template <typename T>
int ensure(bdcu_ctx* ctx, T** p, size_t count, size_t* cap_bytes = nullptr) {
    const size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
    if (cap_bytes) {
        if (*p && *cap_bytes >= bytes) return BDCU_OK;
        if (*p) cudaFree(*p);
        *p = nullptr;
        *cap_bytes = 0;
    } else if (*p) {
        cudaFree(*p);
        *p = nullptr;
    }
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if (cap_bytes) *cap_bytes = bytes;
    return BDCU_OK;
}

struct LaunchPlan {
    int grid, block;
    size_t smem;
    int d_in_smem, v_cap;
    ScratchLayout scl;
};

int plan_launch(bdcu_ctx* ctx, int form, LaunchPlan* pl) {
    const int mixed = (form == BDCU_FORM_MIXED_FP32);
    const int n = ctx->n_max;
    // Prefer D in shared memory (plain form with HI), then as many Lanczos
    // basis vectors in shared memory as fit (all 30, the 8 of a warm start, none).
    std::vector<int> d_opts = (!mixed && ctx->any_hi) ? std::vector<int>{1, 0} : std::vector<int>{0};
    std::vector<int> v_opts = ctx->any_cheb ? std::vector<int>{kLanczosCold, kLanczosWarm, 0} : std::vector<int>{0};
    bool found = false;
    for (int dsm : d_opts) {
        for (int vc : v_opts) {
            const size_t bytes = (size_t)smem_layout(n, dsm, vc, mixed).total * sizeof(double);
            if (bytes <= ctx->max_smem) {
                pl->d_in_smem = dsm;
                pl->v_cap = vc;
                pl->smem = bytes;
                found = true;
                break;
            }
        }
        if (found) break;
    }
    if (!found) return fail(ctx, BDCU_E_LIMIT, "chain too large for the shared-memory layout");
    int block = ((std::min(n, 512) + 31) / 32) * 32;
    if (block < 64) block = 64;
    pl->block = block;
    pl->scl = scratch_layout(n, pl->d_in_smem, pl->v_cap, ctx->need_chol, mixed, ctx->any_hi, ctx->any_cheb);
    int per_sm = 0;
    cudaError_t e;
    // (the kernels are instantiated only in their own translation units:
    // the plain form's must keep --fmad=false)
    e = mixed ? occupancy_mixed(block, pl->smem, &per_sm) : occupancy_plain(block, pl->smem, &per_sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) per_sm = 1;
    pl->grid = std::min(ctx->n_chains, per_sm * ctx->sm_count);
    if (pl->grid < 1) pl->grid = 1;
    return BDCU_OK;
}

// The FP32-mixed form for batches of chains with N <= 64 (no Cholesky-method
// chains): one chain per warp (integrator_warp.cuh).
int run_mixed_warp(bdcu_ctx* ctx, double* R, int32_t* rng, double* cache, int32_t* cache_valid,
                   const double* t_start, const int32_t* n_steps, int32_t* status, bdcu_counters* counters,
                   int cache_mode) {
    const size_t smem = (size_t)warp_smem_bytes(ctx->n_max);
    if (smem > ctx->max_smem) return fail(ctx, BDCU_E_LIMIT, "warp kernel shared memory exceeds the device limit");
    int per_sm = 0;
    cudaError_t e = occupancy_mixed_warp(smem, &per_sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "occupancy_mixed_warp");
    if (per_sm < 1) per_sm = 1;
    const int blocks_needed = (ctx->n_chains + kWarpsPerCta - 1) / kWarpsPerCta;
    const int grid = std::max(1, std::min(blocks_needed, per_sm * ctx->sm_count));
    const int64_t stride = ctx->any_hi ? warp_scratch_doubles(ctx->n_max) : 1;
    const size_t sdoubles = (size_t)stride * grid * kWarpsPerCta;
    int rc = ensure(ctx, &ctx->scratch_d, sdoubles, &ctx->scratch_bytes);
    if (rc) return rc;
    RunArgs a;
    memset(&a, 0, sizeof(a));
    a.chains = ctx->chains_d;
    a.n_chains = ctx->n_chains;
    a.n_max = ctx->n_max;
    a.arena = ctx->arena_d;
    a.seed_table = ctx->seed_d;
    a.R = R;
    a.rng = rng;
    a.cache = cache;
    a.cache_valid = cache_valid;
    a.t_start = t_start;
    a.n_steps = n_steps;
    a.status = status;
    a.counters = counters;
    a.cache_mode = cache_mode;
    a.need_chol = ctx->need_chol;
    a.need_d = ctx->any_hi;
    a.need_lz = ctx->any_cheb;
    a.work_counter = ctx->work_d;
    a.scratch = ctx->scratch_d;
    a.scratch_stride = stride;
    a.xs_pow = ctx->xs_pow_d;
    a.a_pow = ctx->a_pow_d;
    CK(cudaMemsetAsync(ctx->work_d, 0, sizeof(int32_t), ctx->stream));
    e = launch_mixed_warp(a, grid, smem, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "integrate_warp_kernel launch");
    return BDCU_OK;
}

}  // namespace

extern "C" {

const char* bdcu_version(void) { return "bdsim_b200 0.1 (sm_100a)"; }

int bdcu_create(int device, bdcu_ctx** out) {
    if (!out) return BDCU_E_ARG;
    bdcu_ctx* ctx = new bdcu_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete ctx;
        *out = nullptr;
        return BDCU_E_CUDA;
    }
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    if (v > 0) ctx->sm_count = v;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    ctx->max_smem = v > 0 ? (size_t)v : 232448;
    *out = ctx;
    return BDCU_OK;
}

int bdcu_destroy(bdcu_ctx* ctx) {
    if (!ctx) return BDCU_OK;
    cudaSetDevice(ctx->device);
    void* ptrs[] = {ctx->chains_d, ctx->arena_d, ctx->seed_d, ctx->work_d, ctx->scratch_d, ctx->hR, ctx->hrng,
                    ctx->hcache, ctx->hvalid, ctx->ht0, ctx->hsteps, ctx->hstatus, ctx->hcnt, ctx->xs_pow_d,
                    ctx->a_pow_d};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete ctx;
    return BDCU_OK;
}

int bdcu_set_stream(bdcu_ctx* ctx, void* stream) {
    if (!ctx) return BDCU_E_ARG;
    ctx->stream = static_cast<cudaStream_t>(stream);
    return BDCU_OK;
}

const char* bdcu_last_error(bdcu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int bdcu_count_steps(const bdcu_sim* sim, int64_t* n_steps_out) {
    if (!sim || !n_steps_out || !(sim->dt > 0.0)) return BDCU_E_ARG;
    int64_t n = 0;
    for (double t = sim->time_start; t <= sim->time_end + sim->dt / 2.0; t += sim->dt) {
        ++n;
        if (n > ((int64_t)1 << 40)) return BDCU_E_LIMIT;
    }
    *n_steps_out = n;
    return BDCU_OK;
}

int bdcu_set_chains(bdcu_ctx* ctx, int n_chains, const bdcu_phys* phys, const bdcu_sim* sim, const double* arena,
                    int64_t arena_len) {
    if (!ctx) return BDCU_E_ARG;
    if (n_chains < 1 || !phys || !sim) return fail(ctx, BDCU_E_ARG, "need n_chains >= 1 and phys/sim records");
    CK(cudaSetDevice(ctx->device));
    ctx->chains_h.resize(n_chains);
    ctx->sims_h.assign(sim, sim + n_chains);
    int64_t off = 0;
    int n_max = 0, any_hi = 0, any_cheb = 0, need_chol = 0, any_chol_method = 0;
    for (int i = 0; i < n_chains; ++i) {
        const bdcu_phys& p = phys[i];
        if (p.n_beads < 2 || p.n_beads > kMaxBeads)
            return fail(ctx, BDCU_E_LIMIT, "chain " + std::to_string(i) + ": n_beads must be in [2, " +
                                               std::to_string(kMaxBeads) + "]");
        if (!(sim[i].dt > 0.0)) return fail(ctx, BDCU_E_ARG, "chain " + std::to_string(i) + ": dt must be > 0");
        if (p.spring_type < 1 || p.spring_type > 7) return fail(ctx, BDCU_E_ARG, "invalid spring type");
        if (p.ev_type < 0 || p.ev_type > 4) return fail(ctx, BDCU_E_ARG, "invalid EV type");
        const int64_t nn = (int64_t)p.n_beads * p.n_beads;
        if (p.phi_offset >= 0 && (!arena || p.phi_offset + nn > arena_len))
            return fail(ctx, BDCU_E_ARG, "phi table outside the arena");
        if (p.flow_n_times > 0 && (!arena || p.flow_offset + 10 * (int64_t)p.flow_n_times > arena_len))
            return fail(ctx, BDCU_E_ARG, "flow table outside the arena");
        if (p.ext_n_entries > 0) {
            int64_t o = p.ext_offset;
            for (int k = 0; k < p.ext_n_entries; ++k) {
                if (!arena || o + 6 > arena_len) return fail(ctx, BDCU_E_ARG, "external force list outside the arena");
                const int64_t nt = (int64_t)arena[o + 5];
                o += 6 + 4 * nt;
                if (o > arena_len) return fail(ctx, BDCU_E_ARG, "external force list outside the arena");
            }
        }
        ctx->chains_h[i] = derive(p, sim[i], off);
        off += p.n_beads;
        n_max = std::max(n_max, 3 * p.n_beads);
        if (p.hstar > 0.0) {
            any_hi = 1;
            need_chol = 1;  // Cholesky method, or the Chebyshev fallback
            if (p.hi_method == BDCU_HI_CHEBYSHEV) any_cheb = 1;
            if (p.hi_method == BDCU_HI_CHOLESKY) any_chol_method = 1;
        }
    }
    ctx->n_chains = n_chains;
    ctx->any_chol_method = any_chol_method;
    ctx->n_max = n_max;
    ctx->total_beads = off;
    ctx->any_hi = any_hi;
    ctx->any_cheb = any_cheb;
    ctx->need_chol = need_chol;
    int rc;
    if ((rc = ensure(ctx, &ctx->chains_d, n_chains))) return rc;
    CK(cudaMemcpy(ctx->chains_d, ctx->chains_h.data(), sizeof(DevChain) * n_chains, cudaMemcpyHostToDevice));
    if ((rc = ensure(ctx, &ctx->arena_d, arena_len > 0 ? arena_len : 1))) return rc;
    if (arena_len > 0 && arena)
        CK(cudaMemcpy(ctx->arena_d, arena, sizeof(double) * arena_len, cudaMemcpyHostToDevice));
    if (n_max > ctx->seed_len) {
        std::vector<double> seed(n_max);
        for (int i = 0; i < n_max; ++i) seed[i] = sin(0.7654321 * (i + 1)) + 0.5;  // default_seed
        if ((rc = ensure(ctx, &ctx->seed_d, n_max))) return rc;
        CK(cudaMemcpy(ctx->seed_d, seed.data(), sizeof(double) * n_max, cudaMemcpyHostToDevice));
        ctx->seed_len = n_max;
    }
    if (!ctx->work_d)
        if ((rc = ensure(ctx, &ctx->work_d, 1))) return rc;
    if (!ctx->xs_pow_d) {
        // RNG jump-ahead tables: columns of M^k for the xorshift step M
        // (ux ^= ux<<13; ux ^= ux>>17; ux ^= ux<<5, linear over GF(2)) and
        // 16807^k mod (2^31-1), k = 0..kMaxDraws
        std::vector<uint32_t> cols((size_t)(kMaxDraws + 1) * 32);
        std::vector<uint32_t> apow(kMaxDraws + 1);
        for (int i = 0; i < 32; ++i) cols[i] = 1u << i;
        apow[0] = 1;
        for (int k = 1; k <= kMaxDraws; ++k) {
            for (int i = 0; i < 32; ++i) {
                uint32_t u = cols[(size_t)(k - 1) * 32 + i];
                u ^= (u << 13);
                u ^= (u >> 17);
                u ^= (u << 5);
                cols[(size_t)k * 32 + i] = u;
            }
            apow[k] = (uint32_t)(((uint64_t)apow[k - 1] * 16807ull) % 2147483647ull);
        }
        if ((rc = ensure(ctx, &ctx->xs_pow_d, cols.size()))) return rc;
        if ((rc = ensure(ctx, &ctx->a_pow_d, apow.size()))) return rc;
        CK(cudaMemcpy(ctx->xs_pow_d, cols.data(), sizeof(uint32_t) * cols.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ctx->a_pow_d, apow.data(), sizeof(uint32_t) * apow.size(), cudaMemcpyHostToDevice));
    }
    return BDCU_OK;
}

int bdcu_run(bdcu_ctx* ctx, double* R, int32_t* rng, double* cache, int32_t* cache_valid, const double* t_start,
             const int32_t* n_steps, int32_t* status, bdcu_counters* counters, int form, int cache_mode) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_run before bdcu_set_chains");
    if (!R || !rng || !cache || !cache_valid || !t_start || !n_steps || !status || !counters)
        return fail(ctx, BDCU_E_ARG, "null device pointer");
    if (form != BDCU_FORM_PLAIN_FP64 && form != BDCU_FORM_MIXED_FP32) return fail(ctx, BDCU_E_ARG, "unknown form");
    CK(cudaSetDevice(ctx->device));
    if (form == BDCU_FORM_MIXED_FP32 && ctx->n_max <= kWarpMaxn && !ctx->any_chol_method)
        return run_mixed_warp(ctx, R, rng, cache, cache_valid, t_start, n_steps, status, counters, cache_mode);
    LaunchPlan pl;
    int rc = plan_launch(ctx, form, &pl);
    if (rc) return rc;
    const size_t sbytes = sizeof(double) * (size_t)std::max<int64_t>(pl.scl.total, 1) * pl.grid;
    if ((rc = ensure(ctx, &ctx->scratch_d, sbytes / sizeof(double), &ctx->scratch_bytes))) return rc;
    RunArgs a;
    memset(&a, 0, sizeof(a));
    a.chains = ctx->chains_d;
    a.n_chains = ctx->n_chains;
    a.n_max = ctx->n_max;
    a.arena = ctx->arena_d;
    a.seed_table = ctx->seed_d;
    a.R = R;
    a.rng = rng;
    a.cache = cache;
    a.cache_valid = cache_valid;
    a.t_start = t_start;
    a.n_steps = n_steps;
    a.status = status;
    a.counters = counters;
    a.cache_mode = cache_mode;
    a.d_in_smem = pl.d_in_smem;
    a.v_cap = pl.v_cap;
    a.need_chol = ctx->need_chol;
    a.need_d = ctx->any_hi;
    a.need_lz = ctx->any_cheb;
    a.work_counter = ctx->work_d;
    a.scratch = ctx->scratch_d;
    a.scratch_stride = std::max<int64_t>(pl.scl.total, 1);
    a.xs_pow = ctx->xs_pow_d;
    a.a_pow = ctx->a_pow_d;
    CK(cudaMemsetAsync(ctx->work_d, 0, sizeof(int32_t), ctx->stream));
    cudaError_t e = (form == BDCU_FORM_MIXED_FP32) ? launch_mixed(a, pl.grid, pl.block, pl.smem, ctx->stream)
                                                   : launch_plain(a, pl.grid, pl.block, pl.smem, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "integrate kernel launch");
    return BDCU_OK;
}

int bdcu_integrate_host(bdcu_ctx* ctx, double* R_host, int32_t* rng_host, int32_t* status_host,
                        bdcu_counters* counters_host, int form) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_integrate_host before bdcu_set_chains");
    if (!R_host || !rng_host) return fail(ctx, BDCU_E_ARG, "null host pointer");
    CK(cudaSetDevice(ctx->device));
    const int nc = ctx->n_chains;
    const int64_t nb = ctx->total_beads;
    int rc;
    if (nb > ctx->hcap_beads) {
        if ((rc = ensure(ctx, &ctx->hR, 3 * nb))) return rc;
        if ((rc = ensure(ctx, &ctx->hcache, 3 * nb))) return rc;
        ctx->hcap_beads = nb;
    }
    if (nc > ctx->hcap_chains) {
        if ((rc = ensure(ctx, &ctx->hrng, 3 * nc))) return rc;
        if ((rc = ensure(ctx, &ctx->hvalid, nc))) return rc;
        if ((rc = ensure(ctx, &ctx->ht0, nc))) return rc;
        if ((rc = ensure(ctx, &ctx->hsteps, nc))) return rc;
        if ((rc = ensure(ctx, &ctx->hstatus, nc))) return rc;
        if ((rc = ensure(ctx, &ctx->hcnt, nc))) return rc;
        ctx->hcap_chains = nc;
    }
    std::vector<double> t0(nc);
    std::vector<int32_t> steps(nc);
    for (int i = 0; i < nc; ++i) {
        int64_t k = 0;
        if (bdcu_count_steps(&ctx->sims_h[i], &k) != BDCU_OK || k > 0x7fffffff)
            return fail(ctx, BDCU_E_ARG, "chain " + std::to_string(i) + ": bad time span");
        t0[i] = ctx->sims_h[i].time_start;
        steps[i] = (int32_t)k;
    }
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->hR, R_host, sizeof(double) * 3 * nb, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->hrng, rng_host, sizeof(int32_t) * 3 * nc, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->ht0, t0.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->hsteps, steps.data(), sizeof(int32_t) * nc, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(ctx->hvalid, 0, sizeof(int32_t) * nc, s));
    CK(cudaMemsetAsync(ctx->hstatus, 0, sizeof(int32_t) * nc, s));
    CK(cudaMemsetAsync(ctx->hcnt, 0, sizeof(bdcu_counters) * nc, s));
    rc = bdcu_run(ctx, ctx->hR, ctx->hrng, ctx->hcache, ctx->hvalid, ctx->ht0, ctx->hsteps, ctx->hstatus, ctx->hcnt,
                  form, BDCU_CACHE_RESET_PER_CALL);
    if (rc) return rc;
    CK(cudaMemcpyAsync(R_host, ctx->hR, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(rng_host, ctx->hrng, sizeof(int32_t) * 3 * nc, cudaMemcpyDeviceToHost, s));
    if (status_host) CK(cudaMemcpyAsync(status_host, ctx->hstatus, sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, s));
    if (counters_host)
        CK(cudaMemcpyAsync(counters_host, ctx->hcnt, sizeof(bdcu_counters) * nc, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return BDCU_OK;
}

int bdcu_forces(bdcu_ctx* ctx, const double* R, double t, int which, double* F) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_forces before bdcu_set_chains");
    if (!R || !F) return fail(ctx, BDCU_E_ARG, "null device pointer");
    if (which <= 0 || which > 15) return fail(ctx, BDCU_E_ARG, "which must OR BDCU_F_* bits");
    CK(cudaSetDevice(ctx->device));
    cudaError_t e = launch_forces(ctx->chains_d, ctx->n_chains, ctx->n_max, ctx->arena_d, R, t, which, F, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "forces kernel launch");
    return BDCU_OK;
}

int bdcu_total_force(bdcu_ctx* ctx, const double* R, double* F) {
    return bdcu_forces(ctx, R, 0.0, BDCU_F_SPRING | BDCU_F_EV | BDCU_F_BEND, F);
}

int bdcu_ran1(bdcu_ctx* ctx, int n_chains, int32_t* rng, int n_per_chain, double* out) {
    if (!ctx) return BDCU_E_ARG;
    if (n_chains < 1 || n_per_chain < 0 || !rng || !out) return fail(ctx, BDCU_E_ARG, "bad ran1 arguments");
    CK(cudaSetDevice(ctx->device));
    cudaError_t e = launch_ran1(n_chains, rng, n_per_chain, out, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ran1 kernel launch");
    return BDCU_OK;
}

}  // extern "C"

namespace bdcu {
// The per-chain record derivation, for the static-scratch entry point.
DevChain derive_record(const bdcu_phys& p, const bdcu_sim& s, int64_t bead_off) { return derive(p, s, bead_off); }
}  // namespace bdcu
