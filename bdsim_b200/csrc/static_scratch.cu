// static_scratch.cu -- bdcu_run_static: the integrator for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: a host application whose memory pool
// already owns all of the GPU's memory, or a serving loop that must never take
// the implicit device-wide synchronisation cudaMalloc/cudaFree imply. For them
// this entry point runs the same integrator kernel as bdcu_run, but every
// device buffer it needs beyond the caller's inputs and outputs -- the chain
// parameter records, the parameter arena, the Lanczos seed table, the work
// queue counter and the per-block scratch -- lives in one file-scope
// `static __device__` array of kStaticScratchBytes. Every GPU that loads the
// library holds that array until the process exits.
//
// Host code sees only a stand-in for the array's name; its device address is
// taken once per device with cudaGetSymbolAddress (the first call on a device
// does it; make that first call before any stream capture on the device).
// Every call shares the array and it keeps the last call's contents: the work
// counter is cleared on each call, and everything else is written before it
// is read. Calls that overlap on the GPU (two streams, two host threads) race
// on the array and must be serialised by the caller.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "ctx.h"
#include "integrator.cuh"
#include "warp_layout.h"

namespace bdcu {
cudaError_t launch_plain(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s);
cudaError_t launch_mixed(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s);
cudaError_t occupancy_plain(int block, size_t smem, int* per_sm);
cudaError_t occupancy_mixed(int block, size_t smem, int* per_sm);
cudaError_t launch_mixed_warp(const RunArgs& a, int grid, size_t smem, cudaStream_t s);
cudaError_t occupancy_mixed_warp(size_t smem, int* per_sm);
DevChain derive_record(const bdcu_phys& p, const bdcu_sim& s, int64_t bead_off);
}  // namespace bdcu

using namespace bdcu;

namespace {

constexpr size_t kStaticScratchBytes = (size_t)BDCU_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_static_addr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device (taken once).
cudaError_t static_base(int device, void** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_static_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_static_addr[device] = p;
    }
    *out = g_static_addr[device];
    return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

int fail(bdcu_ctx* c, int code, const std::string& msg) {
    c->err = msg;
    return code;
}

// The one-chain-per-warp mixed form, as bdcu_run dispatches it; the RNG
// jump-ahead rows k = 0..n_max it reads are staged into the array too.
int run_static_warp(bdcu_ctx* ctx, int n_chains, const std::vector<DevChain>& recs, const std::vector<double>& seed,
                    const double* arena, int64_t arena_len, int n_max, int any_hi, int any_cheb, double* R,
                    int32_t* rng, double* cache, int32_t* cache_valid, const double* t_start,
                    const int32_t* n_steps, int32_t* status, bdcu_counters* counters, int cache_mode) {
    const size_t smem = (size_t)warp_smem_bytes(n_max);
    if (smem > ctx->max_smem) return fail(ctx, BDCU_E_LIMIT, "bdcu_run_static: warp kernel shared memory too large");
    int per_sm = 0;
    cudaError_t e = occupancy_mixed_warp(smem, &per_sm);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("occupancy query: ") + cudaGetErrorString(e));
    if (per_sm < 1) per_sm = 1;
    std::vector<uint32_t> cols((size_t)(n_max + 1) * 32);
    std::vector<uint32_t> apow(n_max + 1);
    for (int i = 0; i < 32; ++i) cols[i] = 1u << i;
    apow[0] = 1;
    for (int k = 1; k <= n_max; ++k) {
        for (int i = 0; i < 32; ++i) {
            uint32_t u = cols[(size_t)(k - 1) * 32 + i];
            u ^= (u << 13);
            u ^= (u >> 17);
            u ^= (u << 5);
            cols[(size_t)k * 32 + i] = u;
        }
        apow[k] = (uint32_t)(((uint64_t)apow[k - 1] * 16807ull) % 2147483647ull);
    }
    const size_t o_cnt = 0;
    const size_t o_rec = 256;
    const size_t o_seed = align256(o_rec + sizeof(DevChain) * (size_t)n_chains);
    const size_t o_arena = align256(o_seed + sizeof(double) * (size_t)n_max);
    const size_t o_cols = align256(o_arena + sizeof(double) * (size_t)std::max<int64_t>(arena_len, 1));
    const size_t o_apow = align256(o_cols + sizeof(uint32_t) * cols.size());
    const size_t o_scr = align256(o_apow + sizeof(uint32_t) * apow.size());
    const int64_t wstride = any_hi ? warp_scratch_doubles(n_max) : 1;
    const size_t per_block = sizeof(double) * (size_t)wstride * kWarpsPerCta;
    if (o_scr + per_block > kStaticScratchBytes)
        return fail(ctx, BDCU_E_LIMIT,
                    "bdcu_run_static: needs " + std::to_string(o_scr + per_block) + " bytes of static device scratch "
                    "for this batch (parameters plus one block's scratch); the maximum is " +
                    std::to_string(kStaticScratchBytes) + " bytes. Use bdcu_run, or fewer/smaller chains.");
    int grid = std::min((n_chains + kWarpsPerCta - 1) / kWarpsPerCta, per_sm * ctx->sm_count);
    grid = (int)std::min<size_t>((size_t)grid, (kStaticScratchBytes - o_scr) / per_block);
    if (grid < 1) grid = 1;
    void* base = nullptr;
    e = static_base(ctx->device, &base);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    unsigned char* b = static_cast<unsigned char*>(base);
    cudaStream_t s = ctx->stream;
    e = cudaMemsetAsync(b + o_cnt, 0, sizeof(int32_t), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_rec, recs.data(), sizeof(DevChain) * n_chains, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_seed, seed.data(), sizeof(double) * n_max, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && arena_len > 0)
        e = cudaMemcpyAsync(b + o_arena, arena, sizeof(double) * arena_len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_cols, cols.data(), sizeof(uint32_t) * cols.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_apow, apow.data(), sizeof(uint32_t) * apow.size(), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("staging parameters: ") + cudaGetErrorString(e));
    RunArgs a;
    memset(&a, 0, sizeof(a));
    a.chains = reinterpret_cast<const DevChain*>(b + o_rec);
    a.n_chains = n_chains;
    a.n_max = n_max;
    a.arena = reinterpret_cast<const double*>(b + o_arena);
    a.seed_table = reinterpret_cast<const double*>(b + o_seed);
    a.R = R;
    a.rng = rng;
    a.cache = cache;
    a.cache_valid = cache_valid;
    a.t_start = t_start;
    a.n_steps = n_steps;
    a.status = status;
    a.counters = counters;
    a.cache_mode = cache_mode;
    a.need_chol = any_hi;
    a.need_d = any_hi;
    a.need_lz = any_cheb;
    a.work_counter = reinterpret_cast<int32_t*>(b + o_cnt);
    a.scratch = reinterpret_cast<double*>(b + o_scr);
    a.scratch_stride = wstride;
    a.xs_pow = reinterpret_cast<const uint32_t*>(b + o_cols);
    a.a_pow = reinterpret_cast<const uint32_t*>(b + o_apow);
    e = launch_mixed_warp(a, grid, smem, s);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("integrate kernel launch: ") + cudaGetErrorString(e));
    return BDCU_OK;
}

}  // namespace

extern "C" int bdcu_run_static(bdcu_ctx* ctx, int n_chains, const bdcu_phys* phys, const bdcu_sim* sim,
                               const double* arena, int64_t arena_len, double* R, int32_t* rng, double* cache,
                               int32_t* cache_valid, const double* t_start, const int32_t* n_steps,
                               int32_t* status, bdcu_counters* counters, int form, int cache_mode) {
    if (!ctx) return BDCU_E_ARG;
    if (n_chains < 1 || !phys || !sim) return fail(ctx, BDCU_E_ARG, "bdcu_run_static: need n_chains >= 1 and phys/sim");
    if (!R || !rng || !cache || !cache_valid || !t_start || !n_steps || !status || !counters)
        return fail(ctx, BDCU_E_ARG, "bdcu_run_static: null device pointer");
    if (form != BDCU_FORM_PLAIN_FP64 && form != BDCU_FORM_MIXED_FP32)
        return fail(ctx, BDCU_E_ARG, "bdcu_run_static: unknown form");
    if (arena_len < 0 || (arena_len > 0 && !arena)) return fail(ctx, BDCU_E_ARG, "bdcu_run_static: bad arena");
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return fail(ctx, BDCU_E_ARG, "bdcu_run_static: bad device");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));

    // chain records, derived on the host exactly as bdcu_set_chains derives them
    std::vector<DevChain> recs(n_chains);
    int64_t off = 0;
    int n_max = 0, any_hi = 0, any_cheb = 0;
    for (int i = 0; i < n_chains; ++i) {
        const bdcu_phys& p = phys[i];
        if (p.n_beads < 2 || p.n_beads > kMaxBeads || !(sim[i].dt > 0.0))
            return fail(ctx, BDCU_E_ARG, "bdcu_run_static: chain " + std::to_string(i) + " has bad n_beads or dt");
        if (p.spring_type < 1 || p.spring_type > 7 || p.ev_type < 0 || p.ev_type > 4)
            return fail(ctx, BDCU_E_ARG, "bdcu_run_static: chain " + std::to_string(i) + " has a bad spring/EV type");
        const int64_t nn = (int64_t)p.n_beads * p.n_beads;
        if ((p.phi_offset >= 0 && p.phi_offset + nn > arena_len) ||
            (p.flow_n_times > 0 && p.flow_offset + 10 * (int64_t)p.flow_n_times > arena_len) ||
            (p.ext_n_entries > 0 && p.ext_offset + 6 > arena_len))
            return fail(ctx, BDCU_E_ARG, "bdcu_run_static: chain " + std::to_string(i) + " tables outside the arena");
        recs[i] = derive_record(p, sim[i], off);
        off += p.n_beads;
        n_max = std::max(n_max, 3 * p.n_beads);
        if (p.hstar > 0.0) {
            any_hi = 1;
            if (p.hi_method == BDCU_HI_CHEBYSHEV) any_cheb = 1;
        }
    }
    std::vector<double> seed(n_max);
    for (int i = 0; i < n_max; ++i) seed[i] = sin(0.7654321 * (i + 1)) + 0.5;

    int any_chol_method = 0;
    for (int i = 0; i < n_chains; ++i)
        if (phys[i].hstar > 0.0 && phys[i].hi_method == BDCU_HI_CHOLESKY) any_chol_method = 1;
    if (form == BDCU_FORM_MIXED_FP32 && n_max <= kWarpMaxn && !any_chol_method)
        return run_static_warp(ctx, n_chains, recs, seed, arena, arena_len, n_max, any_hi, any_cheb, R, rng, cache,
                               cache_valid, t_start, n_steps, status, counters, cache_mode);

    // launch shape, as bdcu_run plans it
    const int mixed = (form == BDCU_FORM_MIXED_FP32);
    std::vector<int> d_opts = (!mixed && any_hi) ? std::vector<int>{1, 0} : std::vector<int>{0};
    std::vector<int> v_opts = any_cheb ? std::vector<int>{kLanczosCold, kLanczosWarm, 0} : std::vector<int>{0};
    int dsm = -1, vcap = 0;
    size_t smem = 0;
    for (int d : d_opts) {
        for (int v : v_opts) {
            const size_t b = (size_t)smem_layout(n_max, d, v, mixed).total * sizeof(double);
            if (b <= ctx->max_smem) {
                dsm = d;
                vcap = v;
                smem = b;
                break;
            }
        }
        if (dsm >= 0) break;
    }
    if (dsm < 0) return fail(ctx, BDCU_E_LIMIT, "bdcu_run_static: chain too large for the shared-memory layout");
    int block = ((std::min(n_max, 512) + 31) / 32) * 32;
    if (block < 64) block = 64;
    const ScratchLayout scl = scratch_layout(n_max, dsm, vcap, any_hi, mixed, any_hi, any_cheb);
    int per_sm = 0;
    e = mixed ? occupancy_mixed(block, smem, &per_sm) : occupancy_plain(block, smem, &per_sm);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("occupancy query: ") + cudaGetErrorString(e));
    if (per_sm < 1) per_sm = 1;

    // layout of the static array: counter | records | seed table | arena | per-block scratch
    const size_t o_cnt = 0;
    const size_t o_rec = 256;
    const size_t o_seed = align256(o_rec + sizeof(DevChain) * (size_t)n_chains);
    const size_t o_arena = align256(o_seed + sizeof(double) * (size_t)n_max);
    const size_t o_scr = align256(o_arena + sizeof(double) * (size_t)std::max<int64_t>(arena_len, 1));
    const size_t stride = sizeof(double) * (size_t)std::max<int64_t>(scl.total, 1);
    if (o_scr + stride > kStaticScratchBytes)
        return fail(ctx, BDCU_E_LIMIT,
                    "bdcu_run_static: needs " + std::to_string(o_scr + stride) + " bytes of static device scratch "
                    "for this batch (parameters plus one block's scratch); the maximum is " +
                    std::to_string(kStaticScratchBytes) + " bytes. Use bdcu_run, or fewer/smaller chains.");
    int grid = std::min(n_chains, per_sm * ctx->sm_count);
    grid = (int)std::min<size_t>((size_t)grid, (kStaticScratchBytes - o_scr) / stride);
    if (grid < 1) grid = 1;

    void* base = nullptr;
    e = static_base(ctx->device, &base);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    unsigned char* b = static_cast<unsigned char*>(base);
    cudaStream_t s = ctx->stream;
    e = cudaMemsetAsync(b + o_cnt, 0, sizeof(int32_t), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_rec, recs.data(), sizeof(DevChain) * n_chains, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_seed, seed.data(), sizeof(double) * n_max, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && arena_len > 0)
        e = cudaMemcpyAsync(b + o_arena, arena, sizeof(double) * arena_len, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("staging parameters: ") + cudaGetErrorString(e));

    RunArgs a;
    memset(&a, 0, sizeof(a));
    a.chains = reinterpret_cast<const DevChain*>(b + o_rec);
    a.n_chains = n_chains;
    a.n_max = n_max;
    a.arena = reinterpret_cast<const double*>(b + o_arena);
    a.seed_table = reinterpret_cast<const double*>(b + o_seed);
    a.R = R;
    a.rng = rng;
    a.cache = cache;
    a.cache_valid = cache_valid;
    a.t_start = t_start;
    a.n_steps = n_steps;
    a.status = status;
    a.counters = counters;
    a.cache_mode = cache_mode;
    a.d_in_smem = dsm;
    a.v_cap = vcap;
    a.need_chol = any_hi;
    a.need_d = any_hi;
    a.need_lz = any_cheb;
    a.work_counter = reinterpret_cast<int32_t*>(b + o_cnt);
    a.scratch = reinterpret_cast<double*>(b + o_scr);
    a.scratch_stride = std::max<int64_t>(scl.total, 1);
    e = mixed ? launch_mixed(a, grid, block, smem, s) : launch_plain(a, grid, block, smem, s);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("integrate kernel launch: ") + cudaGetErrorString(e));
    return BDCU_OK;
}
