// static_scratch.cu -- bdcu_run_static: the integrator for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: a host application whose memory pool
// already owns all of the GPU's memory, or a serving loop that must never take
// the implicit device-wide synchronisation cudaMalloc/cudaFree imply. For them
// this entry point runs the same kernels as bdcu_run, bucket by bucket, but
// every device buffer it needs beyond the caller's inputs and outputs -- the
// chain parameter records, the work lists, the parameter arena, the Lanczos
// seed table, the RNG jump-ahead tables, the work queue counters and the
// per-block scratch -- lives in one file-scope
// `static __device__` array of kStaticScratchBytes. Every GPU that loads the
// library holds that array until the process exits.
//
// Host code sees only a stand-in for the array's name; its device address is
// taken once per device with cudaGetSymbolAddress (the first call on a device
// does it, and the first call after the device's context was replaced, e.g.
// by cudaDeviceReset). The entry point cannot be captured in a graph: it
// stages its records and tables from pageable host vectors freed on return.
// Every call shares the array and it keeps the last call's contents: the work
// counters are cleared on each call, and everything else is written before it
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
#include "plan.h"
#include "team_layout.h"

namespace bdcu {
cudaError_t launch_plain(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s);
cudaError_t launch_mixed(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s);
cudaError_t occupancy_plain(int block, size_t smem, int* per_sm);
cudaError_t occupancy_mixed(int block, size_t smem, int* per_sm);
cudaError_t launch_mixed_team(int team_warps, int team_q, const RunArgs& a, int grid, size_t smem, cudaStream_t s);
cudaError_t occupancy_mixed_team(int team_warps, int team_q, size_t smem, int* per_sm);
DevChain derive_record(const bdcu_phys& p, const bdcu_sim& s, int64_t bead_off);
int validate_chain(bdcu_ctx* ctx, int i, const bdcu_phys& p, const bdcu_sim& s, const double* arena,
                   int64_t arena_len);
}  // namespace bdcu

using namespace bdcu;

namespace {

constexpr size_t kStaticScratchBytes = (size_t)BDCU_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_static_addr[kMaxDevices] = {};
void* g_static_ctx[kMaxDevices] = {};

// The current CUDA context's handle (cuCtxGetCurrent, looked up through the
// runtime so the library needs no link against the driver library); null if
// unavailable.
void* current_context() {
    typedef int (*CtxGetCurrent)(void**);
    static CtxGetCurrent fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrent>(p);
    });
    void* c = nullptr;
    if (fn && fn(&c) != 0) c = nullptr;
    return c;
}

// Device address of g_static_scratch on the current device. Taken at the first
// call on a device, and again whenever the device's context has changed since
// (after cudaDeviceReset the old address belongs to a destroyed context).
cudaError_t static_base(int device, void** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    void* cur = current_context();
    if (!g_static_addr[device] || cur != g_static_ctx[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_static_addr[device] = p;
        g_static_ctx[device] = current_context();
    }
    *out = g_static_addr[device];
    return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

int fail(bdcu_ctx* c, int code, const std::string& msg) {
    c->err = msg;
    return code;
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

    // chain records: the checks bdcu_set_chains makes (every table inside the
    // arena), then the derivation bdcu_set_chains does -- all before the GPU
    // is touched
    std::vector<DevChain> recs(n_chains);
    int64_t off = 0;
    int n_max = 0;
    for (int i = 0; i < n_chains; ++i) {
        const int rc = validate_chain(ctx, i, phys[i], sim[i], arena, arena_len);
        if (rc != BDCU_OK) {
            ctx->err = "bdcu_run_static: " + ctx->err;
            return rc;
        }
        recs[i] = derive_record(phys[i], sim[i], off);
        off += phys[i].n_beads;
        n_max = std::max(n_max, 3 * phys[i].n_beads);
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    std::vector<double> seed(n_max);
    for (int i = 0; i < n_max; ++i) seed[i] = sin(0.7654321 * (i + 1)) + 0.5;

    // buckets, as bdcu_run plans them (largest chains first within a bucket)
    const int mixed = (form == BDCU_FORM_MIXED_FP32);
    std::vector<std::vector<int32_t>> lists(kMaxBuckets);
    for (int i = 0; i < n_chains; ++i) lists[bucket_of(recs[i], form)].push_back(i);
    struct Launch {
        int id, team_warps, team_q, block, grid, v_cap, d_in_smem, n_max, need_d, need_lz, count;
        size_t smem, per_block;
        int64_t stride, order_off;
    };
    std::vector<Launch> launches;
    std::vector<int32_t> order;
    bool any_team = false;
    size_t max_block_scratch = 0;
    for (int id = kMaxBuckets - 1; id >= 0; --id) {
        std::vector<int32_t>& L = lists[id];
        if (L.empty()) continue;
        std::stable_sort(L.begin(), L.end(), [&](int32_t x, int32_t y) { return recs[x].N > recs[y].N; });
        Launch l;
        memset(&l, 0, sizeof(l));
        l.id = id;
        l.count = (int)L.size();
        l.n_max = 3 * recs[L.front()].N;
        for (int32_t c : L)
            if (recs[c].hstar > 0.0) {
                l.need_d = 1;
                if (recs[c].hi_method == BDCU_HI_CHEBYSHEV) l.need_lz = 1;
            }
        l.order_off = (int64_t)order.size();
        order.insert(order.end(), L.begin(), L.end());
        int per_sm = 0;
        if (id < kFirstBlockBucket) {
            any_team = true;
            l.team_warps = kDefaultTeamShape[id][0];
            l.team_q = kDefaultTeamShape[id][1];
            l.smem = (size_t)team_smem(l.team_warps, l.team_q, l.n_max);
            if (l.smem > ctx->max_smem) return fail(ctx, BDCU_E_LIMIT, "bdcu_run_static: team kernel shared memory too large");
            e = occupancy_mixed_team(l.team_warps, l.team_q, l.smem, &per_sm);
            l.stride = l.need_d ? team_scratch_doubles(l.n_max) : 1;
            l.per_block = sizeof(double) * (size_t)l.stride * teams_per_cta(l.team_warps, l.team_q);
            l.block = 32 * l.team_warps * teams_per_cta(l.team_warps, l.team_q);
            l.grid = (l.count + teams_per_cta(l.team_warps, l.team_q) - 1) / teams_per_cta(l.team_warps, l.team_q);
        } else {
            std::vector<int> d_opts = (!mixed && l.need_d) ? std::vector<int>{1, 0} : std::vector<int>{0};
            std::vector<int> v_opts = l.need_lz ? std::vector<int>{kLanczosCold, kLanczosWarm, 0} : std::vector<int>{0};
            l.d_in_smem = -1;
            for (int d : d_opts) {
                for (int v : v_opts) {
                    const size_t bytes = (size_t)smem_layout(l.n_max, d, v, mixed).total * sizeof(double);
                    if (bytes <= ctx->max_smem) {
                        l.d_in_smem = d;
                        l.v_cap = v;
                        l.smem = bytes;
                        break;
                    }
                }
                if (l.d_in_smem >= 0) break;
            }
            if (l.d_in_smem < 0) return fail(ctx, BDCU_E_LIMIT, "bdcu_run_static: chain too large for the shared-memory layout");
            l.block = widest_block(l.n_max);
            const ScratchLayout scl = scratch_layout(l.n_max, l.d_in_smem, l.v_cap, l.need_d, mixed, l.need_d, l.need_lz);
            l.stride = std::max<int64_t>(scl.total, 1);
            l.per_block = sizeof(double) * (size_t)l.stride;
            e = mixed ? occupancy_mixed(l.block, l.smem, &per_sm) : occupancy_plain(l.block, l.smem, &per_sm);
            l.grid = l.count;
        }
        if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("occupancy query: ") + cudaGetErrorString(e));
        if (per_sm < 1) return fail(ctx, BDCU_E_LIMIT, "bdcu_run_static: kernel shape cannot be resident");
        l.grid = std::max(1, std::min(l.grid, per_sm * ctx->sm_count));
        max_block_scratch = std::max(max_block_scratch, l.per_block);
        launches.push_back(l);
    }

    // RNG jump-ahead rows k = 0..n_max for the team kernel's noise
    std::vector<uint32_t> cols, apow;
    if (any_team) {
        cols.resize((size_t)(n_max + 1) * 32);
        apow.resize(n_max + 1);
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
    }

    // layout of the static array: queue counters | records | work lists | seed
    // table | arena | jump-ahead tables | scratch (reused by each bucket in turn)
    const size_t o_cnt = 0;
    const size_t o_rec = 256;
    const size_t o_ord = align256(o_rec + sizeof(DevChain) * (size_t)n_chains);
    const size_t o_seed = align256(o_ord + sizeof(int32_t) * order.size());
    const size_t o_arena = align256(o_seed + sizeof(double) * (size_t)n_max);
    const size_t o_cols = align256(o_arena + sizeof(double) * (size_t)std::max<int64_t>(arena_len, 1));
    const size_t o_apow = align256(o_cols + sizeof(uint32_t) * cols.size());
    const size_t o_scr = align256(o_apow + sizeof(uint32_t) * apow.size());
    if (o_scr + max_block_scratch > kStaticScratchBytes)
        return fail(ctx, BDCU_E_LIMIT,
                    "bdcu_run_static: needs " + std::to_string(o_scr + max_block_scratch) +
                    " bytes of static device scratch for this batch (parameters plus one block's scratch); the "
                    "maximum is " + std::to_string(kStaticScratchBytes) + " bytes. Use bdcu_run, or fewer/smaller chains.");
    for (Launch& l : launches)
        l.grid = (int)std::max<size_t>(1, std::min<size_t>((size_t)l.grid, (kStaticScratchBytes - o_scr) / l.per_block));

    void* base = nullptr;
    e = static_base(ctx->device, &base);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    unsigned char* b = static_cast<unsigned char*>(base);
    cudaStream_t s = ctx->stream;
    e = cudaMemsetAsync(b + o_cnt, 0, sizeof(int32_t) * kMaxBuckets, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_rec, recs.data(), sizeof(DevChain) * n_chains, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_ord, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b + o_seed, seed.data(), sizeof(double) * n_max, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && arena_len > 0)
        e = cudaMemcpyAsync(b + o_arena, arena, sizeof(double) * arena_len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && any_team)
        e = cudaMemcpyAsync(b + o_cols, cols.data(), sizeof(uint32_t) * cols.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && any_team)
        e = cudaMemcpyAsync(b + o_apow, apow.data(), sizeof(uint32_t) * apow.size(), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return fail(ctx, BDCU_E_CUDA, std::string("staging parameters: ") + cudaGetErrorString(e));

    for (const Launch& l : launches) {
        RunArgs a;
        memset(&a, 0, sizeof(a));
        a.chains = reinterpret_cast<const DevChain*>(b + o_rec);
        a.n_chains = n_chains;
        a.order = reinterpret_cast<const int32_t*>(b + o_ord) + l.order_off;
        a.n_work = l.count;
        a.n_max = l.n_max;
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
        a.d_in_smem = l.d_in_smem;
        a.v_cap = l.v_cap;
        a.need_chol = l.need_d;
        a.need_d = l.need_d;
        a.need_lz = l.need_lz;
        a.work_counter = reinterpret_cast<int32_t*>(b + o_cnt) + l.id;
        a.scratch = reinterpret_cast<double*>(b + o_scr);
        a.scratch_stride = l.stride;
        a.xs_pow = reinterpret_cast<const uint32_t*>(b + o_cols);
        a.a_pow = reinterpret_cast<const uint32_t*>(b + o_apow);
        if (l.id < kFirstBlockBucket)
            e = launch_mixed_team(l.team_warps, l.team_q, a, l.grid, l.smem, s);
        else
            e = mixed ? launch_mixed(a, l.grid, l.block, l.smem, s) : launch_plain(a, l.grid, l.block, l.smem, s);
        if (e != cudaSuccess)
            return fail(ctx, BDCU_E_CUDA, std::string("integrate kernel launch: ") + cudaGetErrorString(e));
    }
    return BDCU_OK;
}
