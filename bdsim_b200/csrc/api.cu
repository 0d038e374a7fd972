// api.cu -- host side of the C ABI (include/bdsim_cuda.h): contexts, the
// per-chain parameter derivation, launch plans (buckets by bead count, device
// work lists, autotuned shapes), slot pools and the reference-facing
// host-buffer integrate.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "bdcu_internal.h"
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
cudaError_t launch_forces(const DevChain* chains, int n_chains, int n_max, const double* arena, const double* R,
                          double t, int which, double* F, cudaStream_t s);
cudaError_t launch_ran1(int n_chains, int32_t* rng, int n_per, double* out, cudaStream_t s);
cudaError_t launch_observables(const DevChain* chains, int n_chains, const double* R, const double* F, double* out,
                               cudaStream_t s);
cudaError_t launch_scatter_records(DevChain* dst, const DevChain* src, const int32_t* slots, int count,
                                   cudaStream_t s);
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
DevChain derive(const bdcu_phys& p, const bdcu_sim& s, int64_t bead_off, double seed_norm) {
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
    c.seed_norm = seed_norm;
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

// default_seed(n) (src/hydrodynamics.cpp:83-87) for n up to 3*kMaxBeads on the
// device, and the norms of its prefixes on the host: |default_seed(n)| sums
// v_0^2 .. v_{n-1}^2 in order, so the prefix sums are the reference's sums.
int ensure_tables(bdcu_ctx* ctx) {
    int rc;
    const int n_all = 3 * kMaxBeads;
    if (ctx->seed_len < n_all) {
        std::vector<double> seed(n_all);
        ctx->seed_norm_h.assign(n_all + 1, 0.0);
        double ss = 0.0;
        for (int i = 0; i < n_all; ++i) {
            const double v = sin(0.7654321 * (i + 1)) + 0.5;
            seed[i] = v;
            ss += v * v;
            ctx->seed_norm_h[i + 1] = sqrt(ss);
        }
        if ((rc = ensure(ctx, &ctx->seed_d, n_all))) return rc;
        CK(cudaMemcpy(ctx->seed_d, seed.data(), sizeof(double) * n_all, cudaMemcpyHostToDevice));
        ctx->seed_len = n_all;
    }
    if (!ctx->work_d) {
        if ((rc = ensure(ctx, &ctx->work_d, kMaxBuckets))) return rc;
        CK(cudaMemset(ctx->work_d, 0, sizeof(int32_t) * kMaxBuckets));
    }
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

// The checks bdcu_set_chains and bdcu_update_chains make on one chain record.
int validate(bdcu_ctx* ctx, int i, const bdcu_phys& p, const bdcu_sim& s, const double* arena, int64_t arena_len) {
    const std::string who = "chain " + std::to_string(i) + ": ";
    if (p.n_beads < 2 || p.n_beads > kMaxBeads)
        return fail(ctx, BDCU_E_LIMIT, who + "n_beads must be in [2, " + std::to_string(kMaxBeads) + "]");
    if (!(s.dt > 0.0)) return fail(ctx, BDCU_E_ARG, who + "dt must be > 0");
    if (p.spring_type < 1 || p.spring_type > 7) return fail(ctx, BDCU_E_ARG, who + "invalid spring type");
    if (p.ev_type < 0 || p.ev_type > 4) return fail(ctx, BDCU_E_ARG, who + "invalid EV type");
    const int64_t nn = (int64_t)p.n_beads * p.n_beads;
    if (p.phi_offset >= 0 && (!arena || p.phi_offset + nn > arena_len))
        return fail(ctx, BDCU_E_ARG, who + "phi table outside the arena");
    if (p.flow_n_times > 0 && (!arena || p.flow_offset < 0 || p.flow_offset + 10 * (int64_t)p.flow_n_times > arena_len))
        return fail(ctx, BDCU_E_ARG, who + "flow table outside the arena");
    if (p.ext_n_entries > 0) {
        int64_t o = p.ext_offset;
        for (int k = 0; k < p.ext_n_entries; ++k) {
            if (!arena || o < 0 || o + 6 > arena_len) return fail(ctx, BDCU_E_ARG, who + "external force list outside the arena");
            const int64_t nt = (int64_t)arena[o + 5];
            o += 6 + 4 * nt;
            if (nt < 0 || o > arena_len) return fail(ctx, BDCU_E_ARG, who + "external force list outside the arena");
        }
    }
    return BDCU_OK;
}

void retire_done(Staging& st) {
    while (!st.inflight.empty() && cudaEventQuery(st.inflight.front().second) == cudaSuccess) {
        st.spare.push_back(st.inflight.front().second);
        st.inflight.pop_front();
    }
}

int wait_oldest(bdcu_ctx* ctx, Staging& st) {
    CK(cudaEventSynchronize(st.inflight.front().second));
    st.spare.push_back(st.inflight.front().second);
    st.inflight.pop_front();
    return BDCU_OK;
}

// Whether [s, s+n) overlaps a region still in flight.
bool overlaps_inflight(const Staging& st, size_t s, size_t n) {
    for (const auto& r : st.inflight)
        if (s < r.first.second && r.first.first < s + n) return true;
    return false;
}

int reserve_staging(bdcu_ctx* ctx, Staging& st, size_t bytes) {
    if (st.bytes >= bytes) return BDCU_OK;
    while (!st.inflight.empty()) {
        const int rc = wait_oldest(ctx, st);
        if (rc) return rc;
    }
    if (st.p) CK(cudaFreeHost(st.p));
    st.p = nullptr;
    st.bytes = 0;
    st.head = 0;
    const size_t want = std::max<size_t>(bytes, 4096);
    CK(cudaHostAlloc(reinterpret_cast<void**>(&st.p), want, cudaHostAllocDefault));
    st.bytes = want;
    return BDCU_OK;
}

int stage_upload(bdcu_ctx* ctx, Staging& st, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return BDCU_OK;
    int rc;
    const size_t n = (bytes + 255) / 256 * 256;
    if (2 * n > st.bytes && (rc = reserve_staging(ctx, st, 4 * n))) return rc;
    retire_done(st);
    size_t s = st.head;
    for (;;) {
        if (s + n > st.bytes) s = 0;  // wrap
        if (!overlaps_inflight(st, s, n)) break;
        if ((rc = wait_oldest(ctx, st))) return rc;
    }
    memcpy(st.p + s, src, bytes);
    CK(cudaMemcpyAsync(dst, st.p + s, bytes, cudaMemcpyHostToDevice, ctx->stream));
    cudaEvent_t ev;
    if (!st.spare.empty()) {
        ev = st.spare.back();
        st.spare.pop_back();
    } else {
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    CK(cudaEventRecord(ev, ctx->stream));
    st.inflight.push_back({{s, s + n}, ev});
    st.head = s + n;
    return BDCU_OK;
}

void free_staging(Staging& st) {
    for (auto& r : st.inflight) {
        cudaEventSynchronize(r.second);
        cudaEventDestroy(r.second);
    }
    for (cudaEvent_t e : st.spare) cudaEventDestroy(e);
    if (st.p) cudaFreeHost(st.p);
    st = Staging();
}

// ------------------------------------------------------------ launch plans

// Launch shapes of the block kernel for a bucket, the heuristic's choice first:
// widest block, dense D in shared memory when it fits (plain form), then as
// many Lanczos vectors in shared memory as fit.
std::vector<Shape> block_shapes(const bdcu_ctx* ctx, const Bucket& b, int form) {
    const int mixed = form == BDCU_FORM_MIXED_FP32;
    const std::vector<int> d_opts = (!mixed && b.need_d) ? std::vector<int>{1, 0} : std::vector<int>{0};
    const std::vector<int> v_opts = b.need_lz ? std::vector<int>{kLanczosCold, kLanczosWarm, 0} : std::vector<int>{0};
    const int wide = widest_block(b.n_max);
    std::vector<int> blocks{wide};
    for (int x : {512, 256, 128, 64})
        if (x < wide) blocks.push_back(x);
    std::vector<Shape> out;
    for (int blk : blocks)
        for (int d : d_opts)
            for (int v : v_opts) {
                if ((size_t)smem_layout(b.n_max, d, v, mixed).total * sizeof(double) > ctx->max_smem) continue;
                Shape s;
                s.block = blk;
                s.v_cap = v;
                s.d_in_smem = d;
                out.push_back(s);
            }
    return out;
}

// The heuristic's shape (when none is tuned): the widest block, with D in
// shared memory unless keeping D in global memory lets more blocks share an
// SM. D in global stays L2-resident: a D that fits shared memory is at most
// ~195 KB, ~87 MB over three blocks on each of 148 SMs. Measured at
// 4096 x N=50 (plain form): D in global with three blocks per SM runs 1.7x
// the D-in-shared shape's one block per SM.
Shape default_shape(const Bucket& b, int mixed, const std::vector<Shape>& shapes) {
    const Shape& first = shapes.front();
    if (mixed || !first.d_in_smem) return first;
    for (const Shape& s : shapes) {
        if (s.block != first.block || s.d_in_smem) continue;
        int per_d = 0, per_g = 0;
        const size_t sm_d = (size_t)smem_layout(b.n_max, 1, first.v_cap, 0).total * sizeof(double);
        const size_t sm_g = (size_t)smem_layout(b.n_max, 0, s.v_cap, 0).total * sizeof(double);
        if (occupancy_plain(first.block, sm_d, &per_d) != cudaSuccess) return first;
        if (occupancy_plain(s.block, sm_g, &per_g) != cudaSuccess) return first;
        return per_g > per_d ? s : first;
    }
    return first;
}

// Fill the launch fields of a bucket for a shape (block kernel) or for the
// team kernel; 0 when the shape cannot run.
int fill_launch(bdcu_ctx* ctx, int form, Bucket& b, const Shape* s) {
    const int mixed = form == BDCU_FORM_MIXED_FP32;
    int per_sm = 0;
    cudaError_t e;
    if (b.kernel == BDCU_KERNEL_TEAM) {
        if (s && s->team_warps > 0) {
            b.team_warps = s->team_warps;
            b.team_q = s->team_q;
        }
        const int T = b.team_warps, Q = b.team_q;
        if (!team_shape_fits(T, Q, b.max_beads)) return fail(ctx, BDCU_E_ARG, "team shape does not hold the bucket");
        b.smem = (size_t)team_smem(T, Q, b.n_max);
        if (b.smem > ctx->max_smem) return fail(ctx, BDCU_E_LIMIT, "team kernel shared memory exceeds the device limit");
        e = occupancy_mixed_team(T, Q, b.smem, &per_sm);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "occupancy_mixed_team");
        if (per_sm < 1) return fail(ctx, BDCU_E_LIMIT, "team kernel cannot be resident");
        const int tpc = teams_per_cta(T, Q);
        b.block = 32 * T * tpc;
        b.grid = std::max(1, std::min((b.count + tpc - 1) / tpc, per_sm * ctx->sm_count));
        b.v_cap = 0;
        b.d_in_smem = 0;
        b.scratch_stride = b.need_d ? team_scratch_doubles(b.n_max) : 1;
        return BDCU_OK;
    }
    b.block = s->block;
    b.v_cap = s->v_cap;
    b.d_in_smem = s->d_in_smem;
    b.smem = (size_t)smem_layout(b.n_max, b.d_in_smem, b.v_cap, mixed).total * sizeof(double);
    if (b.smem > ctx->max_smem) return fail(ctx, BDCU_E_LIMIT, "chain too large for the shared-memory layout");
    e = mixed ? occupancy_mixed(b.block, b.smem, &per_sm) : occupancy_plain(b.block, b.smem, &per_sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) return fail(ctx, BDCU_E_LIMIT, "block kernel shape cannot be resident");
    b.grid = std::max(1, std::min(b.count, per_sm * ctx->sm_count));
    const ScratchLayout scl = scratch_layout(b.n_max, b.d_in_smem, b.v_cap, b.need_chol, mixed, b.need_d, b.need_lz);
    b.scratch_stride = std::max<int64_t>(scl.total, 1);
    return BDCU_OK;
}

// Grow a device buffer in stream order (cudaMallocAsync / cudaFreeAsync on the
// context stream): no device-wide synchronisation, so a serving loop that
// admits larger chains never stalls the kernels already queued.
template <typename T>
int ensure_async(bdcu_ctx* ctx, T** p, size_t count, size_t* cap_bytes) {
    const size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
    if (*p && *cap_bytes >= bytes) return BDCU_OK;
    if (*p) CK(cudaFreeAsync(*p, ctx->stream));
    *p = nullptr;
    *cap_bytes = 0;
    const size_t want = bytes + bytes / 4;  // headroom against repeated growth
    CK(cudaMallocAsync(reinterpret_cast<void**>(p), want, ctx->stream));
    *cap_bytes = want;
    return BDCU_OK;
}

int ensure_bucket_scratch(bdcu_ctx* ctx, const Bucket& b) {
    const int per = b.kernel == BDCU_KERNEL_TEAM ? teams_per_cta(b.team_warps, b.team_q) : 1;
    const size_t doubles = (size_t)b.scratch_stride * b.grid * per;
    return ensure_async(ctx, &ctx->bscratch[b.id], doubles, &ctx->bscratch_bytes[b.id]);
}

// The plan for `form` over the current selection: buckets, their work lists
// (largest chains first) uploaded to order_d, and a launch shape per bucket
// (tuned if bdcu_autotune chose one, else the heuristic's).
int build_plan(bdcu_ctx* ctx, int form) {
    if (!ctx->plan_dirty && ctx->plan_form == form) return BDCU_OK;
    const int mixed = form == BDCU_FORM_MIXED_FP32;
    std::vector<std::vector<int32_t>> lists(kMaxBuckets);
    if (ctx->sel_all) {
        for (int c = 0; c < ctx->n_chains; ++c) lists[bucket_of(ctx->chains_h[c], form)].push_back(c);
    } else {
        for (int32_t c : ctx->sel) lists[bucket_of(ctx->chains_h[c], form)].push_back(c);
    }
    if (ctx->single_launch) {
        // one persistent launch for every team-kernel chain: the widest team
        // bucket present takes the others' chains (and runs its shape)
        int top = -1;
        for (int id = 0; id < kFirstBlockBucket; ++id)
            if (!lists[id].empty()) top = id;
        for (int id = 0; id < top; ++id) {
            lists[top].insert(lists[top].end(), lists[id].begin(), lists[id].end());
            lists[id].clear();
        }
    }
    ctx->plan.clear();
    ctx->order_h.clear();
    int rc;
    // largest chains' buckets are launched first: the block kernel's, then the
    // team kernel's from the widest team down
    for (int id = kMaxBuckets - 1; id >= 0; --id) {
        std::vector<int32_t>& L = lists[id];
        if (L.empty()) continue;
        std::stable_sort(L.begin(), L.end(),
                         [&](int32_t x, int32_t y) { return ctx->chains_h[x].N > ctx->chains_h[y].N; });
        Bucket b;
        b.id = id;
        b.kernel = id < kFirstBlockBucket ? BDCU_KERNEL_TEAM : BDCU_KERNEL_BLOCK;
        b.team_warps = id < kFirstBlockBucket ? kDefaultTeamShape[id][0] : 0;
        b.team_q = id < kFirstBlockBucket ? kDefaultTeamShape[id][1] : 0;
        b.count = (int)L.size();
        b.max_beads = ctx->chains_h[L.front()].N;
        b.min_beads = ctx->chains_h[L.back()].N;
        b.n_max = 3 * b.max_beads;
        for (int32_t c : L) {
            const DevChain& ch = ctx->chains_h[c];
            if (ch.hstar > 0.0) {
                b.need_d = 1;
                b.need_chol = 1;  // Cholesky method, or the Chebyshev fallback
                if (ch.hi_method == BDCU_HI_CHEBYSHEV) b.need_lz = 1;
            }
        }
        b.order_off = (int64_t)ctx->order_h.size();
        ctx->order_h.insert(ctx->order_h.end(), L.begin(), L.end());
        if (b.kernel == BDCU_KERNEL_TEAM) {
            const Shape& t = ctx->tuned[mixed][id];
            const bool use = t.team_warps > 0 && team_shape_fits(t.team_warps, t.team_q, b.max_beads);
            if ((rc = fill_launch(ctx, form, b, use ? &t : nullptr))) return rc;
            b.tuned = use ? 1 : 0;
        } else {
            const std::vector<Shape> shapes = block_shapes(ctx, b, form);
            if (shapes.empty()) return fail(ctx, BDCU_E_LIMIT, "chain too large for the shared-memory layout");
            Shape pick = default_shape(b, mixed, shapes);
            const Shape& t = ctx->tuned[mixed][id];
            if (t.block > 0) {
                // the tuned shape, or the nearest one that still fits this bucket
                for (const Shape& s : shapes)
                    if (s.block == std::min(t.block, shapes.front().block) && s.v_cap == t.v_cap &&
                        s.d_in_smem == t.d_in_smem) {
                        pick = s;
                        b.tuned = 1;
                        break;
                    }
                if (!b.tuned)
                    for (const Shape& s : shapes)
                        if (s.block == std::min(t.block, shapes.front().block)) {
                            pick = s;
                            b.tuned = 1;
                            break;
                        }
            }
            if ((rc = fill_launch(ctx, form, b, &pick))) return rc;
        }
        if ((rc = ensure_bucket_scratch(ctx, b))) return rc;
        ctx->plan.push_back(b);
    }
    if (!ctx->order_h.empty()) {
        if ((rc = ensure_async(ctx, &ctx->order_d, ctx->order_h.size(), &ctx->order_bytes))) return rc;
        if ((rc = stage_upload(ctx, ctx->order_stage, ctx->order_d, ctx->order_h.data(),
                               sizeof(int32_t) * ctx->order_h.size())))
            return rc;
    }
    for (size_t i = 1; i < ctx->plan.size(); ++i) {
        if (!ctx->aux[i]) CK(cudaStreamCreateWithFlags(&ctx->aux[i], cudaStreamNonBlocking));
        if (!ctx->ev_join[i]) CK(cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming));
    }
    if (ctx->plan.size() > 1 && !ctx->ev_fork) CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    ctx->plan_form = form;
    ctx->plan_dirty = 0;
    return BDCU_OK;
}

struct State {
    double* R;
    int32_t* rng;
    double* cache;
    int32_t* cache_valid;
    const double* t_start;
    const int32_t* n_steps;
    int32_t* status;
    bdcu_counters* counters;
    int64_t budget_ns = 0;       // time slice (bdcu_run_slice), 0: none
    int32_t* steps_done = nullptr;
    double* t_end = nullptr;
};

int launch_bucket(bdcu_ctx* ctx, int form, const Bucket& b, const State& st, int cache_mode, cudaStream_t s) {
    RunArgs a;
    memset(&a, 0, sizeof(a));
    a.chains = ctx->chains_d;
    a.n_chains = ctx->n_chains;
    a.n_max = b.n_max;
    a.arena = ctx->arena_d;
    a.seed_table = ctx->seed_d;
    a.R = st.R;
    a.rng = st.rng;
    a.cache = st.cache;
    a.cache_valid = st.cache_valid;
    a.t_start = st.t_start;
    a.n_steps = st.n_steps;
    a.status = st.status;
    a.counters = st.counters;
    a.cache_mode = cache_mode;
    a.d_in_smem = b.d_in_smem;
    a.v_cap = b.v_cap;
    a.need_chol = b.need_chol;
    a.need_d = b.need_d;
    a.need_lz = b.need_lz;
    a.work_counter = ctx->work_d + b.id;
    a.order = ctx->order_d + b.order_off;
    a.n_work = b.count;
    a.scratch = ctx->bscratch[b.id];
    a.scratch_stride = b.scratch_stride;
    a.xs_pow = ctx->xs_pow_d;
    a.a_pow = ctx->a_pow_d;
    a.budget_ns = st.budget_ns;
    a.steps_done = st.steps_done;
    a.t_end = st.t_end;
    a.bounds_every = form == BDCU_FORM_MIXED_FP32 ? ctx->bounds_every : 1;
    cudaError_t e;
    if (b.kernel == BDCU_KERNEL_TEAM)
        e = launch_mixed_team(b.team_warps, b.team_q, a, b.grid, b.smem, s);
    else
        e = (form == BDCU_FORM_MIXED_FP32) ? launch_mixed(a, b.grid, b.block, b.smem, s)
                                           : launch_plain(a, b.grid, b.block, b.smem, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, b.kernel == BDCU_KERNEL_TEAM ? "integrate_team_kernel launch"
                                                                             : "integrate_kernel launch");
    return BDCU_OK;
}

// Every bucket of the plan: the first on the context stream, the others on
// their own streams forked from it and joined back.
int run_plan(bdcu_ctx* ctx, int form, const State& st, int cache_mode) {
    const size_t nb = ctx->plan.size();
    if (nb == 0) return BDCU_OK;
    cudaStream_t s0 = ctx->stream;
    CK(cudaMemsetAsync(ctx->work_d, 0, sizeof(int32_t) * kMaxBuckets, s0));
    if (nb > 1) CK(cudaEventRecord(ctx->ev_fork, s0));
    int rc;
    for (size_t i = 0; i < nb; ++i) {
        cudaStream_t s = i == 0 ? s0 : ctx->aux[i];
        if (i > 0) CK(cudaStreamWaitEvent(s, ctx->ev_fork, 0));
        if ((rc = launch_bucket(ctx, form, ctx->plan[i], st, cache_mode, s))) return rc;
        if (i > 0) CK(cudaEventRecord(ctx->ev_join[i], s));
    }
    for (size_t i = 1; i < nb; ++i) CK(cudaStreamWaitEvent(s0, ctx->ev_join[i], 0));
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
    cudaDeviceSynchronize();
    void* ptrs[] = {ctx->chains_d, ctx->arena_d, ctx->seed_d, ctx->work_d, ctx->hR, ctx->hrng, ctx->hcache,
                    ctx->hvalid, ctx->ht0, ctx->hsteps, ctx->hstatus, ctx->hcnt, ctx->xs_pow_d, ctx->a_pow_d,
                    ctx->order_d, ctx->rec_dev};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (int i = 0; i < kMaxBuckets; ++i) {
        if (ctx->bscratch[i]) cudaFree(ctx->bscratch[i]);
        if (ctx->aux[i]) cudaStreamDestroy(ctx->aux[i]);
        if (ctx->ev_join[i]) cudaEventDestroy(ctx->ev_join[i]);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    free_staging(ctx->order_stage);
    free_staging(ctx->rec_stage);
    free_staging(ctx->arena_stage);
    delete ctx;
    return BDCU_OK;
}

int bdcu_set_stream(bdcu_ctx* ctx, void* stream) {
    if (!ctx) return BDCU_E_ARG;
    ctx->stream = static_cast<cudaStream_t>(stream);
    return BDCU_OK;
}

const char* bdcu_last_error(bdcu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int bdcu_check_chains(int n_chains, const bdcu_phys* phys, const bdcu_sim* sim, const double* arena,
                      int64_t arena_len, char* msg, int msg_len) {
    bdcu_ctx scratch;
    int rc = BDCU_OK;
    if (n_chains < 1 || !phys || !sim) {
        rc = fail(&scratch, BDCU_E_ARG, "need n_chains >= 1 and phys/sim records");
    } else if (arena_len < 0 || (arena_len > 0 && !arena)) {
        rc = fail(&scratch, BDCU_E_ARG, "bad arena");
    } else {
        for (int i = 0; i < n_chains && rc == BDCU_OK; ++i)
            rc = validate(&scratch, i, phys[i], sim[i], arena, arena_len);
    }
    if (msg && msg_len > 0) {
        const size_t n = std::min<size_t>(scratch.err.size(), (size_t)msg_len - 1);
        memcpy(msg, scratch.err.data(), n);
        msg[n] = '\0';
    }
    return rc;
}

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
    if (arena_len < 0) return fail(ctx, BDCU_E_ARG, "negative arena length");
    CK(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = ensure_tables(ctx))) return rc;
    std::vector<DevChain> recs(n_chains);
    int64_t off = 0;
    int n_max = 0, any_hi = 0, any_cheb = 0, any_chol_method = 0;
    for (int i = 0; i < n_chains; ++i) {
        const bdcu_phys& p = phys[i];
        if ((rc = validate(ctx, i, p, sim[i], arena, arena_len))) return rc;
        recs[i] = derive(p, sim[i], off, ctx->seed_norm_h[3 * p.n_beads]);
        off += p.n_beads;
        n_max = std::max(n_max, 3 * p.n_beads);
        if (p.hstar > 0.0) {
            any_hi = 1;
            if (p.hi_method == BDCU_HI_CHEBYSHEV) any_cheb = 1;
            if (p.hi_method == BDCU_HI_CHOLESKY) any_chol_method = 1;
        }
    }
    if ((rc = ensure(ctx, &ctx->chains_d, n_chains))) return rc;
    CK(cudaMemcpy(ctx->chains_d, recs.data(), sizeof(DevChain) * n_chains, cudaMemcpyHostToDevice));
    if ((rc = ensure(ctx, &ctx->arena_d, arena_len > 0 ? arena_len : 1))) return rc;
    if (arena_len > 0 && arena)
        CK(cudaMemcpy(ctx->arena_d, arena, sizeof(double) * arena_len, cudaMemcpyHostToDevice));
    ctx->chains_h.swap(recs);
    ctx->sims_h.assign(sim, sim + n_chains);
    ctx->arena_h.assign(arena ? arena : nullptr, arena ? arena + arena_len : nullptr);
    ctx->arena_len = arena_len;
    ctx->n_chains = n_chains;
    ctx->n_max = n_max;
    ctx->total_beads = off;
    ctx->any_hi = any_hi;
    ctx->any_cheb = any_cheb;
    ctx->need_chol = any_hi;
    ctx->any_chol_method = any_chol_method;
    ctx->pool = 0;
    ctx->bead_capacity = off;
    ctx->sel_all = 1;
    ctx->sel.clear();
    ctx->plan_dirty = 1;
    return BDCU_OK;
}

int bdcu_run(bdcu_ctx* ctx, double* R, int32_t* rng, double* cache, int32_t* cache_valid, const double* t_start,
             const int32_t* n_steps, int32_t* status, bdcu_counters* counters, int form, int cache_mode) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_run before bdcu_set_chains or bdcu_reserve");
    if (!R || !rng || !cache || !cache_valid || !t_start || !n_steps || !status || !counters)
        return fail(ctx, BDCU_E_ARG, "null device pointer");
    if (form != BDCU_FORM_PLAIN_FP64 && form != BDCU_FORM_MIXED_FP32) return fail(ctx, BDCU_E_ARG, "unknown form");
    if (cache_mode != BDCU_CACHE_RESET_PER_CALL && cache_mode != BDCU_CACHE_PERSIST)
        return fail(ctx, BDCU_E_ARG, "unknown cache mode");
    CK(cudaSetDevice(ctx->device));
    int rc = build_plan(ctx, form);
    if (rc) return rc;
    const State st{R, rng, cache, cache_valid, t_start, n_steps, status, counters};
    return run_plan(ctx, form, st, cache_mode);
}

int bdcu_run_slice(bdcu_ctx* ctx, double* R, int32_t* rng, double* cache, int32_t* cache_valid,
                   const double* t_start, const int32_t* n_steps, int32_t* status, bdcu_counters* counters,
                   int form, int cache_mode, int64_t budget_ns, int32_t* steps_done, double* t_end) {
    if (!ctx) return BDCU_E_ARG;
    if (budget_ns < 0) return fail(ctx, BDCU_E_ARG, "negative time budget");
    if (!steps_done || !t_end) return fail(ctx, BDCU_E_ARG, "null steps_done or t_end");
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_run_slice before bdcu_set_chains or bdcu_reserve");
    if (!R || !rng || !cache || !cache_valid || !t_start || !n_steps || !status || !counters)
        return fail(ctx, BDCU_E_ARG, "null device pointer");
    if (form != BDCU_FORM_PLAIN_FP64 && form != BDCU_FORM_MIXED_FP32) return fail(ctx, BDCU_E_ARG, "unknown form");
    if (cache_mode != BDCU_CACHE_RESET_PER_CALL && cache_mode != BDCU_CACHE_PERSIST)
        return fail(ctx, BDCU_E_ARG, "unknown cache mode");
    CK(cudaSetDevice(ctx->device));
    int rc = build_plan(ctx, form);
    if (rc) return rc;
    // chains the selection does not advance, or that are skipped (failed),
    // report no steps
    CK(cudaMemsetAsync(steps_done, 0, sizeof(int32_t) * (size_t)ctx->n_chains, ctx->stream));
    State st{R, rng, cache, cache_valid, t_start, n_steps, status, counters};
    st.budget_ns = budget_ns;
    st.steps_done = steps_done;
    st.t_end = t_end;
    return run_plan(ctx, form, st, cache_mode);
}

int bdcu_set_bounds_refresh(bdcu_ctx* ctx, int every_steps) {
    if (!ctx) return BDCU_E_ARG;
    if (every_steps < 1 || every_steps > 1000000) return fail(ctx, BDCU_E_ARG, "every_steps must be in [1, 1e6]");
    ctx->bounds_every = every_steps;
    return BDCU_OK;
}

int bdcu_describe_plan(bdcu_ctx* ctx, int form, bdcu_bucket_info* out, int cap, int* n_out) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_describe_plan before bdcu_set_chains or bdcu_reserve");
    if (form != BDCU_FORM_PLAIN_FP64 && form != BDCU_FORM_MIXED_FP32) return fail(ctx, BDCU_E_ARG, "unknown form");
    if (!n_out || (cap > 0 && !out)) return fail(ctx, BDCU_E_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    int rc = build_plan(ctx, form);
    if (rc) return rc;
    *n_out = (int)ctx->plan.size();
    for (int i = 0; i < cap && i < (int)ctx->plan.size(); ++i) {
        const Bucket& b = ctx->plan[i];
        bdcu_bucket_info& o = out[i];
        o.bucket = b.id;
        o.kernel = b.kernel;
        o.team_warps = b.team_warps;
        o.team_beads_per_thread = b.team_q;
        o.n_chains = b.count;
        o.min_beads = b.min_beads;
        o.max_beads = b.max_beads;
        o.block = b.block;
        o.grid = b.grid;
        o.v_cap = b.v_cap;
        o.d_in_smem = b.d_in_smem;
        o.tuned = b.tuned;
        o.smem_bytes = (int64_t)b.smem;
    }
    return BDCU_OK;
}

int bdcu_autotune(bdcu_ctx* ctx, int form, const double* R, const int32_t* rng, const double* cache,
                  const int32_t* cache_valid, const double* t_start, int probe_steps) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_autotune before bdcu_set_chains or bdcu_reserve");
    if (form != BDCU_FORM_PLAIN_FP64 && form != BDCU_FORM_MIXED_FP32) return fail(ctx, BDCU_E_ARG, "unknown form");
    if (!R || !rng || !cache || !cache_valid || !t_start) return fail(ctx, BDCU_E_ARG, "null device pointer");
    if (probe_steps < 1 || probe_steps > 1000) return fail(ctx, BDCU_E_ARG, "probe_steps must be in [1, 1000]");
    CK(cudaSetDevice(ctx->device));
    const int mixed = form == BDCU_FORM_MIXED_FP32;
    for (int id = 0; id < kMaxBuckets; ++id) ctx->tuned[mixed][id] = Shape();
    ctx->plan_dirty = 1;
    int rc = build_plan(ctx, form);
    if (rc) return rc;

    const int64_t nb = std::max<int64_t>(ctx->bead_capacity, 1), nc = ctx->n_chains;
    double *tR = nullptr, *tcache = nullptr, *tt0 = nullptr;
    int32_t *trng = nullptr, *tvalid = nullptr, *tsteps = nullptr, *tstatus = nullptr;
    bdcu_counters* tcnt = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {
        void* ptrs[] = {tR, tcache, tt0, trng, tvalid, tsteps, tstatus, tcnt};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
#define TK(call)                                           \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) {                           \
            cleanup();                                     \
            ctx->plan_dirty = 1;                           \
            return cuda_fail(ctx, e_, #call);              \
        }                                                  \
    } while (0)
    TK(cudaMalloc(&tR, sizeof(double) * 3 * nb));
    TK(cudaMalloc(&tcache, sizeof(double) * 3 * nb));
    TK(cudaMalloc(&tt0, sizeof(double) * nc));
    TK(cudaMalloc(&trng, sizeof(int32_t) * 3 * nc));
    TK(cudaMalloc(&tvalid, sizeof(int32_t) * nc));
    TK(cudaMalloc(&tsteps, sizeof(int32_t) * nc));
    TK(cudaMalloc(&tstatus, sizeof(int32_t) * nc));
    TK(cudaMalloc(&tcnt, sizeof(bdcu_counters) * nc));
    TK(cudaEventCreate(&e0));
    TK(cudaEventCreate(&e1));
    {
        std::vector<int32_t> k(nc, probe_steps);
        TK(cudaMemcpy(tsteps, k.data(), sizeof(int32_t) * nc, cudaMemcpyHostToDevice));
    }
    TK(cudaMemcpy(tt0, t_start, sizeof(double) * nc, cudaMemcpyDeviceToDevice));
    const State st{tR, trng, tcache, tvalid, tt0, tsteps, tstatus, tcnt};
    cudaStream_t s = ctx->stream;
    const std::vector<Bucket> plan = ctx->plan;
    for (const Bucket& base : plan) {
        float best_ms = 1e30f;
        Shape best;
        std::vector<Shape> shapes;
        if (base.kernel == BDCU_KERNEL_BLOCK) {
            shapes = block_shapes(ctx, base, form);
        } else {
            // team shapes that hold any chain of the bucket, up to twice its width
            for (int i = 0; i < kNumTeamShapes; ++i) {
                const int T = kTeamShapes[i][0], Q = kTeamShapes[i][1];
                if (team_shape_fits(T, Q, kBucketBeads[base.id]) && 32 * T * Q <= 2 * kBucketBeads[base.id]) {
                    Shape sh;
                    sh.team_warps = T;
                    sh.team_q = Q;
                    shapes.push_back(sh);
                }
            }
        }
        for (const Shape& shape : shapes) {
            Bucket b = base;
            if (fill_launch(ctx, form, b, &shape) != BDCU_OK) continue;  // not resident: skip the shape
            if ((rc = ensure_bucket_scratch(ctx, b))) {
                cleanup();
                ctx->plan_dirty = 1;
                return rc;
            }
            float ms = 0.f;
            for (int rep = 0; rep < 2; ++rep) {  // the second run is timed
                TK(cudaMemcpyAsync(tR, R, sizeof(double) * 3 * nb, cudaMemcpyDeviceToDevice, s));
                TK(cudaMemcpyAsync(tcache, cache, sizeof(double) * 3 * nb, cudaMemcpyDeviceToDevice, s));
                TK(cudaMemcpyAsync(trng, rng, sizeof(int32_t) * 3 * nc, cudaMemcpyDeviceToDevice, s));
                TK(cudaMemcpyAsync(tvalid, cache_valid, sizeof(int32_t) * nc, cudaMemcpyDeviceToDevice, s));
                TK(cudaMemsetAsync(tstatus, 0, sizeof(int32_t) * nc, s));
                TK(cudaMemsetAsync(tcnt, 0, sizeof(bdcu_counters) * nc, s));
                TK(cudaMemsetAsync(ctx->work_d + b.id, 0, sizeof(int32_t), s));
                TK(cudaEventRecord(e0, s));
                if ((rc = launch_bucket(ctx, form, b, st, BDCU_CACHE_PERSIST, s))) {
                    cleanup();
                    ctx->plan_dirty = 1;
                    return rc;
                }
                TK(cudaEventRecord(e1, s));
                TK(cudaEventSynchronize(e1));
                TK(cudaEventElapsedTime(&ms, e0, e1));
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = shape;
            }
        }
        if (best.block > 0 || best.team_warps > 0) ctx->tuned[mixed][base.id] = best;
    }
#undef TK
    cleanup();
    ctx->plan_dirty = 1;
    return BDCU_OK;
}

int bdcu_set_single_launch(bdcu_ctx* ctx, int on) {
    if (!ctx) return BDCU_E_ARG;
    ctx->single_launch = on ? 1 : 0;
    ctx->plan_dirty = 1;
    return BDCU_OK;
}

int bdcu_set_team_shape(bdcu_ctx* ctx, int bucket, int team_warps, int beads_per_thread) {
    if (!ctx) return BDCU_E_ARG;
    if (bucket < 0 || bucket >= kFirstBlockBucket) return fail(ctx, BDCU_E_ARG, "team buckets are 0..3");
    Shape sh;
    if (team_warps != 0) {
        if (!team_shape_fits(team_warps, beads_per_thread, kBucketBeads[bucket]))
            return fail(ctx, BDCU_E_ARG, "not a compiled team shape that holds every chain of the bucket");
        sh.team_warps = team_warps;
        sh.team_q = beads_per_thread;
    }
    ctx->tuned[1][bucket] = sh;
    ctx->plan_dirty = 1;
    return BDCU_OK;
}

int bdcu_reserve(bdcu_ctx* ctx, int n_slots, int64_t bead_capacity, int64_t arena_len) {
    if (!ctx) return BDCU_E_ARG;
    if (n_slots < 1 || bead_capacity < 2 || arena_len < 0)
        return fail(ctx, BDCU_E_ARG, "need n_slots >= 1, bead_capacity >= 2, arena_len >= 0");
    CK(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = ensure_tables(ctx))) return rc;
    CK(cudaDeviceSynchronize());  // the records and arena may be in use by earlier runs
    if ((rc = ensure(ctx, &ctx->chains_d, n_slots))) return rc;
    CK(cudaMemset(ctx->chains_d, 0, sizeof(DevChain) * n_slots));
    if ((rc = ensure(ctx, &ctx->arena_d, arena_len > 0 ? arena_len : 1))) return rc;
    CK(cudaMemset(ctx->arena_d, 0, sizeof(double) * std::max<int64_t>(arena_len, 1)));
    // pinned staging for the uploads of a serving loop, sized once here: a
    // pinned buffer that grew later would have to be freed (cudaFreeHost
    // waits for the whole device)
    if ((rc = reserve_staging(ctx, ctx->rec_stage, 4 * (sizeof(DevChain) + sizeof(int32_t)) * (size_t)n_slots + 4096)))
        return rc;
    if ((rc = reserve_staging(ctx, ctx->order_stage, 4 * sizeof(int32_t) * (size_t)n_slots + 4096))) return rc;
    if ((rc = reserve_staging(ctx, ctx->arena_stage, 2 * sizeof(double) * (size_t)std::max<int64_t>(arena_len, 1) + 4096)))
        return rc;
    const size_t rec_bytes = (sizeof(DevChain) + sizeof(int32_t)) * (size_t)n_slots + 256;
    if (ctx->rec_dev) cudaFree(ctx->rec_dev);
    ctx->rec_dev = nullptr;
    ctx->rec_dev_bytes = 0;
    CK(cudaMalloc(&ctx->rec_dev, rec_bytes));
    ctx->rec_dev_bytes = rec_bytes;
    DevChain empty;
    memset(&empty, 0, sizeof(empty));
    ctx->chains_h.assign(n_slots, empty);
    bdcu_sim zs;
    memset(&zs, 0, sizeof(zs));
    ctx->sims_h.assign(n_slots, zs);
    ctx->arena_h.assign(arena_len, 0.0);
    ctx->arena_len = arena_len;
    ctx->n_chains = n_slots;
    ctx->n_max = 0;
    ctx->total_beads = 0;
    ctx->any_hi = ctx->any_cheb = ctx->need_chol = ctx->any_chol_method = 0;
    ctx->pool = 1;
    ctx->bead_capacity = bead_capacity;
    ctx->sel_all = 0;
    ctx->sel.clear();
    ctx->plan_dirty = 1;
    return BDCU_OK;
}

int bdcu_update_chains(bdcu_ctx* ctx, int count, const int32_t* slots, const bdcu_phys* phys, const bdcu_sim* sim,
                       const int64_t* bead_off) {
    if (!ctx) return BDCU_E_ARG;
    if (!ctx->pool) return fail(ctx, BDCU_E_STATE, "bdcu_update_chains needs a pool (bdcu_reserve)");
    if (count < 0 || (count > 0 && (!slots || !phys || !sim || !bead_off)))
        return fail(ctx, BDCU_E_ARG, "bad bdcu_update_chains arguments");
    if (count == 0) return BDCU_OK;
    if (count > ctx->n_chains) return fail(ctx, BDCU_E_ARG, "more records than slots");
    CK(cudaSetDevice(ctx->device));
    std::vector<unsigned char> buf(sizeof(DevChain) * (size_t)count + sizeof(int32_t) * (size_t)count);
    DevChain* recs = reinterpret_cast<DevChain*>(buf.data());
    int32_t* ids = reinterpret_cast<int32_t*>(buf.data() + sizeof(DevChain) * (size_t)count);
    int rc;
    for (int i = 0; i < count; ++i) {
        const int32_t slot = slots[i];
        if (slot < 0 || slot >= ctx->n_chains) return fail(ctx, BDCU_E_ARG, "slot id out of range");
        if ((rc = validate(ctx, slot, phys[i], sim[i], ctx->arena_h.data(), ctx->arena_len))) return rc;
        if (bead_off[i] < 0 || bead_off[i] + phys[i].n_beads > ctx->bead_capacity)
            return fail(ctx, BDCU_E_ARG, "slot " + std::to_string(slot) + ": beads outside bead_capacity");
        recs[i] = derive(phys[i], sim[i], bead_off[i], ctx->seed_norm_h[3 * phys[i].n_beads]);
        ids[i] = slot;
    }
    for (int i = 0; i < count; ++i) {
        ctx->chains_h[slots[i]] = recs[i];
        ctx->sims_h[slots[i]] = sim[i];
        ctx->n_max = std::max(ctx->n_max, 3 * phys[i].n_beads);
    }
    if ((rc = stage_upload(ctx, ctx->rec_stage, ctx->rec_dev, buf.data(), buf.size()))) return rc;
    const DevChain* drecs = reinterpret_cast<const DevChain*>(ctx->rec_dev);
    const int32_t* dids = reinterpret_cast<const int32_t*>(static_cast<unsigned char*>(ctx->rec_dev) +
                                                           sizeof(DevChain) * (size_t)count);
    cudaError_t e = launch_scatter_records(ctx->chains_d, drecs, dids, count, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "scatter_records launch");
    ctx->plan_dirty = 1;
    return BDCU_OK;
}

int bdcu_write_arena(bdcu_ctx* ctx, int64_t offset, const double* values, int64_t count) {
    if (!ctx) return BDCU_E_ARG;
    if (!ctx->pool) return fail(ctx, BDCU_E_STATE, "bdcu_write_arena needs a pool (bdcu_reserve)");
    if (count < 0 || offset < 0 || offset + count > ctx->arena_len || (count > 0 && !values))
        return fail(ctx, BDCU_E_ARG, "arena write outside the reserved arena");
    if (count == 0) return BDCU_OK;
    CK(cudaSetDevice(ctx->device));
    memcpy(ctx->arena_h.data() + offset, values, sizeof(double) * count);
    return stage_upload(ctx, ctx->arena_stage, ctx->arena_d + offset, values, sizeof(double) * count);
}

int bdcu_select(bdcu_ctx* ctx, int count, const int32_t* slots) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_select before bdcu_set_chains or bdcu_reserve");
    if (count == 0 && !slots) {
        if (ctx->pool) return fail(ctx, BDCU_E_ARG, "a pool needs an explicit selection");
        ctx->sel_all = 1;
        ctx->sel.clear();
        ctx->plan_dirty = 1;
        return BDCU_OK;
    }
    if (count < 0 || (count > 0 && !slots)) return fail(ctx, BDCU_E_ARG, "bad selection");
    std::vector<char> seen(ctx->n_chains, 0);
    std::vector<std::pair<int64_t, int>> ranges;
    ranges.reserve(count);
    for (int i = 0; i < count; ++i) {
        const int32_t c = slots[i];
        if (c < 0 || c >= ctx->n_chains) return fail(ctx, BDCU_E_ARG, "selected slot out of range");
        if (seen[c]) return fail(ctx, BDCU_E_ARG, "slot " + std::to_string(c) + " selected twice");
        seen[c] = 1;
        if (ctx->chains_h[c].N < 2) return fail(ctx, BDCU_E_ARG, "slot " + std::to_string(c) + " is empty");
        ranges.emplace_back(ctx->chains_h[c].bead_off, ctx->chains_h[c].N);
    }
    std::sort(ranges.begin(), ranges.end());
    for (size_t i = 1; i < ranges.size(); ++i)
        if (ranges[i - 1].first + ranges[i - 1].second > ranges[i].first)
            return fail(ctx, BDCU_E_ARG, "selected chains share beads");
    ctx->sel.assign(slots, slots + count);
    ctx->sel_all = 0;
    ctx->plan_dirty = 1;
    return BDCU_OK;
}

int bdcu_integrate_host(bdcu_ctx* ctx, double* R_host, int32_t* rng_host, int32_t* status_host,
                        bdcu_counters* counters_host, int form) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1 || ctx->pool)
        return fail(ctx, BDCU_E_STATE, "bdcu_integrate_host needs chains from bdcu_set_chains");
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

int bdcu_observables(bdcu_ctx* ctx, const double* R, const double* F, double* out) {
    if (!ctx) return BDCU_E_ARG;
    if (ctx->n_chains < 1) return fail(ctx, BDCU_E_STATE, "bdcu_observables before bdcu_set_chains");
    if (!R || !F || !out) return fail(ctx, BDCU_E_ARG, "null device pointer");
    CK(cudaSetDevice(ctx->device));
    cudaError_t e = launch_observables(ctx->chains_d, ctx->n_chains, R, F, out, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "observables kernel launch");
    return BDCU_OK;
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
// The checks bdcu_set_chains makes on one chain record, for the static-scratch
// entry point (so both entry points accept the same inputs).
int validate_chain(bdcu_ctx* ctx, int i, const bdcu_phys& p, const bdcu_sim& s, const double* arena,
                   int64_t arena_len) {
    return validate(ctx, i, p, s, arena, arena_len);
}

// The per-chain record derivation, for the static-scratch entry point.
DevChain derive_record(const bdcu_phys& p, const bdcu_sim& s, int64_t bead_off) {
    double ss = 0.0;
    for (int i = 0; i < 3 * p.n_beads; ++i) {
        const double v = sin(0.7654321 * (i + 1)) + 0.5;
        ss += v * v;
    }
    return derive(p, s, bead_off, sqrt(ss));
}
}  // namespace bdcu
