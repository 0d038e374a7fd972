/*
 * bdsim_cuda.h -- C ABI of the B200 ensemble integrator for bdsim's
 * ChainIntegrator step.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns
 * an int status (BDCU_OK == 0; otherwise a BDCU_E_* code, with a message from
 * bdcu_last_error). No C++ exception crosses this boundary.
 *
 * What each entry point replaces in the reference (paths relative to the
 * bdsim project root):
 *
 *   bdcu_integrate_host   _bdsim.integrate(R, phys, sim, rng)
 *                         bindings/module.cpp:45-50  ->  time_integrate_chain
 *                         src/integrator.hpp:32, src/integrator.cpp:174-177
 *                         (batched: many chains, one call; the RNG state and
 *                         R are updated in place exactly as the reference
 *                         mutates its Rng and returns the evolved R)
 *   bdcu_run              the same step loop on device-resident state
 *                         (ChainIntegrator::run, src/integrator.cpp:66-85)
 *   bdcu_total_force      _bdsim.total_force(R, phys)
 *                         bindings/module.cpp:67-76
 *   bdcu_forces           _bdsim.spring_force / ev_force / bending_force /
 *                         external_force, bindings/module.cpp:52-66,128-132
 *   bdcu_ran1             Rng::ran_1, src/rng.cpp:41-70 (per-chain streams)
 *   bdcu_set_chains       PhysParams / SimParams marshalling
 *                         (src/model.hpp:20-35, src/integrator.hpp:22-28,
 *                         pickled state tuples bindings/module.cpp:184-297)
 *   bdcu_queue_*          many simulate calls (python/bdsim/ensemble.py:179-227)
 *                         served concurrently from one slot pool
 *
 * Parameter layout. One bdcu_phys and one bdcu_sim per chain. Variable-size
 * tables (flow samples, external-force samples, SDK phi) live in one double
 * "arena" the caller passes alongside, addressed by index:
 *
 *   flow table      arena[flow_offset .. +n)           sample times (ascending)
 *                   arena[flow_offset+n .. +9n)        row-major kappa per sample
 *   external list   ext_n_entries records starting at arena[ext_offset], each
 *                   [bead, is_constant, fx, fy, fz, n_times,
 *                    t_0 .. t_{n-1}, f_0x f_0y f_0z .. f_{n-1}z]
 *                   (6 + 4*n_times doubles); negative bead counts from the end
 *   SDK phi         arena[phi_offset .. + N*N) row-major, or phi_offset == -1
 */
#ifndef BDSIM_CUDA_H
#define BDSIM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enums: same numeric values as the reference (src/types.hpp:27-55) ---- */
enum {
    BDCU_SPRING_HOOK = 1,
    BDCU_SPRING_FENE = 2,
    BDCU_SPRING_ILC = 3,
    BDCU_SPRING_WLC = 4,
    BDCU_SPRING_FRAENKEL = 5,
    BDCU_SPRING_FENE_FRAENKEL = 6,
    BDCU_SPRING_WLC_BOUNDED = 7
};
enum { BDCU_EV_NONE = 0, BDCU_EV_GAUSS = 1, BDCU_EV_LJ = 2, BDCU_EV_SDK = 3, BDCU_EV_SDK_STICKERS = 4 };
enum { BDCU_BEND_NONE = 0, BDCU_BEND_ONE_MINUS_COS = 1 };
enum { BDCU_HI_CHEBYSHEV = 0, BDCU_HI_CHOLESKY = 1, BDCU_HI_EXACT_SQRT = 2 };

/* ---- integrator forms ---- */
enum {
    /* FP64, the reference algorithm step for step, one chain per thread block. */
    BDCU_FORM_PLAIN_FP64 = 0,
    /* FP32 matrix-free RPY products and FP32 excluded volume; FP64 positions,
       connector solve, Lanczos bounds and Cholesky. */
    BDCU_FORM_MIXED_FP32 = 1
};

/* ---- spectral-cache policy across calls ---- */
enum {
    /* the reference: each integrate call starts Lanczos cold
       (src/integrator.cpp:176 builds a fresh PhysicalModel per call) */
    BDCU_CACHE_RESET_PER_CALL = 0,
    /* keep the warm-start vector across calls (a chunked run then equals one
       continuous call of the reference) */
    BDCU_CACHE_PERSIST = 1
};

/* ---- per-chain status bits (device word per chain) ---- */
enum {
    BDCU_ST_NONCONVERGED = 1,  /* corrector hit 100N iterations; step accepted
                                  (src/integrator.cpp:160-163) */
    BDCU_ST_NOT_PD = 2,        /* Cholesky pivot <= 0; chain stopped
                                  (src/linalg.cpp:16-25,99) */
    BDCU_ST_CHEB_FALLBACK = 4, /* Chebyshev FD check failed, Cholesky used
                                  (src/mobility.cpp:69-81) */
    BDCU_ST_RTSAFE_FAIL = 8,   /* rtsafe bracket/iteration failure; chain
                                  stopped (the reference aborts,
                                  src/numerics.hpp:31-36,72) */
    BDCU_ST_NONFINITE = 16,    /* positions became NaN/Inf; chain stopped */
    BDCU_ST_BAD_PARAM = 32,    /* WLCbounded sigma>1 or ExactSqrt; chain
                                  stopped (reference aborts) */
    BDCU_ST_TIMEOUT = 64       /* a bounded wait inside the kernel (the
                                  blocked Cholesky's tile copies) gave up;
                                  chain stopped (no counterpart) */
};
#define BDCU_ST_FATAL_MASK \
    (BDCU_ST_NOT_PD | BDCU_ST_RTSAFE_FAIL | BDCU_ST_NONFINITE | BDCU_ST_BAD_PARAM | BDCU_ST_TIMEOUT)

/* ---- error codes returned by entry points ---- */
enum {
    BDCU_OK = 0,
    BDCU_E_ARG = 1,      /* invalid argument */
    BDCU_E_CUDA = 2,     /* CUDA runtime error */
    BDCU_E_STATE = 3,    /* call order (e.g. run before set_chains) */
    BDCU_E_NOMEM = 4,    /* allocation failed */
    BDCU_E_LIMIT = 5     /* size beyond a documented maximum */
};

/* PhysParams (src/model.hpp:20-35) with its SpringParams (src/spring.hpp:12-19),
   EVParams (src/excluded_volume.hpp:17-25), BendingParams (src/bending.hpp:9-12),
   Flow (src/flow.hpp:17-43) and ExternalForce (src/external_force.hpp:32-57). */
typedef struct bdcu_phys {
    int32_t n_beads;
    int32_t spring_type;
    double sqrtb;
    double natural_length;
    int32_t ev_type;
    int32_t contour_dist_for_ev;
    double zstar;
    double dstar;
    double min_cutoff;
    double max_cutoff;
    int64_t phi_offset;
    int32_t bend_type;
    int32_t equilibration;
    double bend_stiffness;
    double hstar;
    int32_t hi_method;
    int32_t flow_n_times;
    double ncheb_multiplier;
    double fd_err_max;
    double flow_kappa[9];
    int64_t flow_offset;
    int32_t ext_n_entries;
    int32_t reserved0;
    int64_t ext_offset;
} bdcu_phys;

/* SimParams (src/integrator.hpp:22-28). time_start/time_end bound the step
   loop exactly as ChainIntegrator::run does (src/integrator.cpp:67). */
typedef struct bdcu_sim {
    double time_start;
    double time_end;
    double dt;
    double implicit_loop_tol;
    int32_t update_center_of_mass;
    int32_t reserved0;
} bdcu_sim;

/* Per-chain counters (device). They replace the reference's only in-code
   counters, SpectralCache::cold_runs/warm_runs (src/hydrodynamics.hpp:33-37),
   and its global nonconvergence_count (src/integrator.cpp:25). */
typedef struct bdcu_counters {
    int64_t steps;            /* integrator steps completed */
    int64_t dx_products;      /* D.x products (the dominant work unit) */
    int64_t cheb_terms;       /* sum of Chebyshev term counts L over attempts */
    int64_t corrector_iters;  /* implicit-corrector iterations */
    int64_t lanczos_cold;
    int64_t lanczos_warm;
    int64_t cheb_fallbacks;   /* FD failures that fell back to Cholesky */
    int64_t nonconverged;     /* steps whose corrector did not converge */
} bdcu_counters;

typedef struct bdcu_ctx bdcu_ctx;

/* Library version string. */
const char* bdcu_version(void);

/* Create a context on CUDA device `device`. Allocates nothing on the device. */
int bdcu_create(int device, bdcu_ctx** out);
int bdcu_destroy(bdcu_ctx* ctx);
/* Stream for all subsequent work (a cudaStream_t; NULL = legacy default). */
int bdcu_set_stream(bdcu_ctx* ctx, void* stream);

/* Spectral-bound refresh policy of the FP32-mixed form (no counterpart in the
   reference, which recomputes the Lanczos bounds every step,
   src/mobility.cpp:64-67): the team kernel (mixed form, N <= 512) keeps a
   chain's padded bounds for every_steps steps and recomputes them early when
   a step's Chebyshev fluctuation-dissipation check fails on the kept bounds
   (then the reference's growth and Cholesky fallback apply). Every launch
   starts with a refresh, so with every_steps > 1 a run cut into launches
   differs from one launch. 1 (the default) is the reference's policy; the
   plain form always refreshes every step. */
int bdcu_set_bounds_refresh(bdcu_ctx* ctx, int every_steps);
/* Message of the last failing call on this context (NUL-terminated). */
const char* bdcu_last_error(bdcu_ctx* ctx);

/* Describe the chains of the batch. phys/sim: n_chains records (host).
   arena: arena_len doubles (host). Derived constants are computed here on the
   host (pow/exp as the reference's constructors do) and uploaded. */
int bdcu_set_chains(bdcu_ctx* ctx, int n_chains, const bdcu_phys* phys,
                    const bdcu_sim* sim, const double* arena, int64_t arena_len);

/* Number of integrator steps the reference loop
   `for (t = time_start; t <= time_end + dt/2; t += dt)` takes for chain i.
   Host-side, no device work. */
int bdcu_count_steps(const bdcu_sim* sim, int64_t* n_steps_out);

/* Run the step loop on device-resident state, asynchronously on the context
   stream. All pointers are device pointers owned by the caller:
     R            total_beads*3 doubles, chains concatenated in set_chains order
     rng          n_chains*3 int32 (ix, iy, seed), advanced in place
     cache        total_beads*3 doubles, spectral warm-start vectors
     cache_valid  n_chains int32 (0 => next Lanczos is cold)
     t_start      n_chains doubles, first step time of this call
     n_steps      n_chains int32, steps to take in this call
     status       n_chains int32, OR-ed with BDCU_ST_* bits
     counters     n_chains bdcu_counters, accumulated
   (for a slot pool: bead_capacity and n_slots in place of total_beads and
   n_chains). Only the selected chains (bdcu_select; default all) are touched.
   A chain whose status has a fatal bit set is skipped. */
int bdcu_run(bdcu_ctx* ctx, double* R, int32_t* rng, double* cache,
             int32_t* cache_valid, const double* t_start, const int32_t* n_steps,
             int32_t* status, bdcu_counters* counters, int form, int cache_mode);

/* bdcu_run with a time slice, for serving loops that share the GPU between
   jobs (no counterpart in the reference, whose integrate calls run to
   completion, ChainIntegrator::run, src/integrator.cpp:66-85): a chain
   starts no new step once budget_ns nanoseconds have passed since its thread
   block started (0: no limit; a step in progress always completes), so one
   slow chain (e.g. a corrector at its 100N-iteration cap) cannot hold the
   launch for long. Per chain (device, n_chains entries, zeroed first for the
   chains it does not advance): steps_done = steps completed, t_end = the
   chain's time after them (the device's running sum t += dt). Continuing with
   t_start = t_end, n_steps = the remainder and the spectral cache kept
   (BDCU_CACHE_PERSIST, cache_valid left as the slice left it) gives the same
   result, bit for bit, as one uninterrupted bdcu_run. */
int bdcu_run_slice(bdcu_ctx* ctx, double* R, int32_t* rng, double* cache,
                   int32_t* cache_valid, const double* t_start, const int32_t* n_steps,
                   int32_t* status, bdcu_counters* counters, int form, int cache_mode,
                   int64_t budget_ns, int32_t* steps_done, double* t_end);

/* The reference-facing batched integrate: host R (total_beads*3), host rng
   (n_chains*3), host status (n_chains). Runs every chain over its own
   bdcu_sim [time_start, time_end] with a cold spectral cache, as
   time_integrate_chain does; copies R, rng and status back. Synchronous. */
int bdcu_integrate_host(bdcu_ctx* ctx, double* R_host, int32_t* rng_host,
                        int32_t* status_host, bdcu_counters* counters_host,
                        int form);

/* Intramolecular force (spring + EV + bending, no external) at R (device
   pointers, total_beads*3 each), FP64. */
int bdcu_total_force(bdcu_ctx* ctx, const double* R, double* F);

/* Force components at R: `which` ORs BDCU_F_* bits. A single bit gives that
   force alone (bindings/module.cpp:52-66,128-132: spring_force, ev_force,
   bending_force, external_force at time t); several bits are summed as
   (spring + (EV + bending)) + external, the reference's grouping. */
enum { BDCU_F_SPRING = 1, BDCU_F_EV = 2, BDCU_F_BEND = 4, BDCU_F_EXTERNAL = 8 };
int bdcu_forces(bdcu_ctx* ctx, const double* R, double t, int which, double* F);

/* Per-chain observables on the device, for snapshots without a host round
   trip: radius_of_gyration_sq and kramers_stress (python/bdsim/properties.py:
   17-19,38-41) of positions R with the forces F (e.g. from bdcu_total_force;
   device pointers, total_beads*3 each). out: n_chains*10 doubles per record,
   [Rg^2, tau_xx, tau_xy, tau_xz, tau_yx, tau_yy, tau_yz, tau_zx, tau_zy,
   tau_zz], tau_ij = sum_mu (R_mu - R_c)_i F_mu,j. */
int bdcu_observables(bdcu_ctx* ctx, const double* R, const double* F, double* out);

/* Draw n_per_chain uniforms per chain from device RNG states (n_chains*3
   int32, advanced in place) into out (device, n_chains*n_per_chain). */
int bdcu_ran1(bdcu_ctx* ctx, int n_chains, int32_t* rng, int n_per_chain, double* out);

/* ---- Launch plans for batches of uneven chains (no counterpart in the
   reference, which integrates one chain per call: time_integrate_chain,
   src/integrator.hpp:32).
   bdcu_run splits the chains it advances into buckets by bead count and runs
   each bucket as one persistent launch over a device work list ordered
   largest chain first; buckets run concurrently, forked from the context
   stream and joined back to it. In the FP32-mixed form a chain of N <= 512
   beads (and no Cholesky method) runs on the team kernel in buckets 0..3 (N <=
   64, 128, 256, 512), by default with (warps per chain, beads per thread) =
   (2,1), (4,1), (4,2), (8,2) unless tuned or pinned; every other chain runs one chain per
   thread block, in buckets 4..7 split at N = 64, 128 and 256. Once a plan is
   built (first bdcu_run after a change of records, selection or form) a
   bdcu_run enqueues only a memset, event records/waits and kernel launches,
   so it may be captured in a CUDA graph. */
enum { BDCU_KERNEL_BLOCK = 0, BDCU_KERNEL_TEAM = 1 };
#define BDCU_MAX_BUCKETS 8
typedef struct bdcu_bucket_info {
    int32_t bucket;      /* 0..3: team kernel; 4..7: block kernel */
    int32_t kernel;      /* BDCU_KERNEL_* */
    int32_t team_warps;  /* team kernel: warps per chain (0 for the block kernel) */
    int32_t n_chains;    /* chains in the bucket */
    int32_t min_beads;
    int32_t max_beads;
    int32_t block;       /* threads per block */
    int32_t grid;        /* persistent blocks */
    int32_t v_cap;       /* Lanczos basis vectors kept in shared memory */
    int32_t d_in_smem;   /* dense D in shared memory (plain form) */
    int32_t tuned;       /* 1: shape chosen by bdcu_autotune */
    int32_t team_beads_per_thread;  /* team kernel: 1 or 2 beads per thread (0 for the block kernel) */
    int64_t smem_bytes;  /* dynamic shared memory per block */
} bdcu_bucket_info;
/* The plan bdcu_run would use for `form` on the current selection; writes up
   to `cap` buckets (cap >= BDCU_MAX_BUCKETS always suffices) and their count. */
int bdcu_describe_plan(bdcu_ctx* ctx, int form, bdcu_bucket_info* out, int cap, int* n_out);

/* Time every launch shape of each bucket of the current selection for
   probe_steps steps on device copies of the given state -- the caller's buffers
   are read, never written -- and keep the fastest shape per (form, bucket) for
   later bdcu_run calls. Block-kernel buckets: threads per block x Lanczos
   vectors in shared memory x, in the plain form, D in shared memory.
   Team-kernel buckets (FP32-mixed form): warps per team x beads per thread,
   every compiled team shape that holds any chain of the bucket, up to twice
   its width. No
   counterpart in the reference (one chain per call on the CPU). Synchronous;
   allocates and frees its copies. The shape changes only the speed and,
   through the order of block and team reductions, the rounding of the
   Lanczos and Chebyshev dot products. */
int bdcu_autotune(bdcu_ctx* ctx, int form, const double* R, const int32_t* rng, const double* cache,
                  const int32_t* cache_valid, const double* t_start, int probe_steps);

/* on = 1: every chain of the FP32-mixed form's team kernel runs in ONE
   persistent launch (the widest team bucket present takes the narrower
   buckets' chains, largest first, and runs its shape) instead of one launch
   per bucket forked onto streams; on = 0 restores the per-bucket plan. A
   chain's result depends on the team shape it runs with (the order of its
   team reductions), not on which launch it is in. No counterpart in the
   reference. */
int bdcu_set_single_launch(bdcu_ctx* ctx, int on);

/* Pin the team shape of team-kernel bucket `bucket` (0..3) of the FP32-mixed
   form: team_warps warps per chain with beads_per_thread (1 or 2) beads per
   thread, a compiled shape that holds every chain the bucket admits (32 *
   team_warps * beads_per_thread >= 64, 128, 256, 512 for buckets 0..3). team_warps = 0 returns the bucket to
   the default shape. Later bdcu_autotune calls replace it. No counterpart in
   the reference. */
int bdcu_set_team_shape(bdcu_ctx* ctx, int bucket, int team_warps, int beads_per_thread);

/* ---- Slot pools, for a serving loop that admits and retires chains between
   runs (no counterpart in the reference).
   bdcu_reserve replaces the context's chains with n_slots empty slots, sized
   for state arrays of bead_capacity beads (R and cache hold bead_capacity*3
   doubles; rng n_slots*3 int32; cache_valid, t_start, n_steps, status n_slots;
   counters n_slots records) and an arena of arena_len doubles (zeroed). */
int bdcu_reserve(bdcu_ctx* ctx, int n_slots, int64_t bead_capacity, int64_t arena_len);
/* Fill `count` slots with chains: slot ids (host), their phys/sim records and
   the first bead of each chain in the state arrays (bead_off + n_beads <=
   bead_capacity). Table offsets in phys refer to the context arena. Enqueued on
   the context stream; the records are derived on the host. */
int bdcu_update_chains(bdcu_ctx* ctx, int count, const int32_t* slots, const bdcu_phys* phys,
                       const bdcu_sim* sim, const int64_t* bead_off);
/* Copy `count` doubles (host) into the context arena at `offset`. */
int bdcu_write_arena(bdcu_ctx* ctx, int64_t offset, const double* values, int64_t count);
/* The chains the following bdcu_run calls advance: `count` slot ids (host),
   distinct, filled, with disjoint bead ranges; count = 0 with slots = NULL
   selects every chain (not allowed for a pool). */
int bdcu_select(bdcu_ctx* ctx, int count, const int32_t* slots);

/* The checks bdcu_set_chains, bdcu_update_chains and bdcu_run_static make on
   chain records (bead count, dt, spring/EV types, every flow, phi and
   external-force table inside the arena), without a GPU or a context. No
   counterpart in the reference, whose constructors trust their inputs. Returns
   the first failing chain's status and copies its message into msg (msg_len
   bytes including the terminator; msg may be NULL). */
int bdcu_check_chains(int n_chains, const bdcu_phys* phys, const bdcu_sim* sim, const double* arena,
                      int64_t arena_len, char* msg, int msg_len);

/* bdcu_run for callers that cannot allocate device memory. No counterpart in
   the reference: bdsim runs on the CPU and never allocates GPU memory.
   Some callers cannot call cudaMalloc -- a host application whose memory pool
   already owns the GPU's memory, or a serving loop that must not take the
   implicit device-wide synchronisation cudaMalloc/cudaFree imply. This entry
   point takes the parameters on the host (as bdcu_set_chains does) and runs
   the same kernels as bdcu_run (its buckets, one after another) on the
   caller's device buffers; the parameter records, work lists, arena, work
   counters and per-block scratch live in one
   file-scope device array of BDCU_STATIC_SCRATCH_BYTES that every GPU using
   the library holds until process exit. It calls no cudaMalloc/cudaFree.
   ctx comes from bdcu_create (which allocates no device memory) and supplies
   the device, the stream and bdcu_last_error; bdcu_set_chains is not used.
   - Chain records get the checks of bdcu_set_chains (bdcu_check_chains)
     before the GPU is touched: a table outside the arena is BDCU_E_ARG, a
     chain beyond the bead limit BDCU_E_LIMIT.
   - Batches whose parameters plus one block's scratch exceed the array return
     BDCU_E_LIMIT with a message; smaller batches run with as many concurrent
     blocks as fit (fewer than bdcu_run may use).
   - The first call on a device takes the array's device address
     (cudaGetSymbolAddress), and so does the first call after the device's
     context was replaced (cudaDeviceReset).
   - It must not be called inside stream capture: each call copies its
     records, work list and tables from pageable host buffers that are freed
     when it returns (the copies finish before it returns; a captured graph
     would replay freed host memory).
   - Every call shares the array and leaves its contents behind; the work
     counters are cleared by each call. Calls that overlap on the GPU race on the
     array: serialise them. */
#define BDCU_STATIC_SCRATCH_BYTES (16u * 1024u * 1024u)
int bdcu_run_static(bdcu_ctx* ctx, int n_chains, const bdcu_phys* phys, const bdcu_sim* sim,
                    const double* arena, int64_t arena_len, double* R, int32_t* rng, double* cache,
                    int32_t* cache_valid, const double* t_start, const int32_t* n_steps, int32_t* status,
                    bdcu_counters* counters, int form, int cache_mode);

/* ---- Serving queue: continuous batching of ensemble jobs on one GPU, for a
   host that is not Python (no counterpart in the reference, whose simulate
   runs one ensemble per call to completion, python/bdsim/ensemble.py:179-227).
   A job is the arguments of one simulate call: n_traj chains of one
   bdcu_phys/bdcu_sim record, their initial positions and RNG states, the total
   steps and the snapshot interval. The queue owns a slot pool (bdcu_reserve)
   and its state buffers on the device and runs the policy of the Python
   bdsim_b200.serving.Server:
   - admission: a job needs n_traj consecutive slots, n_traj*N consecutive
     beads, room for its tables in the arena and room under the active-chain
     cap; queued jobs are admitted first-fit in arrival order over a lookahead
     window (BDCU_QUEUE_FIFO) or smallest n_traj*n_steps*N^2 first
     (BDCU_QUEUE_SJF); submissions beyond queue_limit queued jobs, or larger
     than the pool, are rejected;
   - each iteration is one bdcu_run_slice over the chains of every running
     job: each takes up to slice_steps steps of its current chunk
     (write_every steps, the job's snapshot interval) and none starts a step
     after slice_budget_ns;
   - a chunk of k steps is one integrate span [t0, t0+(k-1)dt] with
     t0 = time_start + step*dt, started with a cold spectral cache under
     BDCU_CACHE_RESET_PER_CALL (the reference's per-call semantics) and
     continued across slices with its cache, so a job's positions equal,
     bit for bit, those of integrating its chains chunk by chunk;
   - when every chain of a job has finished a chunk its positions are copied
     to the host as a snapshot event; after the last chunk (or once every
     chain has a fatal status) a DONE event carries the statuses and the
     summed counters, and the job's slots are freed.
   Threading: with cfg.worker = 1 a library thread drives the queue and
   submit / poll / stats / wait_idle may be called from any thread; with
   worker = 0 the caller drives it with bdcu_queue_step (or wait_idle) from one
   thread, and the other entry points may still be called from any thread. */
typedef struct bdcu_queue bdcu_queue;
enum { BDCU_QUEUE_FIFO = 0, BDCU_QUEUE_SJF = 1 };
typedef struct bdcu_queue_config {
    int32_t form;               /* BDCU_FORM_* */
    int32_t policy;             /* BDCU_QUEUE_FIFO | BDCU_QUEUE_SJF */
    int32_t max_chains;         /* chain slots of the pool (>= 1) */
    int32_t max_active_chains;  /* cap on running chains (0: max_chains) */
    int64_t bead_capacity;      /* beads of the pool (>= 2) */
    int64_t arena_capacity;     /* doubles for the jobs' tables (>= 0) */
    int32_t queue_limit;        /* queued jobs beyond which submit rejects (0: no limit) */
    int32_t lookahead;          /* FIFO: queued jobs examined per admission (0: 16) */
    int32_t slice_steps;        /* steps per chain per iteration (>= 1) */
    int32_t cache_mode;         /* BDCU_CACHE_* at each chunk start */
    int64_t slice_budget_ns;    /* no chain starts a step after this (0: no limit) */
    int32_t worker;             /* 1: a library thread drives the queue */
    int32_t reserved0;
} bdcu_queue_config;
typedef struct bdcu_job {
    int32_t n_traj;             /* chains */
    int32_t snapshots;          /* 1: an event per chunk (and the initial state); 0: the final one */
    int64_t n_steps;            /* steps of the whole job (>= 0) */
    int64_t write_every;        /* steps per chunk (0: one chunk) */
    int64_t tag;                /* the caller's id, echoed in the job's events */
    bdcu_phys phys;             /* every chain's record; table offsets index `arena` */
    bdcu_sim sim;               /* dt, tolerance, centre-of-mass flag, time_start */
    const double* arena;        /* the job's tables (host; may be NULL when arena_len = 0) */
    int64_t arena_len;
    const double* R0;           /* n_traj * n_beads * 3 doubles (host) */
    const int32_t* rng;         /* n_traj * 3 int32: (ix, iy, seed) per chain (host) */
} bdcu_job;
enum { BDCU_QEV_SNAPSHOT = 1, BDCU_QEV_DONE = 2, BDCU_QEV_REJECTED = 3 };
typedef struct bdcu_queue_event {
    int32_t kind;               /* BDCU_QEV_* */
    int32_t n_traj;
    int32_t n_beads;
    int32_t snapshot;           /* SNAPSHOT: index (0 = the initial state) */
    int64_t job;                /* id from bdcu_queue_submit */
    int64_t tag;
    int64_t step;               /* steps completed at this event */
    double time;                /* SNAPSHOT: time of the positions (time_start + step*dt) */
    double t_arrival;           /* seconds since the queue was created */
    double t_admit;             /* (< 0: not admitted) */
    double t_done;              /* DONE: delivery of the last snapshot */
    bdcu_counters counters;     /* DONE: summed over the job's chains */
} bdcu_queue_event;
typedef struct bdcu_queue_stats {
    int64_t submitted, rejected, queued, running, done;
    int64_t active_chains;
    int64_t chain_steps;        /* steps completed by all chains */
    int64_t slices;             /* bdcu_run_slice launches */
    int64_t selected_chains;    /* sum over slices of the chains advanced */
    int64_t pending_events;
    double device_ms;           /* device time of the slice launches */
} bdcu_queue_stats;
/* Allocates the pool's device buffers (R and warm-start vectors of
   bead_capacity*3 doubles, per-slot RNG, status, counters and step arrays)
   and a context; starts the worker thread when cfg->worker = 1. */
int bdcu_queue_create(int device, const bdcu_queue_config* cfg, bdcu_queue** out);
/* Stops the worker (after its current iteration) and frees everything;
   undelivered events are dropped. */
int bdcu_queue_destroy(bdcu_queue* q);
const char* bdcu_queue_last_error(bdcu_queue* q);
/* Copies the job (records, tables, R0, rng) and queues it, or rejects it
   (*accepted = 0, and a REJECTED event) when queue_limit jobs are queued or
   the job is larger than the pool. Records get the checks of bdcu_check_chains
   against the job's own arena: a failing record returns its BDCU_E_* code and
   queues nothing. *job_id receives the job's id either way. */
int bdcu_queue_submit(bdcu_queue* q, const bdcu_job* job, int64_t* job_id, int* accepted);
/* Caller-driven mode: one iteration (admission, one slice launch, waiting
   for it, the events of the chunks it completed). *busy = 1 while jobs are
   queued or running. BDCU_E_STATE in worker mode. */
int bdcu_queue_step(bdcu_queue* q, int* busy);
/* Until no job is queued or running, or timeout_ms passes (< 0: no limit):
   waits for the worker, or in caller-driven mode runs iterations. *busy as in
   bdcu_queue_step. */
int bdcu_queue_wait_idle(bdcu_queue* q, int64_t timeout_ms, int* busy);
/* Takes the oldest undelivered event (*got = 1; 0 when there is none).
   SNAPSHOT events copy n_traj*n_beads*3 doubles into positions and DONE
   events n_traj statuses into status; a buffer that is NULL is skipped, one
   that is too small returns BDCU_E_LIMIT with *ev filled in and the event
   kept, so the caller can size its buffers from ev and poll again. */
int bdcu_queue_poll(bdcu_queue* q, bdcu_queue_event* ev, double* positions, int64_t positions_len,
                    int32_t* status, int32_t status_len, int* got);
int bdcu_queue_get_stats(bdcu_queue* q, bdcu_queue_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* BDSIM_CUDA_H */
