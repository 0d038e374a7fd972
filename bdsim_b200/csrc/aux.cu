// aux.cu -- small kernels beside the integrator: the force evaluations of
// _bdsim.total_force / spring_force / ev_force / bending_force /
// external_force (bindings/module.cpp:52-76,128-132) and bulk ran_1 draws
// (src/rng.cpp:41-70). Compiled with --fmad=false like the plain form.
#include "integrator.cuh"

namespace bdcu {

// One chain per block. `which` selects force components (BDCU_F_*); present
// terms are combined as (spring + (EV + bending)) + external.
__global__ void __launch_bounds__(256) forces_kernel(const RunArgs a, const double* __restrict__ Rg, double t,
                                                     int which, double* __restrict__ Fg) {
    extern __shared__ __align__(16) double sm[];
    __shared__ DevChain chs;
    __shared__ Ctl ctl;
    const int nv = (int)round_up8(a.n_max);
    for (int c = blockIdx.x; c < a.n_chains; c += gridDim.x) {
        {
            const int nw = (int)(sizeof(DevChain) / 8);
            const double* src = reinterpret_cast<const double*>(a.chains + c);
            double* dst = reinterpret_cast<double*>(&chs);
            for (int i = threadIdx.x; i < nw; i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        if (chs.N < 2) {  // an empty slot of a pool
            __syncthreads();
            continue;
        }
        Block<BDCU_FORM_PLAIN_FP64> B(a, ctl, chs);
        const int N = chs.N, n = 3 * N;
        B.N = N;
        B.n = n;
        double* R = sm;
        double* bond = sm + nv;
        double* len = sm + 2 * nv;
        double* Fc = sm + 3 * nv;
        double* Fs = sm + 4 * nv;
        double* u = sm + 5 * nv;
        double* cs = sm + 6 * nv;
        const double* gR = Rg + 3 * chs.bead_off;
        for (int i = threadIdx.x; i < n; i += blockDim.x) R[i] = gR[i];
        __syncthreads();
        B.geometry(R, bond, len);
        __syncthreads();
        if (which & BDCU_F_SPRING) B.spring_from_geometry(bond, len, Fc, Fs);
        const bool bend = (which & BDCU_F_BEND) && chs.bend_type != BDCU_BEND_NONE && N > 2;
        if (bend) {
            for (int b = threadIdx.x; b < N - 1; b += blockDim.x)
                for (int d = 0; d < 3; ++d) u[3 * b + d] = (1.0 / len[b]) * bond[3 * b + d];
            __syncthreads();
            for (int b = threadIdx.x; b < N - 2; b += blockDim.x)
                cs[b] = u[3 * (b + 1)] * u[3 * b] + u[3 * (b + 1) + 1] * u[3 * b + 1] + u[3 * (b + 1) + 2] * u[3 * b + 2];
        }
        __syncthreads();
        double* gF = Fg + 3 * chs.bead_off;
        for (int m = threadIdx.x; m < N; m += blockDim.x) {
            double fe[3] = {0.0, 0.0, 0.0}, fb[3] = {0.0, 0.0, 0.0}, fx[3] = {0.0, 0.0, 0.0};
            if (which & BDCU_F_EV) B.ev_on_bead(R, m, fe);
            if (bend) bending_on_bead(chs, m, u, cs, len, fb);
            if ((which & BDCU_F_EXTERNAL) && chs.ext_n > 0) external_on_bead(chs, a.arena, m, t, fx);
            for (int d = 0; d < 3; ++d) {
                double v;
                const bool has_nsp = (which & (BDCU_F_EV | BDCU_F_BEND)) != 0;
                double nsp = 0.0;
                if ((which & BDCU_F_EV) && (which & BDCU_F_BEND)) nsp = fe[d] + fb[d];
                else if (which & BDCU_F_EV) nsp = fe[d];
                else if (which & BDCU_F_BEND) nsp = fb[d];
                if (which & BDCU_F_SPRING) v = has_nsp ? Fs[3 * m + d] + nsp : Fs[3 * m + d];
                else v = nsp;
                if (which & BDCU_F_EXTERNAL) v = (which & (BDCU_F_SPRING | BDCU_F_EV | BDCU_F_BEND)) ? v + fx[d] : fx[d];
                gF[3 * m + d] = v;
            }
        }
        __syncthreads();
    }
}

cudaError_t launch_forces(const DevChain* chains, int n_chains, int n_max, const double* arena, const double* R,
                          double t, int which, double* F, cudaStream_t s) {
    RunArgs a = {};
    a.chains = chains;
    a.n_chains = n_chains;
    a.n_max = n_max;
    a.arena = arena;
    const size_t smem = sizeof(double) * 7 * (size_t)round_up8(n_max);
    cudaError_t e = cudaFuncSetAttribute(forces_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = n_chains < 4096 ? n_chains : 4096;
    forces_kernel<<<grid, 128, smem, s>>>(a, R, t, which, F);
    return cudaGetLastError();
}

// Per-chain observables of a configuration (python/bdsim/properties.py:13-41):
// out[c*10 + 0] = Rg^2 = trace of the gyration tensor, out[c*10 + 1 + 3i + j]
// = Kramers stress tau_ij = sum_mu (R_mu - R_c)_i F_mu,j. One warp per chain,
// sums over beads in a warp butterfly (not the host's order: last-bit
// differences from numpy).
// One warp per chain, every chain's warp launched at once (no loop over
// chains), so the loads of all chains are in flight together. A chain of up to
// 64 beads is read once into registers (two beads per lane, R and F issued
// together); longer chains take a second pass over R. Each lane sums its beads
// in order, then the lanes' sums are reduced by shuffles: the same arithmetic
// either way.
__global__ void __launch_bounds__(256) observables_kernel(const DevChain* __restrict__ chains, int n_chains,
                                                          const double* __restrict__ R, const double* __restrict__ F,
                                                          double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int c = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (c >= n_chains) return;
    const int N = chains[c].N;
    const double* r = R + 3 * chains[c].bead_off;
    const double* f = F + 3 * chains[c].bead_off;
    double s[10];
    const double inv = N > 0 ? 1.0 / N : 0.0;
    if (N <= 64) {
        double rr[2][3], ff[2][3];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int m = lane + 32 * q;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                rr[q][d] = m < N ? r[3 * m + d] : 0.0;
                ff[q][d] = m < N ? f[3 * m + d] : 0.0;
            }
        }
        for (int d = 0; d < 3; ++d) s[d] = 0.0;
#pragma unroll
        for (int q = 0; q < 2; ++q)
            if (lane + 32 * q < N)
                for (int d = 0; d < 3; ++d) s[d] += rr[q][d];
        for (int d = 0; d < 3; ++d)
            for (int o = 16; o > 0; o >>= 1) s[d] += __shfl_xor_sync(0xffffffffu, s[d], o);
        const double cx = s[0] * inv, cy = s[1] * inv, cz = s[2] * inv;
        for (int k = 0; k < 10; ++k) s[k] = 0.0;
#pragma unroll
        for (int q = 0; q < 2; ++q)
            if (lane + 32 * q < N) {
                const double x[3] = {rr[q][0] - cx, rr[q][1] - cy, rr[q][2] - cz};
                s[0] += x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) s[1 + 3 * i + j] += x[i] * ff[q][j];
            }
    } else {
        for (int d = 0; d < 3; ++d) s[d] = 0.0;
        for (int m = lane; m < N; m += 32)
            for (int d = 0; d < 3; ++d) s[d] += r[3 * m + d];
        for (int d = 0; d < 3; ++d)
            for (int o = 16; o > 0; o >>= 1) s[d] += __shfl_xor_sync(0xffffffffu, s[d], o);
        const double cx = s[0] * inv, cy = s[1] * inv, cz = s[2] * inv;
        for (int k = 0; k < 10; ++k) s[k] = 0.0;
        for (int m = lane; m < N; m += 32) {
            const double x[3] = {r[3 * m] - cx, r[3 * m + 1] - cy, r[3 * m + 2] - cz};
            s[0] += x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) s[1 + 3 * i + j] += x[i] * f[3 * m + j];
        }
    }
    for (int k = 0; k < 10; ++k)
        for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    if (lane == 0) {
        out[10 * (int64_t)c] = s[0] * inv;
        for (int k = 1; k < 10; ++k) out[10 * (int64_t)c + k] = s[k];
    }
}

cudaError_t launch_observables(const DevChain* chains, int n_chains, const double* R, const double* F, double* out,
                               cudaStream_t s) {
    if (n_chains < 1) return cudaSuccess;
    observables_kernel<<<(unsigned)(((int64_t)n_chains + 7) / 8), 256, 0, s>>>(chains, n_chains, R, F, out);
    return cudaGetLastError();
}

// ran_1 with lazy seeding (Rng::maybe_init, src/rng.cpp:31-39), one thread per stream.
__global__ void ran1_kernel(int n_chains, int32_t* rng, int n_per, double* out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_chains) return;
    int32_t ix = rng[3 * c], iy = rng[3 * c + 1], seed = rng[3 * c + 2];
    if (seed <= 0 || iy < 0) {
        const int32_t s = seed < 0 ? -seed : seed;
        iy = (888889999 ^ s) | 1;
        ix = 777755555 ^ s;
        seed = s + 1;
    }
    const float am = __fdiv_rn(__int_as_float(0x3f7fffff), 2147483648.0f);
    uint32_t ux = (uint32_t)ix;
    for (int k = 0; k < n_per; ++k) {
        ux ^= (ux << 13);
        ux ^= (ux >> 17);
        ux ^= (ux << 5);
        const int32_t kk = iy / 127773;
        iy = 16807 * (iy - kk * 127773) - 2836 * kk;
        if (iy < 0) iy += 2147483647;
        const uint32_t mixed = ux ^ (uint32_t)iy;
        const int32_t res = (int32_t)((mixed & 0x7fffffffu) | 1u);
        out[(int64_t)c * n_per + k] = (double)__fmul_rn(am, __int2float_rn(res));
    }
    rng[3 * c] = (int32_t)ux;
    rng[3 * c + 1] = iy;
    rng[3 * c + 2] = seed;
}

cudaError_t launch_ran1(int n_chains, int32_t* rng, int n_per, double* out, cudaStream_t s) {
    ran1_kernel<<<(n_chains + 127) / 128, 128, 0, s>>>(n_chains, rng, n_per, out);
    return cudaGetLastError();
}

// Copy chain records into their pool slots: one block per record.
__global__ void scatter_records_kernel(DevChain* __restrict__ dst, const DevChain* __restrict__ src,
                                       const int32_t* __restrict__ slots, int count) {
    const int i = blockIdx.x;
    if (i >= count) return;
    const int nw = (int)(sizeof(DevChain) / 8);
    const double* s = reinterpret_cast<const double*>(src + i);
    double* d = reinterpret_cast<double*>(dst + slots[i]);
    for (int w = threadIdx.x; w < nw; w += blockDim.x) d[w] = s[w];
}

cudaError_t launch_scatter_records(DevChain* dst, const DevChain* src, const int32_t* slots, int count,
                                   cudaStream_t s) {
    if (count < 1) return cudaSuccess;
    scatter_records_kernel<<<count, 32, 0, s>>>(dst, src, slots, count);
    return cudaGetLastError();
}

}  // namespace bdcu
