// warp_layout.h -- sizes of the one-chain-per-warp kernel's shared and global
// scratch, shared by the host launch code and the kernel.
#pragma once

#include "integrator.cuh"

namespace bdcu {

constexpr int kWarpMaxN = 64;
constexpr int kWarpMaxn = 3 * kWarpMaxN;
constexpr int kWarpsPerCta = 4;
constexpr unsigned kFull = 0xffffffffu;

// Per-warp shared memory (fixed part). The warm Lanczos basis
// (kLanczosWarm x nv doubles) follows it; the Chebyshev node and coefficient
// tables (2 x kCoefCap floats) share that area, as the basis is dead once the
// spectral bounds are known.
struct WarpShared {
    float4 pos[kWarpMaxN];   // FP32 bead coordinates of the tensor's configuration
    float4 xs[kWarpMaxN];    // FP32 staged D.x input
    double s0[kWarpMaxn];    // FP64 neighbour-exchange buffers
    double s1[kWarpMaxn];
    double s2[kWarpMaxn];
    double s3[kWarpMaxN];
    double s4[kWarpMaxN];
    double alpha[32], beta[32], ymin[32], ymax[32];
    DevChain ch;
};

__host__ __device__ inline int64_t warp_smem_bytes(int n_max) {
    const int64_t nv = round_up8(n_max);
    int64_t area = (int64_t)kLanczosWarm * nv * 8;
    if (area < (int64_t)2 * kCoefCap * 4) area = (int64_t)2 * kCoefCap * 4;
    const int64_t per = (int64_t)((sizeof(WarpShared) + 15) / 16 * 16) + area;
    return per * kWarpsPerCta;
}
__host__ __device__ inline int64_t warp_smem_stride(int n_max) { return warp_smem_bytes(n_max) / kWarpsPerCta; }

// Per-warp global scratch (doubles): cold Lanczos basis, Cholesky factor.
__host__ __device__ inline int64_t warp_scratch_doubles(int n_max) {
    return (int64_t)kLanczosCold * round_up8(n_max) + (int64_t)n_max * n_max;
}

}  // namespace bdcu
