// integrator_mixed.cu -- the FP32-mixed form (FMA contraction on).
#include "integrator.cuh"
#include "integrator_team.cuh"

namespace bdcu {

// Launches take no attribute call (so that they can be captured in a graph):
// the occupancy query, made first at plan time, lets the kernel use the
// device's opt-in shared-memory maximum.
static cudaError_t allow_max_smem(const void* k) {
    int dev = 0, v = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    return e;
}

cudaError_t launch_mixed(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s) {
    integrate_kernel<BDCU_FORM_MIXED_FP32><<<grid, block, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t occupancy_mixed(int block, size_t smem, int* per_sm) {
    auto k = integrate_kernel<BDCU_FORM_MIXED_FP32>;
    cudaError_t e = allow_max_smem(reinterpret_cast<const void*>(k));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, block, smem);
}

template <int T>
static cudaError_t launch_team_t(const RunArgs& a, int grid, size_t smem, cudaStream_t s) {
    integrate_team_kernel<T><<<grid, TeamCfg<T>::kCtaThreads, smem, s>>>(a);
    return cudaGetLastError();
}

template <int T>
static cudaError_t occupancy_team_t(size_t smem, int* per_sm) {
    cudaError_t e = allow_max_smem(reinterpret_cast<const void*>(integrate_team_kernel<T>));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, integrate_team_kernel<T>, TeamCfg<T>::kCtaThreads,
                                                         smem);
}

cudaError_t launch_mixed_team(int team_warps, const RunArgs& a, int grid, size_t smem, cudaStream_t s) {
    switch (team_warps) {
        case 1: return launch_team_t<1>(a, grid, smem, s);
        case 2: return launch_team_t<2>(a, grid, smem, s);
        case 4: return launch_team_t<4>(a, grid, smem, s);
        case 8: return launch_team_t<8>(a, grid, smem, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t occupancy_mixed_team(int team_warps, size_t smem, int* per_sm) {
    switch (team_warps) {
        case 1: return occupancy_team_t<1>(smem, per_sm);
        case 2: return occupancy_team_t<2>(smem, per_sm);
        case 4: return occupancy_team_t<4>(smem, per_sm);
        case 8: return occupancy_team_t<8>(smem, per_sm);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace bdcu
