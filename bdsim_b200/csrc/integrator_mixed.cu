// integrator_mixed.cu -- the FP32-mixed form (FMA contraction on).
#include "integrator.cuh"
#include "integrator_team.cuh"
#include "plan.h"

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

template <int T, int Q>
static cudaError_t launch_team_t(const RunArgs& a, int grid, size_t smem, cudaStream_t s) {
    integrate_team_kernel<T, Q><<<grid, TeamCfg<T, Q>::kCtaThreads, smem, s>>>(a);
    return cudaGetLastError();
}

template <int T, int Q>
static cudaError_t occupancy_team_t(size_t smem, int* per_sm) {
    cudaError_t e = allow_max_smem(reinterpret_cast<const void*>(integrate_team_kernel<T, Q>));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, integrate_team_kernel<T, Q>,
                                                         TeamCfg<T, Q>::kCtaThreads, smem);
}

cudaError_t launch_mixed_team(int team_warps, int team_q, const RunArgs& a, int grid, size_t smem, cudaStream_t s) {
#define BDCU_LAUNCH(t, q) launch_team_t<t, q>(a, grid, smem, s)
    return BDCU_TEAM_SHAPE_SWITCH(team_warps, team_q, BDCU_LAUNCH, cudaErrorInvalidValue);
#undef BDCU_LAUNCH
}

cudaError_t occupancy_mixed_team(int team_warps, int team_q, size_t smem, int* per_sm) {
#define BDCU_OCC(t, q) occupancy_team_t<t, q>(smem, per_sm)
    return BDCU_TEAM_SHAPE_SWITCH(team_warps, team_q, BDCU_OCC, cudaErrorInvalidValue);
#undef BDCU_OCC
}

}  // namespace bdcu
