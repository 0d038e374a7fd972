// integrator_mixed.cu -- the FP32-mixed form (FMA contraction on).
#include "integrator.cuh"
#include "integrator_warp.cuh"

namespace bdcu {

cudaError_t launch_mixed(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s) {
    auto k = integrate_kernel<BDCU_FORM_MIXED_FP32>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, block, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t occupancy_mixed(int block, size_t smem, int* per_sm) {
    auto k = integrate_kernel<BDCU_FORM_MIXED_FP32>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, block, smem);
}

cudaError_t launch_mixed_warp(const RunArgs& a, int grid, size_t smem, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(integrate_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    integrate_warp_kernel<<<grid, kWarpsPerCta * 32, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t occupancy_mixed_warp(size_t smem, int* per_sm) {
    cudaError_t e = cudaFuncSetAttribute(integrate_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, integrate_warp_kernel, kWarpsPerCta * 32, smem);
}

}  // namespace bdcu
