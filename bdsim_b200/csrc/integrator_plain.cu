// integrator_plain.cu -- the FP64 plain form. This translation unit is
// compiled with --fmad=false so that every product and sum rounds separately,
// as in the reference's default x86-64 build (no FMA contraction).
#include "integrator.cuh"

namespace bdcu {

cudaError_t launch_plain(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s) {
    auto k = integrate_kernel<BDCU_FORM_PLAIN_FP64>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, block, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t occupancy_plain(int block, size_t smem, int* per_sm) {
    auto k = integrate_kernel<BDCU_FORM_PLAIN_FP64>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, block, smem);
}

}  // namespace bdcu
