// integrator_plain.cu -- the FP64 plain form. This translation unit is
// compiled with --fmad=false so that every product and sum rounds separately,
// as in the reference's default x86-64 build (no FMA contraction).
#include "integrator.cuh"

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

cudaError_t launch_plain(const RunArgs& a, int grid, int block, size_t smem, cudaStream_t s) {
    integrate_kernel<BDCU_FORM_PLAIN_FP64><<<grid, block, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t occupancy_plain(int block, size_t smem, int* per_sm) {
    auto k = integrate_kernel<BDCU_FORM_PLAIN_FP64>;
    cudaError_t e = allow_max_smem(reinterpret_cast<const void*>(k));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, block, smem);
}

}  // namespace bdcu
