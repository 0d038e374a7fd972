// peak.cu -- CUDA-core FMA throughput of this GPU, the roofline denominator
// for the integrator kernels (which run on the FP64 / FP32 pipes, not on
// tensor cores or HBM). Used by bench.py only; not part of the integrator.
#include <cuda_runtime.h>
#include <stdint.h>

template <typename T>
__global__ void fma_loop(T* out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
        x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

template <typename T>
static double run(int iters) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int block = 256, grid = sms * 8;
    T* out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * (size_t)grid * block) != cudaSuccess) return -1.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_loop<T><<<grid, block>>>(out, iters / 10, (T)0.999999, (T)1e-7);
    cudaEventRecord(e0);
    fma_loop<T><<<grid, block>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
    const double flops = 2.0 * 8.0 * (double)iters * grid * block;
    return flops / (ms * 1e-3) / 1e12;
}

// TFLOP/s (FMA = 2 flops) of the FP64 (fp64 != 0) or FP32 pipe.
extern "C" double bdpk_fma_tflops(int fp64, int iters) {
    return fp64 ? run<double>(iters) : run<float>(iters);
}
