// Peak-throughput microbenchmark for the roofline denominators the driver
// does not measure: dense FP64 and FP32 FMA on the CUDA cores.  Every thread
// runs 8 independent FMA chains; the result is stored so nothing is
// eliminated.  Used by bench.py only.
#include <cuda_runtime.h>
#include <cstdio>

template <typename T>
__global__ void k_fma_chain(T *out, int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = (T)(threadIdx.x + i);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = x[i] * a + b;
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += x[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename T>
static double run(int iters) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256;
    T *out = nullptr;
    if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(T)) != cudaSuccess) return -1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_chain<T><<<blocks, threads>>>(out, iters / 10, (T)0.999999, (T)1e-7);   // warm-up
    cudaEventRecord(e0);
    k_fma_chain<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    return flops / (ms * 1e-3) / 1e12;
}

extern "C" __attribute__((visibility("default"))) double pgpu_peak_fma_tflops(int fp32, int iters) {
    return fp32 ? run<float>(iters) : run<double>(iters);
}
