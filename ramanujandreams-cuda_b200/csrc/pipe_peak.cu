// Pipe-throughput probe used as the roofline denominator of the walk
// kernels, which are bound by FP64 (f64), FP32 (float-float) or INT32
// (residue) issue rate rather than by memory: every thread runs eight
// independent fused multiply-add chains for a fixed number of iterations on
// a grid of several CTAs per SM, timed with CUDA events.
#include <cstdio>

#include "cmfw.h"
#include "cmfw_internal.cuh"

namespace {

constexpr int kChains = 8;

template <typename T>
__device__ __forceinline__ T chain_step(T a, T b, T c);
template <>
__device__ __forceinline__ double chain_step<double>(double a, double b, double c) { return __fma_rn(a, b, c); }
template <>
__device__ __forceinline__ float chain_step<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <>
__device__ __forceinline__ unsigned chain_step<unsigned>(unsigned a, unsigned b, unsigned c) { return a * b + c; }

template <typename T>
__global__ void __launch_bounds__(256) pipe_kernel(T *sink, T b, T c, int iters) {
    T acc[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) acc[k] = (T)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) acc[k] = chain_step<T>(acc[k], b, c);
    }
    T s = acc[0];
#pragma unroll
    for (int k = 1; k < kChains; ++k) s = s + acc[k];
    if (s == (T)12345) sink[blockIdx.x] = s;  // keeps the chains live
}

template <typename T>
cmfw_status run(T b, T c, double *tops) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    T *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(T) * blocks) != cudaSuccess) return CMFW_ENOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    pipe_kernel<T><<<blocks, threads>>>(sink, b, c, iters);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(e0);
        pipe_kernel<T><<<blocks, threads>>>(sink, b, c, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return CMFW_ECUDA;
    const double ops = 2.0 * (double)blocks * threads * iters * kChains;  // FMA = 2 ops
    *tops = ops / (best * 1e-3) / 1e12;
    return CMFW_OK;
}

}  // namespace

extern "C" cmfw_status cmfw_pipe_peak(int pipe, double *tera_ops_per_s) {
    if (!tera_ops_per_s) return CMFW_EINVAL;
    switch (pipe) {
        case 0: return run<double>(1.0000001, 1e-9, tera_ops_per_s);
        case 1: return run<float>(1.0001f, 1e-6f, tera_ops_per_s);
        case 2: return run<unsigned>(2654435761u, 12345u, tera_ops_per_s);
    }
    return CMFW_EINVAL;
}
