// Host-only stand-in for <cuda_runtime.h>, used solely to compile the
// reference's kernel bodies (cuda/cmf_walk_{f64,df64,rns}.cu) as plain C++ on
// the CPU, so that they can serve as a checker for this project's own oracle.
//
// Test infrastructure only: nothing in the product links this header.
//
// The kernel qualifiers are defined away on the compiler command line
// (-D__global__= -D__device__= -D__host__= -D__constant__=). The CUDA
// runtime calls that the reference's host drivers make are given inert
// definitions here so that the translation unit links; the shim never calls
// those drivers, it calls the kernel bodies directly, one index at a time.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <algorithm>

using std::isfinite;
using std::isinf;
using std::isnan;

struct ref_dim3 { unsigned x, y, z; };

// The kernel bodies compute idx = blockIdx.x * blockDim.x + threadIdx.x.
// The shim sets blockIdx.x = idx, blockDim.x = 1, threadIdx.x = 0 on the
// calling (OpenMP) thread before each call.
extern thread_local ref_dim3 blockIdx;
extern thread_local ref_dim3 blockDim;
extern thread_local ref_dim3 threadIdx;

typedef int cudaError_t;
typedef void *cudaEvent_t;
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
enum { cudaComputeModeDefault = 0 };

struct cudaDeviceProp {
    char name[256];
    int major, minor, multiProcessorCount, maxThreadsPerMultiProcessor;
    int clockRate, computeMode;
    size_t totalGlobalMem;
};

template <class T> inline cudaError_t cudaMalloc(T **p, size_t n) { *p = (T *)std::malloc(n ? n : 1); return 0; }
inline cudaError_t cudaFree(void *p) { std::free(p); return 0; }
inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) { std::memcpy(d, s, n); return 0; }
inline cudaError_t cudaDeviceSynchronize() { return 0; }
inline cudaError_t cudaEventCreate(cudaEvent_t *e) { *e = nullptr; return 0; }
inline cudaError_t cudaEventRecord(cudaEvent_t) { return 0; }
inline cudaError_t cudaEventSynchronize(cudaEvent_t) { return 0; }
inline cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t, cudaEvent_t) { *ms = 0.f; return 0; }
inline cudaError_t cudaEventDestroy(cudaEvent_t) { return 0; }
inline cudaError_t cudaMemGetInfo(size_t *f, size_t *t) { *f = 0; *t = 0; return 0; }
inline cudaError_t cudaGetDevice(int *d) { *d = 0; return 0; }
inline cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int) { std::memset(p, 0, sizeof(*p)); return 0; }
