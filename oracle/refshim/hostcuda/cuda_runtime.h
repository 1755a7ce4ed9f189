// Host-compiler stand-in for <cuda_runtime.h>, used only to compile the
// reference's CUDA kernels (simulation/kernels.cuh) as ordinary C++ functions
// for the CPU parity oracle and the timed CPU baseline (TEST INFRASTRUCTURE).
// Each "thread" of a kernel becomes one call with blockIdx/threadIdx set in
// thread-local storage; atomics become OpenMP atomics.
#pragma once
#include <cstdint>
#include <cmath>
#include <algorithm>

#define __device__
#define __host__
#define __global__
#define __constant__
#define __shared__
#define __forceinline__ inline

struct icempm_uint3 { unsigned x, y, z; };
extern thread_local icempm_uint3 blockIdx, threadIdx, blockDim;

typedef void *cudaStream_t;
typedef void *cudaEvent_t;
typedef int cudaError_t;
enum { cudaSuccess = 0 };

inline double atomicAdd(double *addr, double v) {
    double old;
#pragma omp atomic capture
    { old = *addr; *addr += v; }
    return old;
}
inline int atomicAdd(int *addr, int v) {
    int old;
#pragma omp atomic capture
    { old = *addr; *addr += v; }
    return old;
}
inline int atomicMax(int *addr, int v) {
    int old;
#pragma omp critical(icempm_atomic_max)
    { old = *addr; if (v > old) *addr = v; }
    return old;
}
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline double min(double a, double b) { return std::fmin(a, b); }
inline double max(double a, double b) { return std::fmax(a, b); }
