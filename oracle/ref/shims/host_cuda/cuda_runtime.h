// Host-only stand-in for <cuda_runtime.h>, used only when the reference's CUDA
// sources are compiled as plain host C++ for the oracle. It supplies the CUDA
// vector types, strips the execution-space qualifiers and gives one serial
// "thread": blockIdx = threadIdx = 0, blockDim = gridDim = 1, so every
// grid-stride loop in the reference kernels walks all of its items in order.
#pragma once
#include <cstring>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#ifndef __device__
#define __device__
#endif
#ifndef __global__
#define __global__
#endif
#ifndef __host__
#define __host__
#endif
#ifndef __shared__
#define __shared__
#endif
#ifndef __constant__
#define __constant__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#include <vector_types.h>

static inline double3 make_double3(double x, double y, double z) {
  double3 r; r.x = x; r.y = y; r.z = z; return r;
}
static inline double4 make_double4(double x, double y, double z, double w) {
  double4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r;
}

typedef int cudaError_t;
#define cudaSuccess 0

static const uint3 threadIdx = {0u, 0u, 0u};
static const uint3 blockIdx = {0u, 0u, 0u};
static const dim3 blockDim(1u, 1u, 1u);
static const dim3 gridDim(1u, 1u, 1u);

static inline void __syncthreads() {}

static inline long long __double_as_longlong(double d) {
  long long r;
  std::memcpy(&r, &d, sizeof r);
  return r;
}
static inline double __longlong_as_double(long long v) {
  double r;
  std::memcpy(&r, &v, sizeof r);
  return r;
}
// Serial compare-and-swap: with one host thread the CAS loop in the
// reference's FP64 atomic add reduces to a plain read-modify-write.
static inline unsigned long long atomicCAS(unsigned long long* a,
                                           unsigned long long cmp,
                                           unsigned long long val) {
  unsigned long long old = *a;
  if (old == cmp) *a = val;
  return old;
}
static inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
static inline cudaError_t cudaGetLastError() { return cudaSuccess; }
static inline const char* cudaGetErrorString(cudaError_t) { return "no error"; }
