// State transfer between the caller's numbering and the device layout, on
// the device: the caller's four field arrays (rho, u, v, w: cells, then one
// ghost per boundary face) are copied up as they are and one kernel
// interleaves and renumbers them into the state records (FP64 double4, or
// the FP32 deviation form's float4 of (u/U, v/U, w/U, rho - rho0)); the
// reverse for a read-back. Checkpoint images move whole records through the
// same renumbering. perm[o] is the device index of caller index o.
#include "plfbs_internal.hpp"

namespace plfbs {
namespace {

constexpr int kIoBlock = 256;

inline int io_blocks(long long n) {
  const long long b = (n + kIoBlock - 1) / kIoBlock;
  return (int)(b > 0 ? b : 1);
}

__global__ void __launch_bounds__(kIoBlock)
    k_state_in64(const int32_t* __restrict__ perm, long long T, const double* __restrict__ rho,
                 const double* __restrict__ u, const double* __restrict__ v,
                 const double* __restrict__ w, double4* __restrict__ state) {
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= T) return;
  state[__ldg(perm + o)] = make_double4(__ldg(u + o), __ldg(v + o), __ldg(w + o), __ldg(rho + o));
}

// Deviation units as the host formula: (float)(u / U), (float)(rho - rho0).
__global__ void __launch_bounds__(kIoBlock)
    k_state_in32(const int32_t* __restrict__ perm, long long T, const double* __restrict__ rho,
                 const double* __restrict__ u, const double* __restrict__ v,
                 const double* __restrict__ w, double U, double r0, float4* __restrict__ state) {
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= T) return;
  state[__ldg(perm + o)] = make_float4((float)(__ldg(u + o) / U), (float)(__ldg(v + o) / U),
                                       (float)(__ldg(w + o) / U), (float)(__ldg(rho + o) - r0));
}

__global__ void __launch_bounds__(kIoBlock)
    k_state_out64(const int32_t* __restrict__ perm, long long T, const double4* __restrict__ state,
                  double* __restrict__ rho, double* __restrict__ u, double* __restrict__ v,
                  double* __restrict__ w) {
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= T) return;
  const double4 q = state[__ldg(perm + o)];
  u[o] = q.x;
  v[o] = q.y;
  w[o] = q.z;
  rho[o] = q.w;
}

// Back to physical units as the host formula: U * f, rho0 + f.
__global__ void __launch_bounds__(kIoBlock)
    k_state_out32(const int32_t* __restrict__ perm, long long T, const float4* __restrict__ state,
                  double U, double r0, double* __restrict__ rho, double* __restrict__ u,
                  double* __restrict__ v, double* __restrict__ w) {
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= T) return;
  const float4 q = state[__ldg(perm + o)];
  u[o] = __dmul_rn(U, (double)q.x);
  v[o] = __dmul_rn(U, (double)q.y);
  w[o] = __dmul_rn(U, (double)q.z);
  rho[o] = __dadd_rn(r0, (double)q.w);
}

// n records of R 16-byte units: to_caller gathers dst[o] = src[perm[o]],
// otherwise scatters dst[perm[o]] = src[o].
template <int R>
__global__ void __launch_bounds__(kIoBlock)
    k_records(const int32_t* __restrict__ perm, long long n, const uint4* __restrict__ src,
              uint4* __restrict__ dst, int to_caller) {
  const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const long long k = __ldg(perm + o);
  const long long s = to_caller ? k : o, d = to_caller ? o : k;
#pragma unroll
  for (int r = 0; r < R; r++) dst[R * d + r] = src[R * s + r];
}

}  // namespace

void launch_state_in(const int32_t* perm, long long T, const double* rho, const double* u,
                     const double* v, const double* w, int precision, double U, double r0,
                     void* state, cudaStream_t s) {
  if (T <= 0) return;
  if (precision == PLFBS_FP32_DEVIATION)
    k_state_in32<<<io_blocks(T), kIoBlock, 0, s>>>(perm, T, rho, u, v, w, U, r0,
                                                   static_cast<float4*>(state));
  else
    k_state_in64<<<io_blocks(T), kIoBlock, 0, s>>>(perm, T, rho, u, v, w,
                                                   static_cast<double4*>(state));
}

void launch_state_out(const int32_t* perm, long long T, const void* state, int precision,
                      double U, double r0, double* rho, double* u, double* v, double* w,
                      cudaStream_t s) {
  if (T <= 0) return;
  if (precision == PLFBS_FP32_DEVIATION)
    k_state_out32<<<io_blocks(T), kIoBlock, 0, s>>>(perm, T, static_cast<const float4*>(state),
                                                    U, r0, rho, u, v, w);
  else
    k_state_out64<<<io_blocks(T), kIoBlock, 0, s>>>(perm, T, static_cast<const double4*>(state),
                                                    rho, u, v, w);
}

void launch_records(const int32_t* perm, long long n, int rec_bytes, const void* src, void* dst,
                    bool to_caller, cudaStream_t s) {
  if (n <= 0) return;
  const uint4* in = static_cast<const uint4*>(src);
  uint4* out = static_cast<uint4*>(dst);
  if (rec_bytes == 16)
    k_records<1><<<io_blocks(n), kIoBlock, 0, s>>>(perm, n, in, out, to_caller ? 1 : 0);
  else
    k_records<2><<<io_blocks(n), kIoBlock, 0, s>>>(perm, n, in, out, to_caller ? 1 : 0);
}

}  // namespace plfbs

namespace plfbs {
namespace {

template <typename T>
__global__ void __launch_bounds__(kIoBlock) k_fill(T* __restrict__ p, long long n, T value) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = value;
}

}  // namespace

// perm[o] = device index of caller cell o (o < C) and of caller ghost C + b
__global__ void __launch_bounds__(kIoBlock)
    k_perm(const int32_t* __restrict__ cell_new, const int32_t* __restrict__ bc_new, int C,
           long long T, int32_t* __restrict__ perm) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  perm[i] = i < C ? cell_new[i] : C + bc_new[i - C];
}

void launch_perm(const int32_t* cell_new, const int32_t* bc_new, int C, int B, int32_t* perm,
                 cudaStream_t s) {
  const long long T = (long long)C + B;
  if (T > 0) k_perm<<<(unsigned)((T + kIoBlock - 1) / kIoBlock), kIoBlock, 0, s>>>(cell_new, bc_new, C, T, perm);
}

void launch_fill(double* p, long long n, double value, cudaStream_t s) {
  if (n > 0) k_fill<double><<<io_blocks(n), kIoBlock, 0, s>>>(p, n, value);
}
void launch_fill(float* p, long long n, float value, cudaStream_t s) {
  if (n > 0) k_fill<float><<<io_blocks(n), kIoBlock, 0, s>>>(p, n, value);
}

}  // namespace plfbs
