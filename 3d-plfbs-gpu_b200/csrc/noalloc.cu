// Residual norms with no device allocation.
//
// Some callers cannot let a library call cudaMalloc while they run: an
// application under a fixed device-memory budget that reserves all of its
// memory at start-up (an allocation mid-run can fail, and cudaMalloc may
// synchronise the device), or a host framework whose own caching allocator
// must own every byte of device memory. plfbs_residual_norms_noalloc serves
// them: it computes the same residual norms as the last RK stage of
// plfbs_run (Solver_gpu.cu:820-833 -> residuals.cpp:95-147) from residuals
// the caller keeps in its own device memory, writing to the caller's output
// buffer, and its only scratch (per-block partial sums and a completion
// counter) is the file-scope array below, which every GPU that loads this
// library holds until the process exits.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "plfbs.h"
#include "plfbs_internal.hpp"

namespace plfbs {
namespace {

constexpr int kNaThreads = 256;
constexpr int kNaCellsPerThread = 16;
constexpr int kNaCellsPerBlock = kNaThreads * kNaCellsPerThread;  // 4096
constexpr int kNaMaxBlocks = 2048;
constexpr long long kNaMaxCells = (long long)kNaMaxBlocks * kNaCellsPerBlock;  // 8,388,608
// 4 partial sums per block, then 32 doubles whose first 8 bytes hold the
// counter: 2048 * 4 * 8 + 256 = 65,792 bytes in all.
constexpr int kNaScratchDoubles = 4 * kNaMaxBlocks + 32;
constexpr int kNaMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNaScratchDoubles];

__device__ __forceinline__ double na_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block b reduces cells [b * 4096, (b + 1) * 4096); the last block to finish
// sums the partials in block order and writes
// out = {max_error, rho_rms, u_rms, v_rms, w_rms}.
// VEC: the residual array is 32-byte aligned and each cell's record moves as
// one 256-bit load; otherwise (a caller's pointer of lesser alignment) as four
// 8-byte loads.
template <bool VEC>
__global__ void __launch_bounds__(kNaThreads)
k_residual_norms_scratch(const double* __restrict__ res, long long n, double inv_ref_rho,
                         double inv_ref_mom, double* scratch, double* out) {
  unsigned long long* counter = reinterpret_cast<unsigned long long*>(scratch + 4 * kNaMaxBlocks);
  const long long base = (long long)blockIdx.x * kNaCellsPerBlock;
  double s[4] = {0.0, 0.0, 0.0, 0.0};  // rho, u, v, w
  for (int k = 0; k < kNaCellsPerThread; k++) {
    const long long i = base + (long long)k * kNaThreads + threadIdx.x;
    if (i < n) {
      double u, v, w, r;
      if (VEC) {
        asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
            : "=d"(u), "=d"(v), "=d"(w), "=d"(r)
            : "l"(res + 4 * i));
      } else {
        u = res[4 * i];
        v = res[4 * i + 1];
        w = res[4 * i + 2];
        r = res[4 * i + 3];
      }
      s[0] = fma(r, r, s[0]);
      s[1] = fma(u, u, s[1]);
      s[2] = fma(v, v, s[2]);
      s[3] = fma(w, w, s[3]);
    }
  }
  __shared__ double red[kNaThreads / 32][4];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const double v = na_warp_sum(s[c]);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int w = 0; w < kNaThreads / 32; w++) v += red[w][threadIdx.x];
    scratch[4LL * blockIdx.x + threadIdx.x] = v;
    __threadfence();  // only the writers of the partials need to publish them
  }
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1ull) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kNaThreads) {
#pragma unroll
    for (int c = 0; c < 4; c++) v[c] += __ldcg(scratch + 4LL * b + c);
  }
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const double t = na_warp_sum(v[c]);
    if (lane == 0) red[warp][c] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[4];
    for (int c = 0; c < 4; c++) {
      tot[c] = 0.0;
      for (int w = 0; w < kNaThreads / 32; w++) tot[c] += red[w][c];
    }
    const double nc = (double)n;
    const double rho_rms = sqrt(tot[0] / nc) * inv_ref_rho;
    const double u_rms = sqrt(tot[1] / nc) * inv_ref_mom;
    const double v_rms = sqrt(tot[2] / nc) * inv_ref_mom;
    const double w_rms = sqrt(tot[3] / nc) * inv_ref_mom;
    out[0] = fmax(fmax(w_rms, u_rms), v_rms);  // residuals::max_error
    out[1] = rho_rms;
    out[2] = u_rms;
    out[3] = v_rms;
    out[4] = w_rms;
    *counter = 0ull;
  }
}

// Device address of g_noalloc_scratch per device: looked up again on every
// call made outside stream capture (so it follows a device reset or another
// driver context), and the last address seen is what a call under capture
// uses.
std::mutex g_na_mutex;
double* g_na_ptr[kNaMaxDevices] = {};

int na_fail(int code, const std::string& m) {
  set_global_error(m);  // read back with plfbs_last_error(NULL)
  return code;
}

}  // namespace
}  // namespace plfbs

extern "C" int plfbs_residual_norms_noalloc(const double* residual, int64_t n_cells,
                                            double ref_rho, double max_velocity, double* out,
                                            void* stream) {
  using namespace plfbs;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!residual || !out)
    return na_fail(PLFBS_ERR_ARG, "residual_norms_noalloc: null residual or output pointer");
  if (n_cells <= 0 || n_cells > kNaMaxCells)
    return na_fail(PLFBS_ERR_ARG,
                   "residual_norms_noalloc: n_cells must be in [1, 8388608] (the static "
                   "scratch holds 2048 block partials of 4096 cells each)");
  if (!(ref_rho > 0) || !(max_velocity > 0))
    return na_fail(PLFBS_ERR_ARG, "residual_norms_noalloc: ref_rho and max_velocity must be > 0");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return na_fail(PLFBS_ERR_NO_DEVICE, std::string("residual_norms_noalloc: cudaGetDevice: ") +
                                            cudaGetErrorString(e));
  if (dev < 0 || dev >= kNaMaxDevices)
    return na_fail(PLFBS_ERR_NO_DEVICE, "residual_norms_noalloc: device ordinal " +
                                            std::to_string(dev) + " is beyond the " +
                                            std::to_string(kNaMaxDevices) +
                                            " devices this entry point supports");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) {
    cap = cudaStreamCaptureStatusActive;  // the query itself is refused during some captures
    cudaGetLastError();
  }
  if (cap == cudaStreamCaptureStatusNone) {
    // the device address of the scratch in the current context
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return na_fail(PLFBS_ERR_CUDA, std::string("residual_norms_noalloc: cudaGetSymbolAddress: ") +
                                         cudaGetErrorString(e));
    g_na_ptr[dev] = p;
  } else if (!g_na_ptr[dev]) {
    return na_fail(PLFBS_ERR_STATE,
                   "residual_norms_noalloc: the first call on a device must come before any "
                   "stream capture (it looks up the scratch's device address)");
  }
  double* scratch = g_na_ptr[dev];
  // the completion counter must start at zero whatever an earlier call left
  e = cudaMemsetAsync(scratch + 4 * kNaMaxBlocks, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess)
    return na_fail(PLFBS_ERR_CUDA, std::string("residual_norms_noalloc: cudaMemsetAsync: ") +
                                       cudaGetErrorString(e));
  const int blocks = (int)((n_cells + kNaCellsPerBlock - 1) / kNaCellsPerBlock);
  const double irr = 1.0 / ref_rho, irm = 1.0 / (ref_rho * max_velocity);
  if ((reinterpret_cast<uintptr_t>(residual) & 31) == 0)
    k_residual_norms_scratch<true><<<blocks, kNaThreads, 0, s>>>(residual, n_cells, irr, irm,
                                                                 scratch, out);
  else
    k_residual_norms_scratch<false><<<blocks, kNaThreads, 0, s>>>(residual, n_cells, irr, irm,
                                                                  scratch, out);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return na_fail(PLFBS_ERR_CUDA, std::string("residual_norms_noalloc: launch: ") +
                                       cudaGetErrorString(e));
  return PLFBS_OK;
}
