// Mesh checks of plfbs_create on the device. The checks are the host's
// (setup.cpp: validate_mesh): per face its owner and neighbour ranges and
// positive finite area, streaming dt and finite normal; per cell a positive
// finite volume and non-decreasing stencil offsets; per stencil entry its
// ranges and that it names a face neighbour of its cell; the largest stencil.
// Each kernel keeps the smallest failing index of its check (atomicMin), which
// is the index the host scan stops at, and the host writes the message for
// it from its own arrays: the same error whichever side scanned. On the
// device the scans read the arrays plfbs_create has already copied there, at
// HBM rate instead of the host's memory bandwidth.
#include <cuda_runtime.h>

#include "plfbs_internal.hpp"

namespace plfbs {
namespace {

constexpr int kScanBlock = 256;

__device__ __forceinline__ bool positive_finite(double x) { return x > 0.0 && isfinite(x); }

__global__ void __launch_bounds__(kScanBlock)
    k_scan_faces(const int32_t* __restrict__ owner, const int32_t* __restrict__ nb,
                 const double* __restrict__ area, const double* __restrict__ sdt,
                 const double* __restrict__ normal, int C, int F, int Fi, MeshScan* out) {
  int first = F;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
    const int o = owner[f], n = nb[f];
    bool bad = o < 0 || o >= C;
    if (f < Fi)
      bad = bad || n < 0 || n >= C || n == o;
    else
      bad = bad || n != C + (f - Fi);
    bad = bad || !positive_finite(area[f]) || !(sdt[f] > 0.0) ||
          !isfinite(normal[3 * (size_t)f]) || !isfinite(normal[3 * (size_t)f + 1]) ||
          !isfinite(normal[3 * (size_t)f + 2]);
    if (bad) {
      first = f;  // a thread's faces ascend: its first is its smallest
      break;
    }
  }
  if (first < F) atomicMin(&out->bad_face, first);
}

__global__ void __launch_bounds__(kScanBlock)
    k_scan_cells(const double* __restrict__ vol, const int32_t* __restrict__ off, int C,
                 MeshScan* out) {
  int first_vol = C, first_off = C, kmax = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x) {
    if (first_vol == C && !positive_finite(vol[i])) first_vol = i;
    const int k = off[i + 1] - off[i];
    if (first_off == C && k < 0) first_off = i;
    kmax = max(kmax, k);
  }
  if (first_vol < C) atomicMin(&out->bad_volume, first_vol);
  if (first_off < C) atomicMin(&out->bad_offset, first_off);
  atomicMax(&out->kmax, kmax);
}

// Entries of cell i lie in [off[i], off[i+1]); a cell whose range leaves
// [0, nnz) is skipped (its offsets fail k_scan_cells or the host's
// offsets[0] check, which the host reports first).
__global__ void __launch_bounds__(kScanBlock)
    k_scan_stencil(const int32_t* __restrict__ off, const int32_t* __restrict__ cells,
                   const int32_t* __restrict__ faces, const int32_t* __restrict__ owner,
                   const int32_t* __restrict__ nb, int C, int F, int Fi, long long T,
                   long long nnz, MeshScan* out) {
  int first = C;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x) {
    const int e0 = off[i], e1 = off[i + 1];
    if (e0 < 0 || e1 < e0 || e1 > nnz) continue;
    bool bad = false;
    for (int e = e0; e < e1 && !bad; e++) {
      const int j = cells[e], f = faces[e];
      if (j < 0 || j >= T || f < 0 || f >= F) {
        bad = true;
      } else {
        const int o = owner[f], n = nb[f];
        bad = !((o == i && n == j) || (f < Fi && n == i && o == j));
      }
    }
    if (bad) {
      first = i;
      break;
    }
  }
  if (first < C) atomicMin(&out->bad_stencil, first);
}

__global__ void k_scan_init(MeshScan* out, int C, int F) { *out = MeshScan{F, C, C, C, 0}; }

int scan_grid(long long n) {
  const long long b = (n + kScanBlock - 1) / kScanBlock;
  return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

}  // namespace

void launch_mesh_scan(const int32_t* owner, const int32_t* nb, const double* area,
                      const double* sdt, const double* normal, const double* vol,
                      const int32_t* off, const int32_t* cells, const int32_t* faces, int C, int F,
                      int Fi, long long nnz, MeshScan* out, cudaStream_t s) {
  k_scan_init<<<1, 1, 0, s>>>(out, C, F);
  k_scan_faces<<<scan_grid(F), kScanBlock, 0, s>>>(owner, nb, area, sdt, normal, C, F, Fi, out);
  k_scan_cells<<<scan_grid(C), kScanBlock, 0, s>>>(vol, off, C, out);
  k_scan_stencil<<<scan_grid(C), kScanBlock, 0, s>>>(off, cells, faces, owner, nb, C, F, Fi,
                                                     (long long)C + (F - Fi), nnz, out);
}

}  // namespace plfbs
