// Device build of the solver layout from the caller's mesh arrays: internal
// face order, face records, least-squares stencil weights, face-to-cell
// gather, inverse volumes and the mesh fingerprint; and the mesh arrays
// themselves from a raw polyMesh (plfbs_polymesh_geometry).
//
// The host keeps validation, the boundary records (a few percent of the
// faces) and, for renumber 1, the cell renumbering (a sequential breadth-first
// search; renumber 2 builds the same order here, level by level); everything
// O(faces) or O(stencil entries) happens here. The result
// is bit-identical to evaluating the same formulas on the host: this file is
// compiled without FMA contraction (-fmad=false), uses x * x where the
// reference writes pow(x, 2.0) (which gcc also folds to one multiply), and
// otherwise only IEEE add, multiply, divide and sqrt in the host's order.
#include <cstdint>

#include "plfbs_internal.hpp"
#include "rcm_levels.hpp"

namespace plfbs {
namespace {

constexpr int kLayoutBlock = 256;
constexpr int kWinBlock = 1024;   // window scan: 4 owners per thread
constexpr int kRankBlock = 256;
constexpr int kSigs = 2187;       // 3^7 upwind signatures
static_assert(kFaceWindow == 4 * kWinBlock, "window scan assumes 4 owners per thread");

__device__ __forceinline__ int new_cell(const DevMesh& m, int old) {
  return old < m.C ? m.cell_new[old] : m.C + m.bc_new[old - m.C];
}

// Branch signature of a face for the 7 opposite lattice pairs of D3Q15 (first
// members x, y, z, (1,1,1), (1,1,-1), (1,-1,1), (-1,1,1)): 1 if e.n > 0.001 dt,
// 2 if e.n < -0.001 dt, 0 in between (LBFS.cu:353-354), packed base 3.
__device__ int upwind_signature(const double* n, double dt) {
  const int E[7][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 1},
                       {1, 1, -1}, {1, -1, 1}, {-1, 1, 1}};
  const double d1 = 0.001 * dt;
  int sig = 0, p3 = 1;
#pragma unroll
  for (int p = 0; p < 7; p++, p3 *= 3) {
    const double s = E[p][0] * n[0] + E[p][1] * n[1] + E[p][2] * n[2];
    sig += p3 * (s > d1 ? 1 : (s < -d1 ? 2 : 0));
  }
  return sig;
}

// Faces per cell: internal faces by (new) owner, and all faces touching a cell.
__global__ void k_count(const DevMesh m, int32_t* own_cnt, int32_t* deg) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.F; f += gridDim.x * blockDim.x) {
    const int o = m.cell_new[m.owner[f]];
    atomicAdd(&deg[o], 1);
    if (f < m.Fi) {
      atomicAdd(&own_cnt[o], 1);
      atomicAdd(&deg[m.cell_new[m.neighbour[f]]], 1);
    }
  }
}

// Block-wide exclusive scan of one int per thread; returns the block total.
template <int BLOCK>
__device__ int block_exclusive_scan(int v, int& excl) {
  __shared__ int warp_sum[BLOCK / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) warp_sum[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < BLOCK / 32 ? warp_sum[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, d);
      if (lane >= d) s += y;
    }
    if (lane < BLOCK / 32) warp_sum[lane] = s;  // inclusive
  }
  __syncthreads();
  const int before = w > 0 ? warp_sum[w - 1] : 0;
  const int total = warp_sum[BLOCK / 32 - 1];
  excl = before + x - v;
  __syncthreads();  // warp_sum is reused by the next call
  return total;
}

// One block per window of kFaceWindow owners: offsets of each owner's internal
// faces within the window, the window's total, and the largest face count of
// a cell (the gather width).
__global__ void __launch_bounds__(kWinBlock) k_window_scan(const DevMesh m, const int32_t* own_cnt,
                                                           const int32_t* deg, int32_t* own_off,
                                                           int32_t* wsum, int32_t* info) {
  const int o0 = blockIdx.x * kFaceWindow + 4 * threadIdx.x;
  int c[4], s = 0, dmax = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    c[j] = o0 + j < m.C ? own_cnt[o0 + j] : 0;
    s += c[j];
    if (o0 + j < m.C) dmax = max(dmax, deg[o0 + j]);
  }
  int excl = 0;
  const int total = block_exclusive_scan<kWinBlock>(s, excl);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    if (o0 + j < m.C) own_off[o0 + j] = excl;
    excl += c[j];
  }
  if (threadIdx.x == 0) wsum[blockIdx.x] = total;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, d));
  if ((threadIdx.x & 31) == 0) atomicMax(&info[1], dmax);
}

// Exclusive scan of the window totals (one block, any number of windows).
__global__ void __launch_bounds__(kWinBlock) k_window_base(const int32_t* wsum, int nwin,
                                                           int32_t* wbase) {
  int carry = 0;
  for (int base = 0; base < nwin; base += kWinBlock) {
    const int i = base + threadIdx.x;
    const int v = i < nwin ? wsum[i] : 0;
    int excl = 0;
    const int total = block_exclusive_scan<kWinBlock>(v, excl);
    if (i < nwin) wbase[i] = carry + excl;
    carry += total;
  }
  if (threadIdx.x == 0) wbase[nwin] = carry;
}

// Internal faces into per-owner segments (in arbitrary order within a segment).
__global__ void k_scatter(const DevMesh m, const int32_t* own_off, const int32_t* wbase,
                          int32_t* cursor, int32_t* seg) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.Fi; f += gridDim.x * blockDim.x) {
    const int o = m.cell_new[m.owner[f]];
    seg[wbase[o / kFaceWindow] + own_off[o] + atomicAdd(&cursor[o], 1)] = f;
  }
}

// Each owner's segment sorted by (new neighbour, face): a few entries, insertion sort.
__global__ void k_owner_sort(const DevMesh m, const int32_t* own_cnt, const int32_t* own_off,
                             const int32_t* wbase, int32_t* seg) {
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < m.C; o += gridDim.x * blockDim.x) {
    const int n = own_cnt[o];
    if (n < 2) continue;
    int32_t* s = seg + wbase[o / kFaceWindow] + own_off[o];
    auto key = [&](int f) { return ((uint64_t)(uint32_t)m.cell_new[m.neighbour[f]] << 32) | (uint32_t)f; };
    for (int i = 1; i < n; i++) {
      const int x = s[i];
      const uint64_t kx = key(x);
      int j = i - 1;
      while (j >= 0 && key(s[j]) > kx) {
        s[j + 1] = s[j];
        j--;
      }
      s[j + 1] = x;
    }
  }
}

// One block per window: faces grouped by upwind signature, owner order (and
// the segment order within an owner) kept inside each group. Signature counts
// and their prefix come from the whole block; the ordered placement is one
// warp walking the window's faces 32 at a time, ranking equal signatures with
// __match_any_sync.
__global__ void __launch_bounds__(kRankBlock) k_window_rank(const DevMesh m, const int32_t* wbase,
                                                            const int32_t* seg, uint16_t* sig_of,
                                                            int32_t* face_order) {
  __shared__ int cnt[kSigs];
  const int lo = wbase[blockIdx.x], hi = wbase[blockIdx.x + 1];
  for (int i = threadIdx.x; i < kSigs; i += kRankBlock) cnt[i] = 0;
  __syncthreads();
  for (int p = lo + threadIdx.x; p < hi; p += kRankBlock) {
    const int f = seg[p];
    const int s = upwind_signature(m.normal + 3 * (size_t)f, m.sdt[f]);
    sig_of[p] = (uint16_t)s;
    atomicAdd(&cnt[s], 1);
  }
  __syncthreads();
  constexpr int kPer = (kSigs + kRankBlock - 1) / kRankBlock;
  const int i0 = threadIdx.x * kPer;
  int sum = 0;
  for (int j = 0; j < kPer; j++)
    if (i0 + j < kSigs) sum += cnt[i0 + j];
  int excl = 0;
  block_exclusive_scan<kRankBlock>(sum, excl);
  for (int j = 0; j < kPer; j++)
    if (i0 + j < kSigs) {
      const int c = cnt[i0 + j];
      cnt[i0 + j] = excl;
      excl += c;
    }
  __syncthreads();
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  const unsigned lt = (1u << lane) - 1u;
  constexpr int kBatch = 8;
  for (int base = lo; base < hi; base += 32 * kBatch) {
    int f[kBatch], s[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; j++) {
      const int p = base + 32 * j + lane;
      f[j] = p < hi ? seg[p] : -1;
      s[j] = p < hi ? (int)sig_of[p] : kSigs + lane;  // unique key for idle lanes
    }
#pragma unroll
    for (int j = 0; j < kBatch; j++) {
      const unsigned mask = __match_any_sync(0xffffffffu, s[j]);
      const bool valid = f[j] >= 0;
      const int old = valid ? cnt[s[j]] : 0;
      __syncwarp();
      if (valid && lane == __ffs(mask) - 1) cnt[s[j]] = old + __popc(mask);
      __syncwarp();
      if (valid) face_order[lo + old + __popc(mask & lt)] = f[j];
    }
  }
}

// Face records and ids in the new face order (boundary faces after the
// internal ones, by new boundary index).
template <typename T4>
__global__ void k_faces(const DevMesh m, double visc3, double pg, int32_t* face_order,
                        int2* face_ids, T4* face0, T4* face1, T4* face2) {
  using T = decltype(T4::x);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m.F; k += gridDim.x * blockDim.x) {
    int f;
    if (k < m.Fi) {
      f = face_order[k];
    } else {
      f = m.Fi + m.bc_old[k - m.Fi];
      face_order[k] = f;
    }
    const int o = m.owner[f], nbo = m.neighbour[f];
    const double* n = m.normal + 3 * (size_t)f;
    const double* xf = m.fcen + 3 * (size_t)f;
    const double* c1 = m.ccen + 3 * (size_t)o;
    const double* c2 = m.ccen + 3 * (size_t)nbo;
    const double dt = m.sdt[f];
    face0[k] = T4{(T)n[0], (T)n[1], (T)n[2], (T)m.area[f]};
    face1[k] = T4{(T)dt, (T)(c1[0] - xf[0]), (T)(c1[1] - xf[1]), (T)(c1[2] - xf[2])};
    face2[k] = T4{(T)(c2[0] - xf[0]), (T)(c2[1] - xf[1]), (T)(c2[2] - xf[2]),
                  (T)(visc3 / dt * pg)};
    face_ids[k] = make_int2(m.cell_new[o], k < m.Fi ? m.cell_new[nbo] : m.C + (k - m.Fi));
  }
}

// Least-squares weights of gradients::pre_fill_LHS_and_RHS_matrix
// (gradients.cpp:214-313, with add_non_macrovariable_contributions,
// gradients.cpp:149-210) and their precombination LHS^-1 . RHS_e into the
// slot-major stencil; the reference's determinant (gradients.cpp:282-284)
// unless `mode` has PLFBS_GRAD_EXACT_INVERSE. Also 1 / volume.
template <typename T>
__global__ void k_cells(const DevMesh m, int mode, int32_t* st_nbr, T* st_wx, T* st_wy, T* st_wz,
                        T* inv_volume, int32_t* info) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.C; i += gridDim.x * blockDim.x) {
    const int in = m.cell_new[i];
    const double vol = m.vol[i];
    inv_volume[in] = (T)(1.0 / vol);
    const double* ci = m.ccen + 3 * (size_t)i;
    const int e0 = m.st_off[i], e1 = m.st_off[i + 1];
    double max_area = 0.0, max_disp = 0.0;
    for (int e = e0; e < e1; e++) {
      const int i1 = m.st_cells[e], f = m.st_faces[e];
      max_area = fmax(max_area, m.area[f]);
      const double* c1 = m.ccen + 3 * (size_t)i1;
      const double dx = c1[0] - ci[0], dy = c1[1] - ci[1], dz = c1[2] - ci[2];
      const double disp = sqrt(dx * dx + dy * dy + dz * dz);
      max_disp = max_disp < disp ? disp : max_disp;
    }
    const double aspect = 2 * fabs(max_disp) * max_area / vol;
    const int base = mode & 0xff;
    double beta = 0.0;
    if (base == PLFBS_GRAD_HYBRID) {
      const double b = 2 / aspect;
      beta = b < 1.0 ? b : 1.0;
    } else if (base == PLFBS_GRAD_LS) {
      beta = 1.0;
    }
    const double diag = 2 * (1 - beta) * vol;
    double L[9] = {0.0 + diag, 0, 0, 0, 0.0 + diag, 0, 0, 0, 0.0 + diag};
    for (int e = e0; e < e1; e++) {
      const int i1 = m.st_cells[e], f = m.st_faces[e];
      const double* xf = m.fcen + 3 * (size_t)f;
      const double* n = m.normal + 3 * (size_t)f;
      const double l_norm = (xf[0] - ci[0]) * n[0] + (xf[1] - ci[1]) * n[1] + (xf[2] - ci[2]) * n[2];
      const double* c1 = m.ccen + 3 * (size_t)i1;
      const double d[3] = {c1[0] - ci[0], c1[1] - ci[1], c1[2] - ci[2]};
      const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      const double L_norm = d[0] * n[0] + d[1] * n[1] + d[2] * n[2];
      const double q = 2 * l_norm / L_norm;
      const double w = q * q * m.area[f] / len;
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) L[3 * r + c] = L[3 * r + c] + w * d[r] * d[c] * beta;
    }
    const double a = L[0], b = L[1], c = L[2], dd = L[3], e = L[4], f = L[5], g = L[6], h = L[7],
                 k = L[8];
    const double det = (mode & PLFBS_GRAD_EXACT_INVERSE)
                           ? a * (e * k - f * h) - b * (dd * k - f * g) + c * (dd * h - e * g)
                           : a * (e * k - f * h) + b * (dd * k - f - g) + c * (dd * h - e * g);
    double Li[9];
    Li[0] = 1 / det * (e * k - f * h);
    Li[1] = 1 / det * (c * h - b * k);
    Li[2] = 1 / det * (b * f - c * e);
    Li[3] = 1 / det * (f * g - dd * k);
    Li[4] = 1 / det * (a * k - c * g);
    Li[5] = 1 / det * (c * dd - a * f);
    Li[6] = 1 / det * (dd * h - e * g);
    Li[7] = 1 / det * (b * g - a * h);
    Li[8] = 1 / det * (a * e - b * dd);
    if (!isfinite(Li[0]) || !isfinite(Li[4]) || !isfinite(Li[8])) atomicMin(&info[0], i);
    int slot = 0;
    for (int ee = e0; ee < e1; ee++, slot++) {
      const int i1 = m.st_cells[ee], fc = m.st_faces[ee];
      const double* n = m.normal + 3 * (size_t)fc;
      const double* c1 = m.ccen + 3 * (size_t)i1;
      const double* xf = m.fcen + 3 * (size_t)fc;
      const double l_norm = (xf[0] - ci[0]) * n[0] + (xf[1] - ci[1]) * n[1] + (xf[2] - ci[2]) * n[2];
      const double d[3] = {c1[0] - ci[0], c1[1] - ci[1], c1[2] - ci[2]};
      const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      const double s = m.area[fc];
      const double L_norm = d[0] * n[0] + d[1] * n[1] + d[2] * n[2];
      const double q = 2 * l_norm / L_norm;
      const double w = q * q * s / len;
      const bool own = m.owner[fc] == i;
      double r[3];
#pragma unroll
      for (int cc = 0; cc < 3; cc++)
        r[cc] = own ? beta * w * d[cc] + 2 * (1 - beta) * 0.5 * n[cc] * s
                    : beta * w * d[cc] + 2 * (1 - beta) * 0.5 * n[cc] * -1 * s;
      const size_t o = (size_t)slot * m.C + in;
      st_nbr[o] = new_cell(m, i1);
      st_wx[o] = (T)(Li[0] * r[0] + Li[1] * r[1] + Li[2] * r[2]);
      st_wy[o] = (T)(Li[3] * r[0] + Li[4] * r[1] + Li[5] * r[2]);
      st_wz[o] = (T)(Li[6] * r[0] + Li[7] * r[1] + Li[8] * r[2]);
    }
  }
}

// Face-to-cell gather: (k << 1) | side appended per cell, then each cell's
// slots sorted ascending (the order of a loop over the new faces).
__global__ void k_gather_fill(const DevMesh m, const int2* face_ids, int32_t* cnt, int32_t* gather) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m.F; k += gridDim.x * blockDim.x) {
    const int2 id = face_ids[k];
    gather[(size_t)atomicAdd(&cnt[id.x], 1) * m.C + id.x] = k << 1;
    if (k < m.Fi) gather[(size_t)atomicAdd(&cnt[id.y], 1) * m.C + id.y] = (k << 1) | 1;
  }
}

__global__ void k_gather_sort(const DevMesh m, const int32_t* cnt, int32_t* gather) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m.C; c += gridDim.x * blockDim.x) {
    const int n = cnt[c];
    for (int i = 1; i < n; i++) {
      const int x = gather[(size_t)i * m.C + c];
      int j = i - 1;
      while (j >= 0 && gather[(size_t)j * m.C + c] > x) {
        gather[(size_t)(j + 1) * m.C + c] = gather[(size_t)j * m.C + c];
        j--;
      }
      gather[(size_t)(j + 1) * m.C + c] = x;
    }
  }
}

// splitmix64's output function (Steele, Lea and Flood, 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

// Sum (mod 2^64) of mix64(word + mix64(tag, index)) over the words of
// owner, neighbour, face area and cell volume: order-sensitive in the data,
// independent of the summation order.
__global__ void k_fingerprint(const DevMesh m, unsigned long long* out) {
  uint64_t h = 0;
  const long long nF = m.F, nC = m.C;
  const long long total = 3 * nF + nC;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    uint64_t w, tag;
    long long i;
    if (t < nF) {
      i = t, tag = 1, w = (uint32_t)m.owner[i];
    } else if (t < 2 * nF) {
      i = t - nF, tag = 2, w = (uint32_t)m.neighbour[i];
    } else if (t < 3 * nF) {
      i = t - 2 * nF, tag = 3, w = (uint64_t)__double_as_longlong(m.area[i]);
    } else {
      i = t - 3 * nF, tag = 4, w = (uint64_t)__double_as_longlong(m.vol[i]);
    }
    h += mix64(w + mix64((tag << 56) ^ (uint64_t)i));
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) h += __shfl_xor_sync(0xffffffffu, h, d);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)h);
}

// ---------------------------------------------------------------------------
// Mesh geometry from a polyMesh (unstructured_mesh::generate_internal_mesh,
// unstructured_mesh.cpp:1133-1233): every sum in the reference's order.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void point(const DevPolyMesh& pm, int i, double v[3]) {
  v[0] = (double)pm.points[3 * (size_t)i];  // points are single precision (unstructured_mesh.h:50)
  v[1] = (double)pm.points[3 * (size_t)i + 1];
  v[2] = (double)pm.points[3 * (size_t)i + 2];
}

// (b - a) x (c - a) of the fan triangle (0, t+1, t+2) of face f and the
// vertex a (tet_volume, unstructured_mesh.cpp:577-607; cell_tet_area, :732-766).
__device__ __forceinline__ void fan_triangle(const DevPolyMesh& pm, int o0, int t, double a[3],
                                             double b[3], double c[3], double cr[3]) {
  point(pm, pm.face_points[o0], a);
  point(pm, pm.face_points[o0 + t + 1], b);
  point(pm, pm.face_points[o0 + t + 2], c);
  const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const double w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  cr[0] = u[1] * w[2] - u[2] * w[1];
  cr[1] = u[2] * w[0] - u[0] * w[2];
  cr[2] = u[0] * w[1] - u[1] * w[0];
}

// Per face: area, unit normal, centroid (area-weighted triangle centroids),
// the un-normalised centroid sum the cell centroids accumulate, the streaming
// dt min(sqrt(A)/2, ref_dt) (calc_face_delta_t, :979-983), and faces per cell.
__global__ void k_face_geometry(const DevPolyMesh pm, double ref_dt, const GeometryOut o,
                                double* fcsum, int32_t* cnt) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < pm.F; f += gridDim.x * blockDim.x) {
    const int o0 = pm.face_offsets[f], nv = pm.face_offsets[f + 1] - o0;
    double A = 0.0, cs[3] = {0.0, 0.0, 0.0}, n[3] = {0.0, 0.0, 0.0};
    for (int t = 0; t < nv - 2; t++) {
      double a[3], b[3], c[3], cr[3];
      fan_triangle(pm, o0, t, a, b, c, cr);
      const double ar = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      A = A + ar;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double d = (a[k] + b[k] + c[k]) / 3;
        cs[k] = cs[k] + d / (1 / ar);
        n[k] = n[k] + cr[k];
      }
    }
    const double mag = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    o.area[f] = A;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      fcsum[3 * (size_t)f + k] = cs[k];
      o.fcen[3 * (size_t)f + k] = cs[k] / A;
      o.normal[3 * (size_t)f + k] = n[k] / mag;
    }
    const double sd = 0.5 * sqrt(A);
    o.sdt[f] = ref_dt < sd ? ref_dt : sd;
    atomicAdd(&cnt[pm.owner[f]], 1);
    if (f < pm.Fi) atomicAdd(&cnt[pm.neighbour[f]], 1);
  }
}

__global__ void k_csr_offsets(int C, const int32_t* own_off, const int32_t* wbase, int nwin,
                              int32_t* off) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= C; c += gridDim.x * blockDim.x)
    off[c] = c < C ? wbase[c / kFaceWindow] + own_off[c] : wbase[nwin];
}

__global__ void k_csr_scatter(const DevPolyMesh pm, const int32_t* off, int32_t* cursor,
                              int32_t* faces) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < pm.F; f += gridDim.x * blockDim.x) {
    const int o = pm.owner[f];
    faces[off[o] + atomicAdd(&cursor[o], 1)] = f;
    if (f < pm.Fi) {
      const int n = pm.neighbour[f];
      faces[off[n] + atomicAdd(&cursor[n], 1)] = f;
    }
  }
}

// Per cell: its faces ascending (the gradient stencil, :1186-1206), volume
// (owner +, neighbour - per fan triangle, face by face), centroid (sum of the
// faces' centroid sums over the sum of their areas, :1170-1217).
__global__ void k_cell_geometry(const DevPolyMesh pm, const GeometryOut o, const double* fcsum) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < pm.C; c += gridDim.x * blockDim.x) {
    const int e0 = o.st_off[c], e1 = o.st_off[c + 1];
    int32_t* fs = o.st_faces;
    for (int i = e0 + 1; i < e1; i++) {
      const int x = fs[i];
      int j = i - 1;
      while (j >= e0 && fs[j] > x) {
        fs[j + 1] = fs[j];
        j--;
      }
      fs[j + 1] = x;
    }
    double vol = 0.0, tca = 0.0, cen[3] = {0.0, 0.0, 0.0};
    for (int e = e0; e < e1; e++) {
      const int f = fs[e];
      const bool own = pm.owner[f] == c;
      o.st_cells[e] = own ? (f < pm.Fi ? pm.neighbour[f] : pm.C + (f - pm.Fi)) : pm.owner[f];
      tca = tca + o.area[f];
#pragma unroll
      for (int k = 0; k < 3; k++) cen[k] = cen[k] + fcsum[3 * (size_t)f + k];
      const int q0 = pm.face_offsets[f], nv = pm.face_offsets[f + 1] - q0;
      for (int t = 0; t < nv - 2; t++) {
        double a[3], b[3], cc[3], cr[3];
        fan_triangle(pm, q0, t, a, b, cc, cr);
        const double v = (a[0] * cr[0] + a[1] * cr[1] + a[2] * cr[2]) / 6;
        vol = own ? vol + v : vol + -v;
      }
    }
    o.vol[c] = vol;
#pragma unroll
    for (int k = 0; k < 3; k++) o.ccen[3 * (size_t)c + k] = cen[k] / tca;
  }
}

// Ghost cells (populate_ghost_cell_from_foam_face, :1346-1375): owner centroid
// + 2 (face centroid - owner centroid) scaled componentwise by |n|; volume 0.
__global__ void k_ghost_geometry(const DevPolyMesh pm, const GeometryOut o) {
  const int B = pm.F - pm.Fi;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    const int f = pm.Fi + b;
    const double* oc = o.ccen + 3 * (size_t)pm.owner[f];
    double* g = o.ccen + 3 * ((size_t)pm.C + b);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double rel = (o.fcen[3 * (size_t)f + k] - oc[k]) / 0.5;
      g[k] = oc[k] + rel * fabs(o.normal[3 * (size_t)f + k]);
    }
    o.vol[pm.C + b] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// Exact deduplication of per-item records (face records, cells' weight sets):
// items whose records are bitwise equal share one table entry. Claim: each
// item's hash takes an open-addressed slot, the lowest item index with that
// hash becomes the slot's representative. Resolve: an item equal to its
// representative bit for bit maps to it, otherwise (a hash collision) to
// itself. Representatives are numbered in item order by the window scans.
// ---------------------------------------------------------------------------
constexpr int kMaxProbe = 1 << 12;

// Element j of item i's record, as its bits (FP64 or FP32).
__device__ __forceinline__ uint64_t rec_bits(const RecordSource& r, int i, int j) {
  const void* p;
  size_t e;
  if (r.kind == 0) {  // three 4-vector arrays [n]
    p = j < 4 ? r.p0 : (j < 8 ? r.p1 : r.p2);
    e = 4 * (size_t)i + (j & 3);
  } else {  // three slot-major arrays [K][n]
    const int k = j / 3, c = j - 3 * k;
    p = c == 0 ? r.p0 : (c == 1 ? r.p1 : r.p2);
    e = (size_t)k * r.n + i;
  }
  return r.fp32 ? (uint64_t)static_cast<const uint32_t*>(p)[e] : static_cast<const uint64_t*>(p)[e];
}
__device__ __forceinline__ int rec_width(const RecordSource& r) { return r.kind == 0 ? 12 : 3 * r.K; }

// Lanes of a warp with equal hashes claim once: the lowest of them (the
// smallest item index) does the atomics and hands the slot to the others, so
// the thousands of equal records of a structured mesh do not serialise on one
// slot.
__global__ void k_dedupe_claim(const RecordSource r, int P, unsigned long long* slot_hash,
                               int32_t* slot_rep, int32_t* item_slot, int32_t* overflow) {
  const int stride = gridDim.x * blockDim.x;
  const int W = rec_width(r);
  for (int base = blockIdx.x * blockDim.x; base < r.n; base += stride) {
    const int i = base + (int)threadIdx.x;
    const bool valid = i < r.n;
    uint64_t h = 0;
    if (valid) {
      h = 0x9e3779b97f4a7c15ull;
      for (int j = 0; j < W; j++)
        h = mix64(h ^ (rec_bits(r, i, j) + 0x632be59bd9b4e019ull * j));
      h |= 1;  // 0 marks an empty slot (and idle lanes)
    }
    const unsigned group = __match_any_sync(0xffffffffu, (unsigned long long)h);
    const int leader = __ffs(group) - 1;
    int slot = -1;
    if (valid && (int)(threadIdx.x & 31) == leader) {
      int pos = (int)(h & (uint64_t)(P - 1));
      for (int probe = 0; probe < kMaxProbe; probe++) {
        const unsigned long long prev = atomicCAS(slot_hash + pos, 0ull, (unsigned long long)h);
        if (prev == 0ull || prev == h) {
          atomicMin(slot_rep + pos, i);
          slot = pos;
          break;
        }
        pos = (pos + 1) & (P - 1);
      }
      if (slot < 0) atomicExch(overflow, 1);
    }
    slot = __shfl_sync(0xffffffffu, slot, leader);
    if (valid) item_slot[i] = slot;
  }
}

__global__ void k_dedupe_resolve(const RecordSource r, const int32_t* slot_rep,
                                 const int32_t* item_slot, int32_t* rep_of, int32_t* is_rep) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x) {
    const int s = item_slot[i];
    int rep = s < 0 ? i : slot_rep[s];
    if (rep != i) {
      const int W = rec_width(r);
      for (int j = 0; j < W; j++)
        if (rec_bits(r, i, j) != rec_bits(r, rep, j)) {
          rep = i;
          break;
        }
    }
    rep_of[i] = rep;
    is_rep[i] = rep == i;
  }
}

__device__ __forceinline__ void put_bits(void* t, size_t e, uint64_t v, int fp32) {
  if (fp32)
    static_cast<uint32_t*>(t)[e] = (uint32_t)v;
  else
    static_cast<uint64_t*>(t)[e] = v;
}

// Item -> table index, and the representatives' records into the table
// (kind 0: three 4-vector arrays [U]; kind 1: [U][K][3]), bit for bit.
__global__ void k_dedupe_emit(const RecordSource r, const int32_t* rep_of, const int32_t* off,
                              const int32_t* wbase, int32_t* index, void* t0, void* t1, void* t2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x) {
    const int rep = rep_of[i];
    const int id = wbase[rep / kFaceWindow] + off[rep];
    index[i] = id;
    if (rep != i) continue;
    if (r.kind == 0) {
      for (int j = 0; j < 12; j++)
        put_bits(j < 4 ? t0 : (j < 8 ? t1 : t2), 4 * (size_t)id + (j & 3), rec_bits(r, i, j),
                 r.fp32);
    } else {
      for (int j = 0; j < 3 * r.K; j++)
        put_bits(t0, (size_t)id * 3 * r.K + j, rec_bits(r, i, j), r.fp32);
    }
  }
}

// --- Cuthill-McKee order by breadth-first levels (renumber 2) ---------------
// The per-thread steps are rcm_levels.hpp's; the host drives one level at a
// time (capi_layout.cpp device_cell_order). Index checks that fail count in
// info[2] instead of touching memory.

__device__ __forceinline__ rcm::Graph rcm_graph(const RcmDev& r) {
  return rcm::Graph{r.C, r.off, r.adj, r.deg};
}

__global__ void k_rcm_degree(const RcmDev r) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < r.Fi; f += gridDim.x * blockDim.x) {
    atomicAdd(&r.deg[r.owner[f]], 1);
    atomicAdd(&r.deg[r.neighbour[f]], 1);
  }
}

// Each internal face into both cells' adjacency (arbitrary order within a cell).
__global__ void k_rcm_scatter(const RcmDev r) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < r.Fi; f += gridDim.x * blockDim.x) {
    const int o = r.owner[f], n = r.neighbour[f];
    r.adj_key[r.off[o] + atomicAdd(&r.cursor[o], 1)] = rcm::adj_entry(f, n);
    r.adj_key[r.off[n] + atomicAdd(&r.cursor[n], 1)] = rcm::adj_entry(f, o);
  }
}

// Each cell's adjacency into face order.
__global__ void k_rcm_sort(const RcmDev r) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < r.C; c += gridDim.x * blockDim.x) {
    const int e0 = r.off[c], e1 = r.off[c + 1];
    rcm::sort_entries(r.adj_key + e0, e1 - e0);
    for (int e = e0; e < e1; e++) r.adj[e] = (int32_t)(r.adj_key[e] & 0xffffffffu);
  }
}

__global__ void k_rcm_isolated(const RcmDev r) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < r.C; c += gridDim.x * blockDim.x)
    r.cnt[c] = r.deg[c] == 0 ? 1 : 0;
}

// Cells without internal faces first, by index (the window scan of the flags).
__global__ void k_rcm_place_isolated(const RcmDev r) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < r.C; c += gridDim.x * blockDim.x) {
    if (r.deg[c] != 0) continue;
    const int q = r.wbase[c / kFaceWindow] + r.win_off[c];
    r.order[q] = c;
    r.pos[c] = q;
  }
}

// Smallest (degree, cell) among the unvisited cells into *start.
__global__ void k_rcm_start(const RcmDev r) {
  unsigned long long best = rcm::kUnclaimed;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < r.C; c += gridDim.x * blockDim.x)
    if (r.pos[c] < 0) {
      const unsigned long long k = rcm::start_key(r.deg[c], c);
      best = k < best ? k : best;
    }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, best, d);
    best = o < best ? o : best;
  }
  if ((threadIdx.x & 31) == 0 && best != rcm::kUnclaimed) atomicMin(r.start, best);
}

// One thread: the start at order[q]; *start reset for the next component.
__global__ void k_rcm_place_start(const RcmDev r, int q) {
  const unsigned long long s = *r.start;
  *r.start = rcm::kUnclaimed;
  const long long c = (long long)(s & 0xffffffffu);
  if (s == rcm::kUnclaimed || c >= r.C || q < 0 || q >= r.C) {
    atomicAdd(&r.info[2], 1);
    return;
  }
  r.order[q] = (int32_t)c;
  r.pos[c] = q;
}

__global__ void k_rcm_claim(const RcmDev r, int lo, int hi) {
  const rcm::Graph g = rcm_graph(r);
  for (int p = lo + blockIdx.x * blockDim.x + threadIdx.x; p < hi; p += gridDim.x * blockDim.x) {
    const int v = r.order[p];
    if (v < 0 || v >= r.C) {
      atomicAdd(&r.info[2], 1);
      continue;
    }
    rcm::claim(g, r.pos, r.key, p, v,
               [](unsigned long long* a, unsigned long long x) { atomicMin(a, x); });
  }
}

__global__ void k_rcm_count(const RcmDev r, int lo, int hi) {
  const rcm::Graph g = rcm_graph(r);
  for (int p = lo + blockIdx.x * blockDim.x + threadIdx.x; p < hi; p += gridDim.x * blockDim.x) {
    const int v = r.order[p];
    r.cnt[p - lo] = (v >= 0 && v < r.C) ? rcm::count_children(g, r.key, p, v) : 0;
  }
}

__global__ void k_rcm_emit(const RcmDev r, int lo, int hi) {
  const rcm::Graph g = rcm_graph(r);
  for (int p = lo + blockIdx.x * blockDim.x + threadIdx.x; p < hi; p += gridDim.x * blockDim.x) {
    const int v = r.order[p];
    if (v < 0 || v >= r.C) continue;  // counted by k_rcm_claim
    const long long first = (long long)hi + r.wbase[(p - lo) / kFaceWindow] + r.win_off[p - lo];
    const int bad = rcm::emit_children(g, r.key, p, v, first, r.order, r.pos);
    if (bad) atomicAdd(&r.info[2], bad);
  }
}

int grid_for(long long n) {
  const long long g = (n + kLayoutBlock - 1) / kLayoutBlock;
  return (int)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

}  // namespace

void launch_polymesh_geometry(const DevPolyMesh& pm, double ref_dt, const GeometryOut& o,
                              const GeometryScratch& s, cudaStream_t st) {
  const int nwin = (pm.C + kFaceWindow - 1) / kFaceWindow;
  k_face_geometry<<<grid_for(pm.F), kLayoutBlock, 0, st>>>(pm, ref_dt, o, s.fcsum, s.cnt);
  DevMesh m{};
  m.C = pm.C;
  k_window_scan<<<nwin, kWinBlock, 0, st>>>(m, s.cnt, s.cnt, s.own_off, s.wsum, s.info);
  k_window_base<<<1, kWinBlock, 0, st>>>(s.wsum, nwin, s.wbase);
  k_csr_offsets<<<grid_for(pm.C + 1LL), kLayoutBlock, 0, st>>>(pm.C, s.own_off, s.wbase, nwin,
                                                               o.st_off);
  k_csr_scatter<<<grid_for(pm.F), kLayoutBlock, 0, st>>>(pm, o.st_off, s.cursor, o.st_faces);
  k_cell_geometry<<<grid_for(pm.C), kLayoutBlock, 0, st>>>(pm, o, s.fcsum);
  if (pm.F > pm.Fi)
    k_ghost_geometry<<<grid_for(pm.F - pm.Fi), kLayoutBlock, 0, st>>>(pm, o);
}

void launch_layout_order(const DevMesh& m, const LayoutScratch& s, int32_t* face_order,
                         cudaStream_t st) {
  const int nwin = (m.C + kFaceWindow - 1) / kFaceWindow;
  k_count<<<grid_for(m.F), kLayoutBlock, 0, st>>>(m, s.own_cnt, s.deg);
  k_window_scan<<<nwin, kWinBlock, 0, st>>>(m, s.own_cnt, s.deg, s.own_off, s.wsum, s.info);
  k_window_base<<<1, kWinBlock, 0, st>>>(s.wsum, nwin, s.wbase);
  if (m.Fi > 0) {
    k_scatter<<<grid_for(m.Fi), kLayoutBlock, 0, st>>>(m, s.own_off, s.wbase, s.cursor, s.seg);
    k_owner_sort<<<grid_for(m.C), kLayoutBlock, 0, st>>>(m, s.own_cnt, s.own_off, s.wbase, s.seg);
    k_window_rank<<<nwin, kRankBlock, 0, st>>>(m, s.wbase, s.seg, s.sig, face_order);
  }
  k_fingerprint<<<grid_for(3LL * m.F + m.C), kLayoutBlock, 0, st>>>(m, s.fingerprint);
}

void launch_layout_records(const DevMesh& m, const LayoutScratch& s, int precision, int mode,
                           double visc3, double pg, int32_t* face_order, int32_t* face_ids,
                           void* face0, void* face1, void* face2, int32_t* st_nbr, void* st_wx,
                           void* st_wy, void* st_wz, void* inv_volume, cudaStream_t st) {
  int2* ids = reinterpret_cast<int2*>(face_ids);
  if (precision == PLFBS_FP32_DEVIATION) {
    k_faces<float4><<<grid_for(m.F), kLayoutBlock, 0, st>>>(
        m, visc3, pg, face_order, ids, static_cast<float4*>(face0), static_cast<float4*>(face1),
        static_cast<float4*>(face2));
    k_cells<float><<<grid_for(m.C), kLayoutBlock, 0, st>>>(
        m, mode, st_nbr, static_cast<float*>(st_wx), static_cast<float*>(st_wy),
        static_cast<float*>(st_wz), static_cast<float*>(inv_volume), s.info);
  } else {
    k_faces<double4><<<grid_for(m.F), kLayoutBlock, 0, st>>>(
        m, visc3, pg, face_order, ids, static_cast<double4*>(face0), static_cast<double4*>(face1),
        static_cast<double4*>(face2));
    k_cells<double><<<grid_for(m.C), kLayoutBlock, 0, st>>>(
        m, mode, st_nbr, static_cast<double*>(st_wx), static_cast<double*>(st_wy),
        static_cast<double*>(st_wz), static_cast<double*>(inv_volume), s.info);
  }
}

void launch_dedupe_scan(const RecordSource& r, const DedupeScratch& d, cudaStream_t st) {
  const int nwin = (r.n + kFaceWindow - 1) / kFaceWindow;
  k_dedupe_claim<<<grid_for(r.n), kLayoutBlock, 0, st>>>(r, d.P, d.slot_hash, d.slot_rep,
                                                         d.item_slot, d.info);
  k_dedupe_resolve<<<grid_for(r.n), kLayoutBlock, 0, st>>>(r, d.slot_rep, d.item_slot, d.rep_of,
                                                           d.is_rep);
  DevMesh m{};
  m.C = r.n;
  k_window_scan<<<nwin, kWinBlock, 0, st>>>(m, d.is_rep, d.is_rep, d.off, d.wsum, d.info + 2);
  k_window_base<<<1, kWinBlock, 0, st>>>(d.wsum, nwin, d.wbase);
}

void launch_dedupe_emit(const RecordSource& r, const DedupeScratch& d, int32_t* index, void* t0,
                        void* t1, void* t2, cudaStream_t st) {
  k_dedupe_emit<<<grid_for(r.n), kLayoutBlock, 0, st>>>(r, d.rep_of, d.off, d.wbase, index, t0,
                                                        t1, t2);
}

void launch_layout_gather(const DevMesh& m, const LayoutScratch& s, const int32_t* face_ids,
                          int32_t* gather, cudaStream_t st) {
  const int2* ids = reinterpret_cast<const int2*>(face_ids);
  k_gather_fill<<<grid_for(m.F), kLayoutBlock, 0, st>>>(m, ids, s.gcnt, gather);
  k_gather_sort<<<grid_for(m.C), kLayoutBlock, 0, st>>>(m, s.gcnt, gather);
}

void launch_rcm_graph(const RcmDev& r, cudaStream_t st) {
  const int nwin = (r.C + kFaceWindow - 1) / kFaceWindow;
  DevMesh m{};
  m.C = r.C;
  if (r.Fi > 0) k_rcm_degree<<<grid_for(r.Fi), kLayoutBlock, 0, st>>>(r);
  k_window_scan<<<nwin, kWinBlock, 0, st>>>(m, r.deg, r.deg, r.win_off, r.wsum, r.info);
  k_window_base<<<1, kWinBlock, 0, st>>>(r.wsum, nwin, r.wbase);
  k_csr_offsets<<<grid_for(r.C + 1LL), kLayoutBlock, 0, st>>>(r.C, r.win_off, r.wbase, nwin,
                                                              r.off);
  if (r.Fi > 0) {
    k_rcm_scatter<<<grid_for(r.Fi), kLayoutBlock, 0, st>>>(r);
    k_rcm_sort<<<grid_for(r.C), kLayoutBlock, 0, st>>>(r);
  }
  k_rcm_isolated<<<grid_for(r.C), kLayoutBlock, 0, st>>>(r);
  k_window_scan<<<nwin, kWinBlock, 0, st>>>(m, r.cnt, r.cnt, r.win_off, r.wsum, r.info);
  k_window_base<<<1, kWinBlock, 0, st>>>(r.wsum, nwin, r.wbase);
  k_rcm_place_isolated<<<grid_for(r.C), kLayoutBlock, 0, st>>>(r);
}

void launch_rcm_start(const RcmDev& r, int q, cudaStream_t st) {
  k_rcm_start<<<grid_for(r.C), kLayoutBlock, 0, st>>>(r);
  k_rcm_place_start<<<1, 1, 0, st>>>(r, q);
}

void launch_rcm_level(const RcmDev& r, int lo, int hi, cudaStream_t st) {
  const int n = hi - lo, nwin = (n + kFaceWindow - 1) / kFaceWindow;
  DevMesh m{};
  m.C = n;
  k_rcm_claim<<<grid_for(n), kLayoutBlock, 0, st>>>(r, lo, hi);
  k_rcm_count<<<grid_for(n), kLayoutBlock, 0, st>>>(r, lo, hi);
  k_window_scan<<<nwin, kWinBlock, 0, st>>>(m, r.cnt, r.cnt, r.win_off, r.wsum, r.info);
  k_window_base<<<1, kWinBlock, 0, st>>>(r.wsum, nwin, r.wbase);
  k_rcm_emit<<<grid_for(n), kLayoutBlock, 0, st>>>(r, lo, hi);
}

}  // namespace plfbs
