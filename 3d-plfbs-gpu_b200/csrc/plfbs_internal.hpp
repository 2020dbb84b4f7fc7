// Internal declarations shared by the host setup (setup.cpp), the C ABI
// (capi.cpp) and the kernels (kernels.cu). Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "plfbs.h"

namespace plfbs {

// ---------------------------------------------------------------------------
// Host layout: every array the device needs, in the solver's own numbering.
//
// Cells are renumbered (RCM when requested) and faces reordered: internal
// faces sorted by (owner, neighbour) in the new numbering, then boundary faces
// sorted by owner. Ghost cell C + b belongs to the b-th boundary face of the
// new order. The permutations map both ways so that every public entry point
// reads and writes the caller's numbering.
// ---------------------------------------------------------------------------
struct Layout {
  int C = 0, F = 0, Fi = 0, B = 0;
  int K = 0;      // gradient-stencil slots per cell (max stencil size)
  int K2 = 0;     // face slots per cell in the gather (max faces per cell)
  int quirk_b = -1;  // new bc index of the caller's first ghost (index C), see kernels.cu

  std::vector<int32_t> cell_new_of_old, cell_old_of_new;  // [C]
  std::vector<int32_t> bc_new_of_old, bc_old_of_new;      // [B]
  std::vector<int32_t> face_new_of_old, face_old_of_new;  // [F]

  // Face records, 3 x 4 doubles per face (structure of arrays):
  //   face0 = (n.x, n.y, n.z, area)
  //   face1 = (streaming dt, t1.x, t1.y, t1.z)   t1 = owner centroid - face centroid
  //   face2 = (t2.x, t2.y, t2.z, tau)            t2 = neighbour centroid - face centroid,
  //                                              tau = 3 nu / (dt_s gamma)
  std::vector<double> face0, face1, face2;  // [4F] each
  std::vector<int32_t> face_ids;            // [2F] new owner, new neighbour (or C + bc)

  // Boundary records, 4 x 4 doubles per boundary face (structure of arrays):
  //   bc0 = raw boundary value (u, v, w, rho)
  //   bc1 = ghost Dirichlet target (u or parabolic u_target, v, w, rho)
  //   bc2 = (d.x, d.y, d.z, |d|) unit owner->ghost direction and distance
  //   bc3 = (1-|n.x|, 1-|n.y|, 1-|n.z|, types) types = rho_type | vel_type << 8
  std::vector<double> bc0, bc1, bc2, bc3;  // [4B] each

  // Gradient stencil in slot-major (ELL) layout: slot k of cell i at k*C + i.
  // Neighbour -1 marks an empty slot. Weights are the precombined
  // LHS^-1 . RHS_e (three arrays, x/y/z).
  std::vector<int32_t> st_nbr;                 // [K*C]
  std::vector<double> st_wx, st_wy, st_wz;     // [K*C]

  // Face-to-cell gather, slot-major: (face << 1) | (cell is the neighbour), -1 empty.
  std::vector<int32_t> gather;                 // [K2*C]
  std::vector<double> inv_volume;              // [C]

  // Cell centroids in the new numbering, kept for host-side diagnostics.
  std::vector<double> centroid;                // [3(C+B)]
};

// FP32 copies of the layout for the deviation form (PLFBS_FP32_DEVIATION):
// geometry and weights rounded once from the FP64 records (weights are built
// in FP64 first), boundary values expressed as deviations (rho - rho0,
// velocity / U), face ids moved to their own int2 array.
struct Layout32 {
  std::vector<float> face0, face1, face2;        // [4F] (n, A), (dt_s, t1), (t2, tau)
  std::vector<float> bc0, bc1, bc2, bc3;         // [4B]
  std::vector<float> st_wx, st_wy, st_wz;        // [K*C]
  std::vector<float> inv_volume;                 // [C]
};
void build_layout32(const Layout& L, double rho0, double uref, Layout32& L32);

// Least-squares weights exactly as gradients::pre_fill_LHS_and_RHS_matrix
// (gradients.cpp:214-313): lhs_inv [9C], rhs [3 nnz], caller numbering.
int ls_weights(const plfbs_mesh_view& m, int mode, double* lhs_inv, double* rhs,
               std::string& err);

// The error string plfbs_last_error(NULL) returns (capi.cpp).
void set_global_error(const std::string& m);

// Validate the views and build the device layout.
int build_layout(const plfbs_config& cfg, const plfbs_mesh_view& m, const plfbs_bc_view& bc,
                 Layout& L, std::string& err);

// ---------------------------------------------------------------------------
// Device side
// ---------------------------------------------------------------------------

constexpr int kHistoryCap = 4096;   // per-step residual records kept on the device
constexpr int kBlock = 256;         // threads per block of the cell kernels
constexpr int kFluxBlock = 128;     // threads per block of the face-flux kernel (128 registers, 4 blocks/SM)
constexpr int kFinishBlock = 1024;  // the one block that reduces the per-block residual sums
constexpr int kIbmBlock = 256;      // IBM kernel: 32 nodes x 8 stencil cells per block
constexpr int kMaxDevices = 64;     // per-device caches of launch shapes

// Run status shared by all kernels of a step, in device memory. The halt flag
// is read by every block of every kernel; k_finish writes it once per step.
struct DevStats {
  int halt;                    // 1 once converged or diverged: kernels return at entry
  int converged;
  int diverged;
  int pad0;
  long long steps;             // completed time steps
  long long converged_step;
  double last[6];              // t, max_error, rho, u, v, w rms of the last step
  alignas(128) double history[kHistoryCap][6];
};

struct KernelArgs {
  // sizes
  int C, F, B, K, K2, quirk_b, N, nblk_update;
  int ibm_xc, ibm_yc;
  // scalars
  double dt;            // RK time step
  double pg;            // 1 / gamma
  double visc3;         // 3 nu (relaxation factor is 3 nu / (dt_s gamma))
  double pressure_gradient;
  double tolerance;
  double inv_ref_rho, inv_ref_mom;
  double ibm_dx, ibm_inv_dx3, ibm_area_k;   // spacing, 1/dx^3, stiffness * node area
  double origin[3];
  // FP32 deviation form
  double rho0, uref;
  // arrays (FP64 path)
  void* state;          // double4 [C+B]
  void* t0;             // double4 [C]
  void* t1;             // double4 [C]
  void* grad;           // 3 x double4 per cell [3C]
  void* flux;           // double4 [F]
  const void* face0; const void* face1; const void* face2;  // double4 [F]
  const void* bc0; const void* bc1; const void* bc2; const void* bc3;  // double4 [B]
  const int32_t* st_nbr;
  const void* st_wx; const void* st_wy; const void* st_wz;
  const int32_t* gather;
  const void* inv_volume;
  double* force_x; double* force_y; double* force_z;  // [C] or null without IBM
  double* node_x; double* node_x0; const double* node_ref; double* node_vel;
  double* node_force;   // [3N] interleaved
  const int32_t* ibm_map;  // caller cell index -> new cell index
  double* partial;      // [nblk_update * 4] per-block squared-residual sums
  DevStats* stats;
  void* res_debug;      // double4 [C] (FP32 form: float4) or null
  // FP32 deviation form only
  const int32_t* face_ids;                     // int2 [F]
  float* fforce_x; float* fforce_y; float* fforce_z;  // [C] body force / U, or null
  float rho0f, inv_uref_f;
};

// Launchers (kernels.cu; the FP32 deviation form in kernels_fp32.cu). All
// enqueue on `stream`, never synchronise.
void launch_ibm(const KernelArgs& a, int precision, cudaStream_t stream);
void launch_gradient(const KernelArgs& a, int precision, cudaStream_t stream);
void launch_flux(const KernelArgs& a, int precision, cudaStream_t stream);
void launch_update(const KernelArgs& a, int precision, int rk, cudaStream_t stream);
void launch_seed(const KernelArgs& a, int precision, bool conserved, cudaStream_t stream);
void launch_wall_forces(const KernelArgs& a, int precision, const int* walls, int n,
                        double visc_gamma, double gamma, double* out, cudaStream_t stream);
void launch_ibm32(const KernelArgs& a, cudaStream_t stream);
void launch_gradient32(const KernelArgs& a, cudaStream_t stream);
void launch_flux32(const KernelArgs& a, cudaStream_t stream);
void launch_update32(const KernelArgs& a, int rk, cudaStream_t stream);
void launch_seed32(const KernelArgs& a, bool conserved, cudaStream_t stream);

#ifdef __CUDACC__
// Blocks of a grid-stride kernel: as many as are resident on the device at
// once (occupancy x SMs, cached per device), at most one per `block` items.
template <typename Kernel>
int persistent_blocks(Kernel kernel, int block, long long n, std::atomic<int>* cache) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = 0;
  int r = cache[dev].load(std::memory_order_relaxed);
  if (r <= 0) {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        per_sm <= 0 || sms <= 0) {
      per_sm = 1;
      sms = 148;
    }
    r = per_sm * sms;
    cache[dev].store(r, std::memory_order_relaxed);
  }
  const long long need = (n + block - 1) / block;
  return (int)(need < r ? (need > 0 ? need : 1) : r);
}
#endif

}  // namespace plfbs
