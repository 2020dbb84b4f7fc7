// Internal declarations shared by the host setup (setup.cpp), the C ABI
// (capi.cpp) and the kernels (kernels.cu). Not part of the public ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <functional>
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
// Host-side part of a context's layout: sizes, the permutations between the
// caller's numbering and the device's, and the boundary records (built on
// the host; the face, stencil and gather arrays are built on the device).
struct Layout {
  int C = 0, F = 0, Fi = 0, B = 0;
  int K = 0;      // gradient-stencil slots per cell (max stencil size)
  int K2 = 0;     // face slots per cell in the gather (max faces per cell)
  int quirk_b = -1;  // new bc index of the caller's first ghost (index C), see kernels.cu

  std::vector<int32_t> cell_new_of_old, cell_old_of_new;  // [C]
  std::vector<int32_t> bc_new_of_old, bc_old_of_new;      // [B]

  // Boundary records, 4 x 4 doubles per boundary face (structure of arrays):
  //   bc0 = raw boundary value (u, v, w, rho)
  //   bc1 = ghost Dirichlet target (u or parabolic u_target, v, w, rho)
  //   bc2 = (d.x, d.y, d.z, |d|) unit owner->ghost direction and distance
  //   bc3 = (1-|n.x|, 1-|n.y|, 1-|n.z|, types) types = rho_type | vel_type << 8
  std::vector<double> bc0, bc1, bc2, bc3;  // [4B] each
};

// Device layout (layout.cu), per context:
//   face0 = (n.x, n.y, n.z, area)                 [F] double4 (FP32 form: float4)
//   face1 = (streaming dt, t1.x, t1.y, t1.z)      t1 = owner centroid - face centroid
//   face2 = (t2.x, t2.y, t2.z, tau)               t2 = neighbour centroid - face centroid,
//                                                 tau = 3 nu / (dt_s gamma)
//   face_ids = (new owner, new neighbour or C + new bc)   [F] int2
//   st_nbr, st_wx, st_wy, st_wz: gradient stencil, slot k of cell i at k*C + i,
//     neighbour -1 in empty slots, weights the precombined LHS^-1 . RHS_e
//   gather: (face << 1) | (cell is the neighbour), slot-major [K2*C], -1 empty
//   inv_volume [C]
// Faces: internal ones by (owner window of kFaceWindow new cells, upwind
// signature, new owner, new neighbour, caller face), then boundary faces by
// new boundary index. Within a window, faces of one signature take the same
// branches in the flux kernel and the window keeps the cells they read
// resident in L2 across the signature classes.
constexpr int kFaceWindow = 4096;

// The caller's mesh arrays copied to the device, plus the renumbering.
struct DevMesh {
  int C, F, Fi, B;
  const int32_t* owner;      // [F]
  const int32_t* neighbour;  // [F]
  const double* area;        // [F]
  const double* normal;      // [3F]
  const double* fcen;        // [3F]
  const double* sdt;         // [F]
  const double* vol;         // [C]
  const double* ccen;        // [3(C+B)]
  const int32_t* st_off;     // [C+1]
  const int32_t* st_cells;   // [nnz]
  const int32_t* st_faces;   // [nnz]
  const int32_t* cell_new;   // [C] caller cell -> new
  const int32_t* bc_new;     // [B] caller boundary face -> new
  const int32_t* bc_old;     // [B] new boundary face -> caller
};

// Device scratch of the layout build, zeroed before use except seg and sig.
struct LayoutScratch {
  int32_t* own_cnt;   // [C] internal faces per new owner
  int32_t* own_off;   // [C] offset of an owner's faces within its window
  int32_t* cursor;    // [C]
  int32_t* deg;       // [C] faces per new cell
  int32_t* gcnt;      // [C]
  int32_t* wsum;      // [windows]
  int32_t* wbase;     // [windows + 1]
  int32_t* seg;       // [Fi] internal faces grouped by owner
  uint16_t* sig;      // [Fi]
  int32_t* info;      // [0] first cell with a singular LS matrix (C if none), [1] max faces per cell
  unsigned long long* fingerprint;
};

// Internal face order (face_order[k] = caller face; boundary entries are
// filled by launch_layout_records), the gather width and the fingerprint.
void launch_layout_order(const DevMesh& m, const LayoutScratch& s, int32_t* face_order,
                         cudaStream_t stream);
// Face records, ids, stencil weights and inverse volumes.
void launch_layout_records(const DevMesh& m, const LayoutScratch& s, int precision, int mode,
                           double visc3, double pg, int32_t* face_order, int32_t* face_ids,
                           void* face0, void* face1, void* face2, int32_t* st_nbr, void* st_wx,
                           void* st_wy, void* st_wz, void* inv_volume, cudaStream_t stream);
// The face-to-cell gather (pre-filled with -1).
void launch_layout_gather(const DevMesh& m, const LayoutScratch& s, const int32_t* face_ids,
                          int32_t* gather, cudaStream_t stream);

// A polyMesh on the device: single-precision points, faces as vertex lists.
struct DevPolyMesh {
  int P, F, Fi, C;
  const float* points;        // [3P]
  const int32_t* face_offsets;  // [F+1]
  const int32_t* face_points;   // [face_offsets[F]]
  const int32_t* owner;       // [F]
  const int32_t* neighbour;   // [Fi]
};
// Device outputs of the geometry build (plfbs_mesh_view's arrays; owner and
// neighbour are the caller's).
struct GeometryOut {
  double* area;      // [F]
  double* normal;    // [3F]
  double* fcen;      // [3F]
  double* sdt;       // [F]
  double* vol;       // [C+B]
  double* ccen;      // [3(C+B)]
  int32_t* st_off;   // [C+1]
  int32_t* st_cells; // [2Fi + B]
  int32_t* st_faces; // [2Fi + B]
};
struct GeometryScratch {
  double* fcsum;     // [3F] un-normalised face centroid sums
  int32_t* cnt;      // [C] faces per cell (zeroed)
  int32_t* cursor;   // [C] (zeroed)
  int32_t* own_off;  // [C]
  int32_t* wsum;     // [windows]
  int32_t* wbase;    // [windows + 1]
  int32_t* info;     // [2] (zeroed)
};
void launch_polymesh_geometry(const DevPolyMesh& pm, double ref_dt, const GeometryOut& o,
                              const GeometryScratch& s, cudaStream_t stream);
// Host checks of a polyMesh's indices (setup.cpp).
int validate_polymesh(const plfbs_polymesh_view& pm, std::string& err);

// Exact deduplication of per-item records for the compact layout
// (layout.cu): kind 0, face records (three 4-vector arrays [n]); kind 1, a
// cell's K precombined weight triples (three slot-major arrays [K][n]);
// elements FP64, or FP32 with fp32 = 1 (the deviation form's layout).
struct RecordSource {
  int kind, n, K, fp32;
  const void* p0;
  const void* p1;
  const void* p2;
};
struct DedupeScratch {
  int P;                          // hash slots, a power of two >= 2n
  unsigned long long* slot_hash;  // [P] zeroed
  int32_t* slot_rep;              // [P] filled with 0x7f7f7f7f
  int32_t* item_slot;             // [n]
  int32_t* rep_of;                // [n]
  int32_t* is_rep;                // [n]
  int32_t* off;                   // [n]
  int32_t* wsum;                  // [windows]
  int32_t* wbase;                 // [windows + 1]: wbase[windows] = number of unique records
  int32_t* info;                  // [4] zeroed: [0] probe overflow
};
// Claim, resolve and number the unique records (wbase[windows] = their count).
void launch_dedupe_scan(const RecordSource& r, const DedupeScratch& d, cudaStream_t stream);
// Per-item table index and the unique records into the table.
void launch_dedupe_emit(const RecordSource& r, const DedupeScratch& d, int32_t* index, void* t0,
                        void* t1, void* t2, cudaStream_t stream);

// The Cuthill-McKee order built on the device by breadth-first levels
// (renumber 2, rcm_levels.hpp): the order setup.cpp's rcm_order computes,
// before its reversal.
struct RcmDev {
  int C, Fi;
  const int32_t* owner;          // [Fi] caller internal faces
  const int32_t* neighbour;      // [Fi]
  int32_t* deg;                  // [C] zeroed: internal faces per cell
  int32_t* cursor;               // [C] zeroed
  int32_t* cnt;                  // [C] flags, then children per frontier position
  int32_t* win_off;              // [C] offsets within a window of kFaceWindow
  int32_t* wsum;                 // [windows of C]
  int32_t* wbase;                // [windows of C + 1]: wbase[windows] = the scan's total
  int32_t* off;                  // [C + 1] adjacency offsets
  unsigned long long* adj_key;   // [2 Fi] (face << 32) | neighbour, sorted per cell
  int32_t* adj;                  // [2 Fi] neighbours in face order
  int32_t* pos;                  // [C] filled with -1: position in the order
  unsigned long long* key;       // [C] filled with ~0: claim keys
  int32_t* order;                // [C] zeroed
  unsigned long long* start;     // [1]
  int32_t* info;                 // [4] zeroed: [1] window-scan scratch, [2] refused placements
};
// Degrees, face-ordered adjacency, and the cells without internal faces at
// the front of the order by index (their count at wbase[windows of C]).
void launch_rcm_graph(const RcmDev& r, cudaStream_t stream);
// The next component's start (smallest (degree, cell) unvisited) at order[q].
void launch_rcm_start(const RcmDev& r, int q, cudaStream_t stream);
// The level after order[lo, hi) at order[hi ..]; its size at
// wbase[windows of (hi - lo)].
void launch_rcm_level(const RcmDev& r, int lo, int hi, cudaStream_t stream);

// FP32 boundary records for the deviation form (PLFBS_FP32_DEVIATION):
// rounded once from the FP64 records, values as deviations (rho - rho0,
// velocity / U).
struct BoundaryRecords32 {
  std::vector<float> bc0, bc1, bc2, bc3;         // [4B]
};
void boundary_records32(const Layout& L, double rho0, double uref, BoundaryRecords32& o);

// The checks of a caller's mesh arrays that everything indexing with them
// relies on (setup.cpp); *K_out (may be null) receives the largest stencil.
// First failing index of each mesh check (the count where none fails) and the
// largest stencil, found on the device by launch_mesh_scan; validate_mesh
// takes them in place of its own scans.
struct MeshScan {
  int bad_face;     // face checks: owner / neighbour ranges, area, dt, normal
  int bad_volume;   // cell volume positive and finite
  int bad_offset;   // stencil_offsets[i + 1] < stencil_offsets[i]
  int bad_stencil;  // a cell with a stencil entry out of range or not a face neighbour
  int kmax;         // largest stencil
};
int validate_mesh(const plfbs_mesh_view& m, std::string& err, int* K_out,
                  const MeshScan* scan = nullptr);
// the checks of validate_mesh over the copies of the mesh arrays on the
// device, into *out (device memory) on stream s
void launch_mesh_scan(const int32_t* owner, const int32_t* nb, const double* area,
                      const double* sdt, const double* normal, const double* vol,
                      const int32_t* off, const int32_t* cells, const int32_t* faces, int C, int F,
                      int Fi, long long nnz, MeshScan* out, cudaStream_t s);

// Least-squares weights exactly as gradients::pre_fill_LHS_and_RHS_matrix
// (gradients.cpp:214-313): lhs_inv [9C], rhs [3 nnz], caller numbering. The
// mesh must have passed validate_mesh.
int ls_weights(const plfbs_mesh_view& m, int mode, double* lhs_inv, double* rhs,
               std::string& err);

// The error string plfbs_last_error(NULL) returns (capi.cpp).
void set_global_error(const std::string& m);

// The cell order (order[new] = caller cell): identity, or RCM for renumber 1
// and 2 (setup.cpp; renumber 2 is the same order built on the device).
std::vector<int32_t> cell_order(int C, int Fi, const int32_t* owner, const int32_t* nb,
                                int renumber);

// Validate the views, renumber the cells, order the boundary faces and build
// their records (setup.cpp). For renumber 2 it stops after the validation:
// the caller builds the order on the device and calls order_layout.
// With `scan`, the mesh checks' results found on the device; with
// `wait_scan` (renumber 0 and 2), they are still being found: the host work
// that is safe on unchecked arrays runs first, then wait_scan blocks for them.
int prepare_layout(const plfbs_config& cfg, const plfbs_mesh_view& m, const plfbs_bc_view& bc,
                   Layout& L, std::string& err, const MeshScan* scan = nullptr,
                   const std::function<int(MeshScan&)>& wait_scan = nullptr);

// The order-dependent part of prepare_layout for a given cell order (a
// permutation of the cells): boundary face order and records.
int order_layout(const plfbs_config& cfg, const plfbs_mesh_view& m, const plfbs_bc_view& bc,
                 std::vector<int32_t> order, Layout& L, std::string& err);

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
  int fault;                   // a kernel's bounded wait ran out (the step is invalid)
  long long steps;             // completed time steps
  long long converged_step;
  double last[6];              // t, max_error, rho, u, v, w rms of the last step
  alignas(128) double history[kHistoryCap][6];
};

// Tensor maps of the FP64 state and gradient rows for the TMA-staged flux
// kernel (k_flux_tma): 2D, one cell per row, boxes one row high.
struct FluxMaps {
  CUtensorMap state;  // [C rows][4 doubles]
  CUtensorMap grad;   // [C rows][12 doubles]
};

struct KernelArgs {
  // sizes
  int C, F, Fi, B, K, K2, quirk_b, N, nblk_update;
  int flavour;  // PLFBS_FLAVOUR_*: whose reconstruction and boundary tables
  int ibm_xc, ibm_yc;
  // scalars
  double dt;            // RK time step
  double pg;            // 1 / gamma
  // equilibrium constants of the flux kernel per weight class (centre 2/9,
  // axis 1/9, diagonal 1/72): (w, 3 w, 4.5 w / gamma, 1.5 w / gamma)
  double eq[3][4];
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
  const int32_t* ibm_order;  // [N] nodes in spatial order (by the cell of node_ref)
  double* partial;      // [nblk_update * 4] per-block squared-residual sums
  DevStats* stats;
  void* res_debug;      // double4 [C] (FP32 form: float4) or null
  // FP32 deviation form only
  const int32_t* face_ids;                     // int2 [F]
  float* fforce_x; float* fforce_y; float* fforce_z;  // [C] body force / U, or null
  float rho0f, inv_uref_f;
  // host side: tensor maps of the TMA-staged FP64 flux kernel, or null for
  // the per-thread gathers (read by launch_flux, not by kernels)
  const FluxMaps* flux_maps;
  // compact layout: bitwise-equal face records and cell weight sets
  // stored once (null where the mesh's records do not repeat)
  const int32_t* face_rec;                        // [F] index into frec0/1/2
  const void* frec0; const void* frec1; const void* frec2;  // double4 (FP32: float4) [unique]
  const int32_t* cell_wset;                       // [C] index into wtab
  const void* wtab;                               // [unique sets][K][3] double (FP32: float)
  const int32_t* frec_sides;                      // [unique records] branch bits (FP64)
  const double* frec_relax;                       // [2 x unique records] (1 - tau) A, tau A (FP64)
  int compact;                                    // 1: the kernels read the tables
};

// Launchers (kernels.cu; the FP32 deviation form in kernels_fp32.cu). All
// enqueue on `stream`, never synchronise.
void launch_ibm(const KernelArgs& a, int precision, cudaStream_t stream);
void launch_gradient(const KernelArgs& a, int precision, cudaStream_t stream);
void launch_flux(const KernelArgs& a, int precision, cudaStream_t stream);
// Sets the TMA-staged flux kernel's shared-memory size on the current device
// (once) and returns its resident block count; call before capturing it.
int prepare_flux_tma();
// RK stage rk's update; the last stage (rk 3) ends with the residual reduction
// (k_finish) unless `finish` is false (launch_finish runs it alone).
void launch_update(const KernelArgs& a, int precision, int rk, cudaStream_t stream,
                   bool finish = true);
void launch_finish(const KernelArgs& a, int precision, cudaStream_t stream);
void launch_seed(const KernelArgs& a, int precision, bool conserved, cudaStream_t stream);
void launch_wall_forces(const KernelArgs& a, int precision, const int* walls, int n,
                        double visc_gamma, double gamma, double* out, cudaStream_t stream);
void launch_ibm32(const KernelArgs& a, cudaStream_t stream);
// Branch bits (the flux kernel's seven lattice-pair sides) of n unique FP64
// face records of the compact layout, and their relaxation pairs
// relax[2r] = (1 - tau) A, relax[2r + 1] = tau A.
void launch_record_sides(const void* frec0, const void* frec1, const void* frec2, int n,
                         int flavour, int32_t* out, double* relax, cudaStream_t stream);
void launch_gradient32(const KernelArgs& a, cudaStream_t stream);
void launch_flux32(const KernelArgs& a, cudaStream_t stream);
void launch_update32(const KernelArgs& a, int rk, cudaStream_t stream, bool finish = true);
void launch_finish32(const KernelArgs& a, cudaStream_t stream);

// State transfer on the device (state_io.cu). perm[o] is the device index of
// caller index o (cells, then one ghost per boundary face), T = C + B.
// state_in: the caller's four FP64 field arrays (device copies) into the state
// records (FP32 form: deviation units, velocity / U and rho - r0); state_out
// the reverse; records: n records of rec_bytes (16 or 32) gathered into the
// caller's order (to_caller) or scattered from it.
void launch_state_in(const int32_t* perm, long long T, const double* rho, const double* u,
                     const double* v, const double* w, int precision, double U, double r0,
                     void* state, cudaStream_t stream);
void launch_state_out(const int32_t* perm, long long T, const void* state, int precision,
                      double U, double r0, double* rho, double* u, double* v, double* w,
                      cudaStream_t stream);
void launch_records(const int32_t* perm, long long n, int rec_bytes, const void* src, void* dst,
                    bool to_caller, cudaStream_t stream);
// perm[C + B]: the device index of each caller cell (cell_new) and ghost (C + bc_new)
void launch_perm(const int32_t* cell_new, const int32_t* bc_new, int C, int B, int32_t* perm,
                 cudaStream_t stream);
// p[0, n) = value
void launch_fill(double* p, long long n, double value, cudaStream_t stream);
void launch_fill(float* p, long long n, float value, cudaStream_t stream);
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
