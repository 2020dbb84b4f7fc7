// Internals shared by the C-ABI translation units (capi.cpp: context
// lifetime, time step, state and checkpoints; capi_layout.cpp: the device
// layout builders and the polyMesh geometry entry point).
#ifndef PLFBS_CAPI_INTERNAL_HPP
#define PLFBS_CAPI_INTERNAL_HPP

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <string>
#include <vector>

#include "plfbs.h"
#include "plfbs_internal.hpp"

struct plfbs_ctx {
  int device = 0;
  plfbs_config cfg{};
  plfbs::Layout L;
  int N = 0;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t step_exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  plfbs::KernelArgs args{};
  std::vector<void*> allocs;
  int64_t bytes = 0;
  plfbs::DevStats* stats_host = nullptr;  // pinned copy of the stats header
  long long stages_done = 0;       // stages run through plfbs_run_stages in the current step
  bool debug = false;
  bool have_state = false;
  int* wall_buf = nullptr;   // device wall list of plfbs_wall_forces (grown on demand)
  int wall_cap = 0;
  uint64_t fingerprint = 0;  // of the caller's mesh, checked when a checkpoint is loaded
  int32_t* face_order = nullptr;  // device [F]: caller face of each device face
  int32_t* perm = nullptr;        // device [C + B]: device index of each caller cell / ghost
  plfbs::FluxMaps flux_maps{};    // tensor maps of the TMA-staged flux kernel (FP64)
  int compact_faces = 0;          // unique face records in the compact layout (0: none)
  int compact_cells = 0;          // unique cell weight sets in the compact layout (0: none)
  bool flux_maps_ok = false;
  // The caller's mesh arrays, copied to the device at the start of
  // plfbs_create, checked there (launch_mesh_scan) and read by the layout
  // only after the checks passed: owner, neighbour [F] int; area, sdt [F],
  // normal, fcen [3F], vol [C], ccen [3(C+B)] double; the stencil offsets
  // [C+1], cells and faces [nnz] int (with `stencil` set). Freed once the
  // layout is built.
  // Host-built layout arrays copied to the device from a page-locked staging
  // buffer while plfbs_create waits for the mesh copies (prestage_layout):
  // the caller-to-device cell map [C], the boundary orders [B] (int32) and
  // the boundary records [B] (FP64 double4, FP32 float4); null where they go
  // up later from pageable memory instead.
  struct Prestaged {
    const void* cell_new = nullptr;
    const void* bc_new = nullptr;
    const void* bc_old = nullptr;
    const void* bc[4] = {nullptr, nullptr, nullptr, nullptr};
  } pre;
  void* staging = nullptr;  // the page-locked buffer, held until plfbs_create ends
  size_t staging_bytes = 0;
  struct MeshStage {
    bool ok = false, stencil = false;
    const int32_t* owner = nullptr;
    const int32_t* neighbour = nullptr;
    const double *area = nullptr, *normal = nullptr, *fcen = nullptr, *sdt = nullptr,
                 *vol = nullptr, *ccen = nullptr;
    const int32_t *st_off = nullptr, *st_cells = nullptr, *st_faces = nullptr;
    long long nnz = 0;
    int C = 0, F = 0, Fi = 0;
    plfbs::MeshScan* scan = nullptr;  // device
    std::vector<void*> bufs;
  } stage;
  double timeout_s = 0;  // bound on plfbs_run's waits for its step batches (0: none)
  bool busy = false;     // a timed-out run's steps are still in flight (ev1 marks their end)
  std::string err;
};

namespace plfbs_capi {

// A named NVTX range over a scope (visible to Nsight Systems and ncu; without a
// tool attached the calls return at once).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Records `m` as the context's error (or the global one for a null context)
// and returns `code`.
int set_err(plfbs_ctx* c, int code, const std::string& m);

// The per-device stream-ordered memory pool (created on first use).
cudaMemPool_t device_pool(int device);
int pool_alloc(plfbs_ctx* ctx, void** dst, size_t n);
// A transient buffer from the same pool, on the context's stream; give it
// back with scratch_free (stream-ordered) when the work using it is enqueued.
int scratch_alloc(plfbs_ctx* ctx, void** dst, size_t n);
void scratch_free(plfbs_ctx* ctx, void* p);
int dev_alloc(plfbs_ctx* ctx, void** dst, size_t n);

// PLFBS_OK, or PLFBS_ERR_NO_DEVICE for a missing or non-sm_100 device.
int check_device(int device);

// The face, stencil and gather arrays of a context on the device, and the
// compact layout (capi_layout.cpp).
int build_device_layout(plfbs_ctx* ctx, const plfbs_mesh_view& m);
// Starts the copies of the mesh's arrays (sizes from the view's counts,
// checked positive first) into ctx->stage; returns without staging when the
// counts or pointers are not usable (the layout then uploads them).
int stage_mesh(plfbs_ctx* ctx, const plfbs_mesh_view& m);
// Launches the checks of validate_mesh on the staged arrays and the copy of
// their results into *out (page-locked host memory; valid once the stream
// has reached it). *launched false: nothing staged to check, the host scans
// instead.
int scan_mesh(plfbs_ctx* ctx, plfbs::MeshScan* out, bool* launched);
// Copies the host-built layout arrays to the device through page-locked
// staging (ctx->pre); leaves ctx->pre empty when they are not all built yet
// or no staging buffer can be had. Returns the staging buffer with
// release_staging once the stream has passed the copies.
int prestage_layout(plfbs_ctx* ctx);
void release_staging(plfbs_ctx* ctx);
void free_stage(plfbs_ctx* ctx);
int build_compact_layout(plfbs_ctx* ctx);

// The renumber-1 cell order (reverse Cuthill-McKee, order[new] = caller cell)
// built on the device (renumber 2; capi_layout.cpp).
int device_cell_order(plfbs_ctx* ctx, const plfbs_mesh_view& m, std::vector<int32_t>& order);

}  // namespace plfbs_capi

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return plfbs_capi::set_err(ctx, PLFBS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TRY(x)                \
  do {                        \
    int r_ = (x);             \
    if (r_ != PLFBS_OK) return r_; \
  } while (0)

namespace plfbs_capi {

// Pageable-source copies: cudaMemcpyAsync returns once `src` has been staged,
// so the caller may release it afterwards.
template <typename T>
int dev_upload(plfbs_ctx* ctx, void** dst, const std::vector<T>& src) {
  const size_t n = std::max<size_t>(src.size(), 1) * sizeof(T);
  int rc = pool_alloc(ctx, dst, n);
  if (rc) return rc;
  if (!src.empty())
    CK(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice,
                       ctx->stream));
  return PLFBS_OK;
}

}  // namespace plfbs_capi

#endif  // PLFBS_CAPI_INTERNAL_HPP
