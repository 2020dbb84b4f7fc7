// The extern "C" entry points of include/plfbs.h: context lifetime, device
// memory, the CUDA-graph time step and the host loop around it.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <limits>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "capi_internal.hpp"

using plfbs::DevStats;
using plfbs::KernelArgs;
using plfbs::Layout;


namespace {

thread_local std::string g_err;  // errors without a context, per calling thread

const char* kVersion = "plfbs-b200 0.1 (sm_100a)";



// Device memory comes from one stream-ordered pool per device whose release
// threshold is unbounded: plfbs_destroy returns a context's arrays to the pool
// (no unmapping, which cost up to 0.8 s in a process's first frees) and the
// next plfbs_create on that device reuses them. plfbs_release_cached trims it.
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[plfbs::kMaxDevices] = {};


// Pinned host copies of the run status, recycled across contexts: freeing
// pinned memory can stall for a long time on a busy host, so plfbs_destroy
// returns the buffer here and only plfbs_release_cached frees them.
std::vector<DevStats*> g_pinned_stats;

// Page-locked staging buffers for the host-built layout arrays of
// plfbs_create, recycled the same way (size in bytes beside each).
std::vector<std::pair<void*, size_t>> g_pinned_staging;

}  // namespace

namespace plfbs_capi {

int set_err(plfbs_ctx* c, int code, const std::string& m) {
  if (c)
    c->err = m;
  else
    g_err = m;
  return code;
}

cudaMemPool_t device_pool(int device) {
  std::lock_guard<std::mutex> g(g_pool_mutex);
  if (device < 0 || device >= plfbs::kMaxDevices) return nullptr;
  if (!g_pools[device]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&g_pools[device], &props) != cudaSuccess) return g_pools[device] = nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(g_pools[device], cudaMemPoolAttrReleaseThreshold, &keep);
  }
  return g_pools[device];
}

int pool_alloc(plfbs_ctx* ctx, void** dst, size_t n) {
  cudaMemPool_t pool = device_pool(ctx->device);
  if (!pool) return set_err(ctx, PLFBS_ERR_CUDA, "device memory pool creation failed");
  CK(cudaMallocFromPoolAsync(dst, n, pool, ctx->stream));
  ctx->allocs.push_back(*dst);
  ctx->bytes += (int64_t)n;
  return PLFBS_OK;
}

int scratch_alloc(plfbs_ctx* ctx, void** dst, size_t n) {
  cudaMemPool_t pool = device_pool(ctx->device);
  if (!pool) return set_err(ctx, PLFBS_ERR_CUDA, "device memory pool creation failed");
  CK(cudaMallocFromPoolAsync(dst, std::max<size_t>(n, 16), pool, ctx->stream));
  return PLFBS_OK;
}

void scratch_free(plfbs_ctx* ctx, void* p) {
  if (p) cudaFreeAsync(p, ctx->stream);
}

int dev_alloc(plfbs_ctx* ctx, void** dst, size_t n) {
  n = std::max<size_t>(n, 16);
  int rc = pool_alloc(ctx, dst, n);
  if (rc) return rc;
  CK(cudaMemsetAsync(*dst, 0, n, ctx->stream));
  return PLFBS_OK;
}

int check_device(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0)
    return set_err(nullptr, PLFBS_ERR_NO_DEVICE, "no CUDA device with that index");
  // one attribute (cudaGetDeviceProperties fills every field and can be slow)
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
      major != 10)
    return set_err(nullptr, PLFBS_ERR_NO_DEVICE,
                   "this library is built for sm_100a (B200); device major != 10");
  return PLFBS_OK;
}

}  // namespace plfbs_capi

using namespace plfbs_capi;

namespace {

DevStats* take_pinned_stats() {
  {
    std::lock_guard<std::mutex> g(g_pool_mutex);
    if (!g_pinned_stats.empty()) {
      DevStats* p = g_pinned_stats.back();
      g_pinned_stats.pop_back();
      return p;
    }
  }
  void* p = nullptr;
  return cudaMallocHost(&p, sizeof(DevStats)) == cudaSuccess ? static_cast<DevStats*>(p) : nullptr;
}

void give_pinned_stats(DevStats* p) {
  std::lock_guard<std::mutex> g(g_pool_mutex);
  g_pinned_stats.push_back(p);
}

// A recycled page-locked buffer of at least `bytes` (the smallest that fits),
// else a new one rounded up to 16 MiB; null when none can be had.
void* take_pinned_staging(size_t bytes, size_t* got) {
  {
    std::lock_guard<std::mutex> g(g_pool_mutex);
    size_t best = g_pinned_staging.size();
    for (size_t k = 0; k < g_pinned_staging.size(); k++)
      if (g_pinned_staging[k].second >= bytes &&
          (best == g_pinned_staging.size() ||
           g_pinned_staging[k].second < g_pinned_staging[best].second))
        best = k;
    if (best < g_pinned_staging.size()) {
      const auto b = g_pinned_staging[best];
      g_pinned_staging.erase(g_pinned_staging.begin() + best);
      *got = b.second;
      return b.first;
    }
  }
  const size_t n = (bytes + (16u << 20) - 1) / (16u << 20) * (16u << 20);
  void* p = nullptr;
  if (cudaMallocHost(&p, n) != cudaSuccess) {
    cudaGetLastError();  // a failed page-lock leaves the pageable path, not an error
    return nullptr;
  }
  *got = n;
  return p;
}

void give_pinned_staging(void* p, size_t n) {
  std::lock_guard<std::mutex> g(g_pool_mutex);
  g_pinned_staging.emplace_back(p, n);
}





// One time step: IBM, then 4 x (gradient, flux, update) (Solver_gpu.cu:667-833).
void enqueue_step(const KernelArgs& a, int prec, cudaStream_t s) {
  plfbs::launch_ibm(a, prec, s);
  for (int rk = 0; rk < 4; rk++) {
    plfbs::launch_gradient(a, prec, s);
    plfbs::launch_flux(a, prec, s);
    plfbs::launch_update(a, prec, rk, s);
  }
}

int capture_step(plfbs_ctx* ctx) {
  if (ctx->step_exec) {
    cudaGraphExecDestroy(ctx->step_exec);
    ctx->step_exec = nullptr;
  }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  enqueue_step(ctx->args, ctx->cfg.precision, ctx->stream);
  CK(cudaStreamEndCapture(ctx->stream, &g));
  cudaError_t e = cudaGraphInstantiate(&ctx->step_exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess)
    return set_err(ctx, PLFBS_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  return PLFBS_OK;
}

int reset_force(plfbs_ctx* ctx) {
  const int C = ctx->L.C;
  const KernelArgs& a = ctx->args;
  if (a.fforce_x) {
    plfbs::launch_fill(a.fforce_x, C, (float)(ctx->cfg.pressure_gradient / ctx->cfg.max_velocity),
                       ctx->stream);
    CK(cudaMemsetAsync(a.fforce_y, 0, C * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(a.fforce_z, 0, C * sizeof(float), ctx->stream));
  } else if (a.force_x) {
    plfbs::launch_fill(a.force_x, C, ctx->cfg.pressure_gradient, ctx->stream);
    CK(cudaMemsetAsync(a.force_y, 0, C * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(a.force_z, 0, C * sizeof(double), ctx->stream));
  } else {
    return PLFBS_OK;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return PLFBS_OK;
}

int read_stats(plfbs_ctx* ctx) {
  CK(cudaMemcpyAsync(ctx->stats_host, ctx->args.stats, offsetof(DevStats, history),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PLFBS_OK;
}

// Downloads n four-component records (state-like: u, v, w, rho layout) as FP64.
// The FP32 form stores (u/U, v/U, w/U, rho - rho0): with `increments` the
// records are differences (residuals, fluxes) and only the scaling applies.
int download4(plfbs_ctx* ctx, const void* src, size_t n, std::vector<double>& out,
              bool increments) {
  out.resize(4 * n);
  if (ctx->cfg.precision == PLFBS_FP32_DEVIATION) {
    std::vector<float> f(4 * n);
    CK(cudaMemcpyAsync(f.data(), src, f.size() * sizeof(float), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double U = ctx->cfg.max_velocity, r0 = increments ? 0.0 : ctx->cfg.ref_rho;
    for (size_t i = 0; i < n; i++) {
      out[4 * i] = U * f[4 * i];
      out[4 * i + 1] = U * f[4 * i + 1];
      out[4 * i + 2] = U * f[4 * i + 2];
      out[4 * i + 3] = r0 + f[4 * i + 3];
    }
  } else {
    CK(cudaMemcpyAsync(out.data(), src, out.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return PLFBS_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// A 2D FP64 tensor map of `rows` rows of `cols` doubles (row stride cols * 8
// bytes, a multiple of 16), boxes of one row: what tile::gather4 copies.
bool encode_rows(CUtensorMap* map, const void* base, int cols, long long rows) {
  auto enc = tensor_map_encoder();
  if (!enc || rows <= 0 || (cols * 8) % 16 != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 8};
  const cuuint32_t box[2] = {(cuuint32_t)cols, 1};
  const cuuint32_t elem[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides, box,
             elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int check_fault(plfbs_ctx* ctx) {
  if (ctx->stats_host->fault)
    return set_err(ctx, PLFBS_ERR_CUDA,
                   "a kernel's bounded wait ran out (flux staging); the state is invalid");
  return PLFBS_OK;
}




// Waits at most `seconds` (none if <= 0) for the end of the launched steps
// (ev1). Running out leaves the context busy: the steps are still in flight
// and every call but plfbs_wait and plfbs_destroy returns PLFBS_ERR_TIMEOUT.
int wait_steps(plfbs_ctx* ctx, double seconds) {
  if (!(seconds > 0)) {
    CK(cudaEventSynchronize(ctx->ev1));
    ctx->busy = false;
    return PLFBS_OK;
  }
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(seconds);
  for (;;) {
    const cudaError_t e = cudaEventQuery(ctx->ev1);
    if (e == cudaSuccess) {
      ctx->busy = false;
      return PLFBS_OK;
    }
    if (e != cudaErrorNotReady) CK(e);
    if (std::chrono::steady_clock::now() >= deadline) {
      ctx->busy = true;
      return set_err(ctx, PLFBS_ERR_TIMEOUT,
                     "the launched steps did not finish within the time limit; they are still "
                     "in flight (plfbs_wait, then carry on)");
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

int check_ctx(plfbs_ctx* ctx) {
  if (!ctx) return set_err(nullptr, PLFBS_ERR_ARG, "null context");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess)
    return set_err(ctx, PLFBS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  if (ctx->busy) {  // finished since the time-out?
    e = cudaEventQuery(ctx->ev1);
    if (e == cudaSuccess)
      ctx->busy = false;
    else if (e == cudaErrorNotReady)
      return set_err(ctx, PLFBS_ERR_TIMEOUT,
                     "steps of a timed-out run are still in flight (plfbs_wait first)");
    else
      return set_err(ctx, PLFBS_ERR_CUDA, std::string("cudaEventQuery: ") + cudaGetErrorString(e));
  }
  return PLFBS_OK;
}

}  // namespace

namespace plfbs_capi {

int prestage_layout(plfbs_ctx* ctx) {
  const plfbs::Layout& L = ctx->L;
  const size_t C = (size_t)L.C, B = (size_t)L.B;
  if (C == 0 || L.cell_new_of_old.size() != C || L.bc_new_of_old.size() != B ||
      L.bc_old_of_new.size() != B || L.bc0.size() != 4 * B || L.bc1.size() != 4 * B ||
      L.bc2.size() != 4 * B || L.bc3.size() != 4 * B)
    return PLFBS_OK;  // not built yet (or not at all): the later uploads run
  const bool fp32 = ctx->cfg.precision == PLFBS_FP32_DEVIATION;
  plfbs::BoundaryRecords32 b32;
  if (fp32) plfbs::boundary_records32(L, ctx->cfg.ref_rho, ctx->cfg.max_velocity, b32);
  const void* src[7] = {L.cell_new_of_old.data(), L.bc_new_of_old.data(), L.bc_old_of_new.data(),
                        fp32 ? (const void*)b32.bc0.data() : L.bc0.data(),
                        fp32 ? (const void*)b32.bc1.data() : L.bc1.data(),
                        fp32 ? (const void*)b32.bc2.data() : L.bc2.data(),
                        fp32 ? (const void*)b32.bc3.data() : L.bc3.data()};
  const size_t rec = 4 * B * (fp32 ? sizeof(float) : sizeof(double));
  const size_t len[7] = {4 * C, 4 * B, 4 * B, rec, rec, rec, rec};
  size_t off[8] = {0};
  for (int k = 0; k < 7; k++) off[k + 1] = off[k] + (len[k] + 255) / 256 * 256;
  size_t got = 0;
  void* host = take_pinned_staging(off[7], &got);
  if (!host) return PLFBS_OK;
  ctx->staging = host;
  ctx->staging_bytes = got;
  const void* dev[7];
  for (int k = 0; k < 7; k++) {
    unsigned char* h = static_cast<unsigned char*>(host) + off[k];
    if (len[k]) std::memcpy(h, src[k], len[k]);
    void* d = nullptr;
    TRY(pool_alloc(ctx, &d, std::max<size_t>(len[k], 16)));
    if (len[k]) CK(cudaMemcpyAsync(d, h, len[k], cudaMemcpyHostToDevice, ctx->stream));
    dev[k] = d;
  }
  ctx->pre.cell_new = dev[0];
  ctx->pre.bc_new = dev[1];
  ctx->pre.bc_old = dev[2];
  for (int k = 0; k < 4; k++) ctx->pre.bc[k] = dev[3 + k];
  return PLFBS_OK;
}

void release_staging(plfbs_ctx* ctx) {
  if (!ctx->staging) return;
  give_pinned_staging(ctx->staging, ctx->staging_bytes);
  ctx->staging = nullptr;
  ctx->staging_bytes = 0;
}

}  // namespace plfbs_capi

void plfbs::set_global_error(const std::string& m) { g_err = m; }

extern "C" {

const char* plfbs_version(void) { return kVersion; }

const char* plfbs_last_error(const plfbs_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_err.c_str();
}

int plfbs_cell_order(const plfbs_mesh_view* mesh, int32_t renumber, int32_t* order) {
  if (!mesh || !order || !mesh->owner || !mesh->neighbour)
    return set_err(nullptr, PLFBS_ERR_ARG, "null argument");
  const int C = mesh->n_cells, F = mesh->n_faces, Fi = mesh->n_internal;
  if (C <= 0 || F <= 0 || Fi < 0 || Fi > F || renumber < 0 || renumber > 2)
    return set_err(nullptr, PLFBS_ERR_ARG, "cell order needs valid sizes and renumber 0, 1 or 2");
  for (int f = 0; f < Fi; f++)
    if (mesh->owner[f] < 0 || mesh->owner[f] >= C || mesh->neighbour[f] < 0 ||
        mesh->neighbour[f] >= C)
      return set_err(nullptr, PLFBS_ERR_MESH, "internal face cell out of range");
  const std::vector<int32_t> o =
      plfbs::cell_order(C, Fi, mesh->owner, mesh->neighbour, renumber);
  std::memcpy(order, o.data(), sizeof(int32_t) * (size_t)C);
  return PLFBS_OK;
}

int plfbs_ls_weights(const plfbs_mesh_view* mesh, int32_t gradient_mode, double* lhs_inv,
                     double* rhs) {
  if (!mesh || !lhs_inv || !rhs) return set_err(nullptr, PLFBS_ERR_ARG, "null argument");
  std::string err;
  int rc = plfbs::validate_mesh(*mesh, err, nullptr);  // it indexes with the caller's arrays
  if (rc == PLFBS_OK) rc = plfbs::ls_weights(*mesh, gradient_mode, lhs_inv, rhs, err);
  if (rc) g_err = err;
  return rc;
}

}  // extern "C"

extern "C" {

int plfbs_create(const plfbs_config* cfg, const plfbs_mesh_view* mesh, const plfbs_bc_view* bc,
                 const plfbs_ibm_view* ibm, int device, plfbs_ctx** out) {
  NvtxRange range("plfbs_create");
  if (!cfg || !mesh || !bc || !out) return set_err(nullptr, PLFBS_ERR_ARG, "null argument");
  *out = nullptr;
  if (cfg->precision != PLFBS_FP64 && cfg->precision != PLFBS_FP32_DEVIATION)
    return set_err(nullptr, PLFBS_ERR_ARG, "unknown precision mode");
  if (cfg->flavour != PLFBS_FLAVOUR_GPU && cfg->flavour != PLFBS_FLAVOUR_CPU_SOLVER)
    return set_err(nullptr, PLFBS_ERR_ARG, "unknown flavour");
  if (cfg->renumber < 0 || cfg->renumber > 2)
    return set_err(nullptr, PLFBS_ERR_ARG, "renumber must be 0, 1 or 2");
  if (cfg->flavour == PLFBS_FLAVOUR_CPU_SOLVER &&
      (cfg->precision != PLFBS_FP64 || (ibm && ibm->n_nodes > 0)))
    return set_err(nullptr, PLFBS_ERR_ARG,
                   "the CPU-Solver flavour is FP64 without IBM nodes (the CPU Solver has none)");
  if (!(cfg->time_marching_step > 0) || !(cfg->gamma > 0) || !(cfg->ref_rho > 0) ||
      !(cfg->max_velocity > 0) || !std::isfinite(cfg->visc))
    return set_err(nullptr, PLFBS_ERR_ARG,
                   "config needs time_marching_step, gamma, ref_rho, max_velocity > 0");
  plfbs_ctx* ctx = new (std::nothrow) plfbs_ctx();
  if (!ctx) return set_err(nullptr, PLFBS_ERR_ARG, "out of host memory");
  ctx->device = device;
  ctx->cfg = *cfg;
  std::string err;
  int rc;
  // With the device present, the mesh's arrays start on their way to it now
  // and are checked there (launch_mesh_scan: the host's checks, the same
  // first failing index and message); without it, the host threads check
  // them, and their errors are reported before the missing device.
  const bool have_device = check_device(device) == PLFBS_OK;
  auto drop = [&](int code, const std::string& m) {
    if (ctx->stream)
      plfbs_destroy(ctx);  // waits for the copies, returns the staged memory
    else
      delete ctx;  // nothing on a device
    return set_err(nullptr, code, m);
  };
  if (have_device) {
    NvtxRange r("mesh upload");
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
      return drop(PLFBS_ERR_CUDA, "cudaSetDevice / stream creation failed");
    if (stage_mesh(ctx, *mesh)) return drop(PLFBS_ERR_CUDA, ctx->err);
  }
  {
    // The mesh checks on the device when the arrays are there, their results
    // copied to page-locked memory (the stats buffer, not in use yet); the
    // host's part of the layout runs while the copies and checks proceed
    // (prepare_layout's wait_scan path), else the host threads check.
    bool scanned = false;
    plfbs::MeshScan* scan = nullptr;
    if (have_device) {
      NvtxRange r("mesh checks (device)");
      if (!(ctx->stats_host = take_pinned_stats()))
        return drop(PLFBS_ERR_CUDA, "cudaMallocHost failed");
      static_assert(sizeof(plfbs::MeshScan) <= sizeof(DevStats), "scan results fit");
      scan = reinterpret_cast<plfbs::MeshScan*>(ctx->stats_host);
      if (scan_mesh(ctx, scan, &scanned)) return drop(PLFBS_ERR_CUDA, ctx->err);
    }
    NvtxRange r("prepare_layout (host)");
    if (scanned && cfg->renumber != 1) {
      rc = plfbs::prepare_layout(*cfg, *mesh, *bc, ctx->L, err, nullptr,
                                 [&](plfbs::MeshScan& out) -> int {
                                   // the host would wait for the copies: the
                                   // arrays it has built go up behind them
                                   if (prestage_layout(ctx)) return PLFBS_ERR_CUDA;
                                   if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                                     return PLFBS_ERR_CUDA;
                                   out = *scan;
                                   return PLFBS_OK;
                                 });
    } else {
      if (scanned && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return drop(PLFBS_ERR_CUDA, "the device mesh checks failed");
      rc = plfbs::prepare_layout(*cfg, *mesh, *bc, ctx->L, err, scanned ? scan : nullptr);
    }
  }
  if (rc) return drop(rc, err);
  const Layout& L = ctx->L;
  const bool fp32 = cfg->precision == PLFBS_FP32_DEVIATION;
  const int N = (ibm && ibm->n_nodes > 0) ? ibm->n_nodes : 0;
  if (N > 0) {
    if (!ibm->x || !ibm->x_ref || ibm->object_nodes <= 0 || !(cfg->domain_dt > 0) ||
        !(cfg->lengths[0] > 0) || !(cfg->lengths[1] > 0)) {
      return drop(PLFBS_ERR_ARG,
                  "IBM needs node arrays, object_nodes > 0, domain_dt > 0 and lengths > 0");
    }
  }
  // validation needs no GPU; the device is checked before the layout is built
  if (!have_device) {
    check_device(device);  // sets the message
    const std::string m = g_err;
    return drop(PLFBS_ERR_NO_DEVICE, m);
  }
  ctx->N = N;
  auto fail = [&](int code) {
    std::string m = ctx->err;
    plfbs_destroy(ctx);
    g_err = m;
    return code;
  };
  if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess)
    return fail(set_err(ctx, PLFBS_ERR_CUDA, "event creation failed"));
  if (!ctx->stats_host && !(ctx->stats_host = take_pinned_stats()))
    return fail(set_err(ctx, PLFBS_ERR_CUDA, "cudaMallocHost failed"));
  if (cfg->renumber == 2) {  // the order on the device, then the host's order-dependent part
    NvtxRange r("device cell order");
    std::vector<int32_t> order;
    if ((rc = device_cell_order(ctx, *mesh, order))) return fail(rc);
    if ((rc = plfbs::order_layout(*cfg, *mesh, *bc, std::move(order), ctx->L, err)))
      return fail(set_err(ctx, rc, err));
  }

  KernelArgs& a = ctx->args;
  const long long T = (long long)L.C + L.B;
  a.C = L.C;
  a.F = L.F;
  a.Fi = L.Fi;
  a.B = L.B;
  a.K = L.K;
  a.quirk_b = L.quirk_b;
  a.flavour = cfg->flavour;
  a.N = N;
  a.nblk_update = (L.C + plfbs::kBlock - 1) / plfbs::kBlock;
  a.dt = cfg->time_marching_step;
  a.pg = 1.0 / cfg->gamma;
  {
    const double w[3] = {2.0 / 9.0, 1.0 / 9.0, 1.0 / 72.0};
    for (int k = 0; k < 3; k++) {
      a.eq[k][0] = w[k];
      a.eq[k][1] = 3.0 * w[k];
      a.eq[k][2] = 4.5 * a.pg * w[k];
      a.eq[k][3] = 1.5 * a.pg * w[k];
    }
  }
  a.visc3 = cfg->visc * 3;
  // body force: +pressure_gradient on the GPU path (Solver_gpu.cu:700), the
  // CPU Solver's force = -pressure_gradient (Solver.cpp:213)
  a.pressure_gradient =
      cfg->flavour == PLFBS_FLAVOUR_CPU_SOLVER ? -cfg->pressure_gradient : cfg->pressure_gradient;
  a.tolerance = cfg->tolerance;
  a.inv_ref_rho = 1.0 / cfg->ref_rho;
  // the FP32 form keeps momentum residuals divided by U
  a.inv_ref_mom = fp32 ? 1.0 / cfg->ref_rho : 1.0 / (cfg->ref_rho * cfg->max_velocity);
  a.rho0 = cfg->ref_rho;
  a.uref = cfg->max_velocity;
  a.rho0f = (float)cfg->ref_rho;
  a.inv_uref_f = (float)(1.0 / cfg->max_velocity);
  for (int c = 0; c < 3; c++) a.origin[c] = cfg->origin[c];

  // element sizes: FP64 double4 = 32 B, FP32 float4 = 16 B
  const size_t e4 = fp32 ? 16 : 32;
  void* p = nullptr;
  if ((rc = dev_alloc(ctx, &p, (size_t)T * e4))) return fail(rc);
  a.state = p;
  if ((rc = dev_alloc(ctx, &p, (size_t)L.C * e4))) return fail(rc);
  a.t0 = p;
  if ((rc = dev_alloc(ctx, &p, (size_t)L.C * e4))) return fail(rc);
  a.t1 = p;
  if ((rc = dev_alloc(ctx, &p, (size_t)L.C * 3 * e4))) return fail(rc);
  a.grad = p;
  a.flux_maps = nullptr;
  if (!fp32)
    ctx->flux_maps_ok = encode_rows(&ctx->flux_maps.state, a.state, 4, L.C) &&
                        encode_rows(&ctx->flux_maps.grad, a.grad, 12, L.C);
  if ((rc = dev_alloc(ctx, &p, (size_t)L.F * e4))) return fail(rc);
  a.flux = p;
  {
    NvtxRange r("device layout");
    if ((rc = build_device_layout(ctx, *mesh))) return fail(rc);
    free_stage(ctx);  // stream-ordered: after the layout kernels that read it
  }
  {
    NvtxRange r("compact layout");
    if ((rc = build_compact_layout(ctx))) return fail(rc);
  }
  if (ctx->pre.bc[0]) {  // copied while the mesh copies ran
    a.bc0 = ctx->pre.bc[0];
    a.bc1 = ctx->pre.bc[1];
    a.bc2 = ctx->pre.bc[2];
    a.bc3 = ctx->pre.bc[3];
  } else if (fp32) {
    plfbs::BoundaryRecords32 b32;
    plfbs::boundary_records32(L, cfg->ref_rho, cfg->max_velocity, b32);
    if ((rc = dev_upload(ctx, &p, b32.bc0))) return fail(rc);
    a.bc0 = p;
    if ((rc = dev_upload(ctx, &p, b32.bc1))) return fail(rc);
    a.bc1 = p;
    if ((rc = dev_upload(ctx, &p, b32.bc2))) return fail(rc);
    a.bc2 = p;
    if ((rc = dev_upload(ctx, &p, b32.bc3))) return fail(rc);
    a.bc3 = p;
  } else {
    if ((rc = dev_upload(ctx, &p, L.bc0))) return fail(rc);
    a.bc0 = p;
    if ((rc = dev_upload(ctx, &p, L.bc1))) return fail(rc);
    a.bc1 = p;
    if ((rc = dev_upload(ctx, &p, L.bc2))) return fail(rc);
    a.bc2 = p;
    if ((rc = dev_upload(ctx, &p, L.bc3))) return fail(rc);
    a.bc3 = p;
  }
  if ((rc = dev_alloc(ctx, &p, (size_t)a.nblk_update * 4 * sizeof(double)))) return fail(rc);
  a.partial = static_cast<double*>(p);
  if ((rc = dev_alloc(ctx, &p, sizeof(DevStats)))) return fail(rc);
  a.stats = static_cast<DevStats*>(p);
  a.res_debug = nullptr;
  a.force_x = a.force_y = a.force_z = nullptr;
  a.fforce_x = a.fforce_y = a.fforce_z = nullptr;
  if (N > 0) {
    const double dx = cfg->domain_dt * 2;  // Solver_gpu.cu:517
    a.ibm_dx = dx;
    a.ibm_inv_dx3 = 1 / dx / dx / dx;
    a.ibm_xc = (int)(cfg->lengths[0] / dx);
    a.ibm_yc = (int)(cfg->lengths[1] / dx);
    a.ibm_area_k = ibm->stiffness * (2 * std::acos(-1.0) * ibm->radius / ibm->object_nodes * ibm->depth);
    if (fp32) {
      for (float** f : {&a.fforce_x, &a.fforce_y, &a.fforce_z}) {
        if ((rc = dev_alloc(ctx, &p, (size_t)L.C * sizeof(float)))) return fail(rc);
        *f = static_cast<float*>(p);
      }
    } else {
      for (double** f : {&a.force_x, &a.force_y, &a.force_z}) {
        if ((rc = dev_alloc(ctx, &p, (size_t)L.C * sizeof(double)))) return fail(rc);
        *f = static_cast<double*>(p);
      }
    }
    std::vector<double> x(ibm->x, ibm->x + 3 * (size_t)N), xr(ibm->x_ref, ibm->x_ref + 3 * (size_t)N);
    if ((rc = dev_upload(ctx, &p, x))) return fail(rc);
    a.node_x = static_cast<double*>(p);
    if ((rc = dev_upload(ctx, &p, x))) return fail(rc);
    a.node_x0 = static_cast<double*>(p);
    if ((rc = dev_upload(ctx, &p, xr))) return fail(rc);
    a.node_ref = static_cast<const double*>(p);
    if ((rc = dev_alloc(ctx, &p, 3 * (size_t)N * sizeof(double)))) return fail(rc);
    a.node_vel = static_cast<double*>(p);
    if ((rc = dev_alloc(ctx, &p, 3 * (size_t)N * sizeof(double)))) return fail(rc);
    a.node_force = static_cast<double*>(p);
    {  // the kernels take the nodes by the cell of their reference position
       // (the stencil origin of k_ibm), so a warp's nodes share cells
      std::vector<int64_t> key(N);
      for (int n = 0; n < N; n++) {
        const double* xr = ibm->x_ref + 3 * (size_t)n;
        const double r0 = (xr[0] - cfg->origin[0]) / dx;
        const double r1 = std::fabs((xr[1] - cfg->origin[1]) / dx);
        const double r2 = std::fabs((xr[2] - cfg->origin[2]) / dx);
        const double lo[3] = {std::round(r0) - 1, std::round(r1) - 1, std::round(r2) - 1};
        const bool ok = std::fabs(lo[0]) < 1e9 && std::fabs(lo[1]) < 1e9 &&
                        std::fabs(lo[2]) < 1e9;  // false for NaN too
        key[n] = ok ? (int64_t)lo[0] + (int64_t)lo[1] * a.ibm_xc +
                          (int64_t)lo[2] * a.ibm_xc * (int64_t)a.ibm_yc
                    : std::numeric_limits<int64_t>::max();
      }
      std::vector<int32_t> order(N);
      for (int n = 0; n < N; n++) order[n] = n;
      std::stable_sort(order.begin(), order.end(),
                       [&](int32_t u, int32_t v) { return key[u] < key[v]; });
      if ((rc = dev_upload(ctx, &p, order))) return fail(rc);
      a.ibm_order = static_cast<const int32_t*>(p);
    }
    if ((rc = reset_force(ctx))) return fail(rc);
  }
  if ((rc = capture_step(ctx))) return fail(rc);
  // this context's stream only: a device-wide synchronise would also wait on
  // a stream another thread is capturing into its step graph, which ends that
  // capture with an error
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return fail(set_err(ctx, PLFBS_ERR_CUDA, "setup failed"));
  release_staging(ctx);  // the copies from it have ended
  *out = ctx;
  return PLFBS_OK;
}

void plfbs_destroy(plfbs_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  release_staging(ctx);
  if (ctx->step_exec) cudaGraphExecDestroy(ctx->step_exec);
  if (ctx->stream) free_stage(ctx);
  for (void* p : ctx->allocs) cudaFreeAsync(p, ctx->stream);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->stats_host) give_pinned_stats(ctx->stats_host);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int plfbs_wall_forces(plfbs_ctx* ctx, const int32_t* wall_bc, int32_t n_wall, double* cd,
                      double* cl) {
  NvtxRange range("plfbs_wall_forces");
  TRY(check_ctx(ctx));
  if (!cd || !cl || n_wall < 0 || (n_wall > 0 && !wall_bc))
    return set_err(ctx, PLFBS_ERR_ARG, "wall_forces needs the wall list and two outputs");
  if (!ctx->have_state) return set_err(ctx, PLFBS_ERR_STATE, "wall_forces before set_state");
  const Layout& L = ctx->L;
  std::vector<int> walls(std::max(n_wall, 1) + 4, 0);  // [0, 4): a zero halt word, see below
  for (int k = 0; k < n_wall; k++) {
    const int i = wall_bc[k];
    if (i < 0 || i >= L.B) return set_err(ctx, PLFBS_ERR_ARG, "wall index out of range");
    const int b = L.bc_new_of_old[i];
    const int vt = (int)L.bc3[4 * (size_t)b + 3] >> 8;
    if (vt != 1 && vt != 2)
      return set_err(ctx, PLFBS_ERR_BC, "wall faces need velocity type 1 (Dirichlet) or 2 (Neumann)");
    walls[4 + k] = b;
  }
  // wall_buf: ints [0, 4) zero (a halt flag that reads 0), [4, 4 + n) the
  // walls, then (16-byte aligned) the two sums
  const size_t sums_at = ((size_t)(n_wall + 4) * sizeof(int) + 15) & ~(size_t)15;
  if (!ctx->wall_buf || ctx->wall_cap < n_wall) {
    void* p = nullptr;
    TRY(dev_alloc(ctx, &p, sums_at + 2 * sizeof(double)));
    ctx->wall_buf = static_cast<int*>(p);
    ctx->wall_cap = n_wall;
  }
  int* dev_walls = ctx->wall_buf;
  double* dev_out = reinterpret_cast<double*>(reinterpret_cast<char*>(dev_walls) + sums_at);
  CK(cudaMemcpyAsync(dev_walls, walls.data(), (size_t)(n_wall + 4) * sizeof(int),
                     cudaMemcpyHostToDevice, ctx->stream));
  // gradients (and ghost states) of the current state, as the reference's
  // update_unstructured_bcs + Get_LS_Gradients before cylinder_post_processing;
  // a halted (converged) context still recomputes them: its copy of the
  // arguments reads the halt flag from the zero word
  plfbs::KernelArgs a = ctx->args;
  a.stats = reinterpret_cast<plfbs::DevStats*>(dev_walls);
  plfbs::launch_gradient(a, ctx->cfg.precision, ctx->stream);
  CK(cudaGetLastError());
  const double g = ctx->cfg.gamma;
  plfbs::launch_wall_forces(ctx->args, ctx->cfg.precision, dev_walls + 4, n_wall,
                            ctx->cfg.visc * g, g, dev_out, ctx->stream);
  CK(cudaGetLastError());
  double out[2];
  CK(cudaMemcpyAsync(out, dev_out, sizeof out, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  // post_processing.cpp:168-169: drag on Y Z, lift on X Z
  *cd = 2 * out[0] / ctx->cfg.ref_rho / (ctx->cfg.max_velocity * ctx->cfg.max_velocity) /
        ctx->cfg.lengths[1] / ctx->cfg.lengths[2];
  *cl = 2 * out[1] / ctx->cfg.ref_rho / (ctx->cfg.max_velocity * ctx->cfg.max_velocity) /
        ctx->cfg.lengths[0] / ctx->cfg.lengths[2];
  return PLFBS_OK;
}

int plfbs_release_cached(int32_t device) {
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> g(g_pool_mutex);
    if (device < 0 || device >= plfbs::kMaxDevices)
      return set_err(nullptr, PLFBS_ERR_ARG, "device index out of range");
    pool = g_pools[device];
  }
  std::vector<DevStats*> pinned;
  std::vector<std::pair<void*, size_t>> staging;
  {
    std::lock_guard<std::mutex> g(g_pool_mutex);
    pinned.swap(g_pinned_stats);
    staging.swap(g_pinned_staging);
  }
  for (DevStats* p : pinned) cudaFreeHost(p);
  for (auto& b : staging) cudaFreeHost(b.first);
  if (!pool) return PLFBS_OK;
  cudaError_t e = cudaMemPoolTrimTo(pool, 0);
  if (e != cudaSuccess)
    return set_err(nullptr, PLFBS_ERR_CUDA, std::string("cudaMemPoolTrimTo: ") + cudaGetErrorString(e));
  return PLFBS_OK;
}

namespace {

// Uploads a state given in the caller's numbering (FP32 form: converted to
// deviation units), resets the run status and seeds the RK accumulators. The
// four arrays go up as they are (from pinned memory at the copy engines'
// rate, pageable memory through the driver's staging) and one kernel
// interleaves and renumbers them into the state records.
int seed_state(plfbs_ctx* ctx, const double* rho, const double* u, const double* v,
               const double* w, bool conserved) {
  NvtxRange range(conserved ? "plfbs_warm_start" : "plfbs_set_state");
  const Layout& L = ctx->L;
  const int64_t T = (int64_t)L.C + L.B;
  void* buf = nullptr;
  TRY(scratch_alloc(ctx, &buf, 4 * sizeof(double) * (size_t)T));
  double* d = static_cast<double*>(buf);
  const double* src[4] = {rho, u, v, w};
  int rc = PLFBS_OK;
  for (int k = 0; k < 4 && rc == PLFBS_OK; k++) {
    const cudaError_t e = cudaMemcpyAsync(d + k * T, src[k], sizeof(double) * (size_t)T,
                                          cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess)
      rc = set_err(ctx, PLFBS_ERR_CUDA, std::string("state upload: ") + cudaGetErrorString(e));
  }
  if (rc == PLFBS_OK)
    plfbs::launch_state_in(ctx->perm, T, d, d + T, d + 2 * T, d + 3 * T, ctx->cfg.precision,
                           ctx->cfg.max_velocity, ctx->cfg.ref_rho, ctx->args.state, ctx->stream);
  scratch_free(ctx, buf);
  TRY(rc);
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(ctx->args.stats, 0, sizeof(DevStats), ctx->stream));
  plfbs::launch_seed(ctx->args, ctx->cfg.precision, conserved, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  TRY(reset_force(ctx));
  ctx->stages_done = 0;
  ctx->have_state = true;
  return PLFBS_OK;
}

}  // namespace

int plfbs_set_state(plfbs_ctx* ctx, const double* rho, const double* u, const double* v,
                    const double* w, int64_t n_total) {
  TRY(check_ctx(ctx));
  const int64_t T = (int64_t)ctx->L.C + ctx->L.B;
  if (!rho || !u || !v || !w || n_total != T)
    return set_err(ctx, PLFBS_ERR_ARG, "set_state needs 4 arrays of n_cells + n_boundary values");
  return seed_state(ctx, rho, u, v, w, false);
}

int plfbs_warm_start(plfbs_ctx* ctx, const double* rho, const double* u, const double* v,
                     const double* w, int64_t n_total, const double* node_x, int32_t n_nodes) {
  TRY(check_ctx(ctx));
  const int64_t T = (int64_t)ctx->L.C + ctx->L.B;
  if (!rho || !u || !v || !w || n_total != T)
    return set_err(ctx, PLFBS_ERR_ARG, "warm_start needs 4 arrays of n_cells + n_boundary values");
  if (node_x && n_nodes != ctx->N) return set_err(ctx, PLFBS_ERR_ARG, "node count mismatch");
  if (node_x && ctx->N > 0) {
    const size_t n = 3 * (size_t)ctx->N * sizeof(double);
    CK(cudaMemcpyAsync(ctx->args.node_x, node_x, n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->args.node_x0, node_x, n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(ctx->args.node_vel, 0, n, ctx->stream));
    CK(cudaMemsetAsync(ctx->args.node_force, 0, n, ctx->stream));
  }
  return seed_state(ctx, rho, u, v, w, true);
}

// Checkpoint image: header, then in the caller's numbering the state
// [n_cells + n_boundary][4] and the RK accumulator [n_cells][4] as the
// context stores them (FP64, or FP32 deviation units), then the nodes'
// positions, velocities and forces [n_nodes][3] (FP64).
namespace {
struct CheckpointHeader {
  char magic[8];
  int32_t version, precision;
  int64_t n_cells, n_boundary, n_nodes, n_faces;
  uint64_t fingerprint;
  int32_t halt, converged, diverged, pad;
  int64_t steps, converged_step;
  double last[6];
};
const char kMagic[8] = {'P', 'L', 'F', 'B', 'S', 'C', 'K', '1'};

int64_t checkpoint_size(const plfbs_ctx* ctx) {
  const int64_t v = ctx->cfg.precision == PLFBS_FP32_DEVIATION ? 4 : 8;
  const int64_t T = (int64_t)ctx->L.C + ctx->L.B;
  return (int64_t)sizeof(CheckpointHeader) + 4 * v * (T + ctx->L.C) + 9 * 8 * (int64_t)ctx->N;
}

}  // namespace

int plfbs_checkpoint_bytes(plfbs_ctx* ctx, int64_t* bytes) {
  if (!ctx) return set_err(nullptr, PLFBS_ERR_ARG, "null context");
  if (!bytes) return set_err(ctx, PLFBS_ERR_ARG, "null output");
  *bytes = checkpoint_size(ctx);
  return PLFBS_OK;
}

int plfbs_save_checkpoint(plfbs_ctx* ctx, void* buf, int64_t bytes) {
  NvtxRange range("plfbs_save_checkpoint");
  TRY(check_ctx(ctx));
  if (!buf || bytes < checkpoint_size(ctx))
    return set_err(ctx, PLFBS_ERR_ARG, "checkpoint buffer smaller than plfbs_checkpoint_bytes");
  if (!ctx->have_state) return set_err(ctx, PLFBS_ERR_STATE, "checkpoint before set_state");
  if (ctx->stages_done != 0)
    return set_err(ctx, PLFBS_ERR_STATE, "checkpoint in the middle of a step (after run_stages)");
  TRY(read_stats(ctx));
  const Layout& L = ctx->L;
  const size_t rec = ctx->cfg.precision == PLFBS_FP32_DEVIATION ? 16 : 32;
  const int64_t T = (int64_t)L.C + L.B;
  CheckpointHeader h{};
  std::memcpy(h.magic, kMagic, sizeof kMagic);
  h.version = 1;
  h.precision = ctx->cfg.precision;
  h.n_cells = L.C;
  h.n_boundary = L.B;
  h.n_nodes = ctx->N;
  h.n_faces = L.F;
  h.fingerprint = ctx->fingerprint;
  const DevStats& st = *ctx->stats_host;
  h.halt = st.halt;
  h.converged = st.converged;
  h.diverged = st.diverged;
  h.steps = st.steps;
  h.converged_step = st.converged_step;
  for (int c = 0; c < 6; c++) h.last[c] = st.last[c];
  char* out = static_cast<char*>(buf);
  std::memcpy(out, &h, sizeof h);
  out += sizeof h;
  // the state and the RK accumulator gathered into the caller's order on the
  // device, then copied out
  void* stage = nullptr;
  TRY(scratch_alloc(ctx, &stage, rec * (size_t)T));
  plfbs::launch_records(ctx->perm, T, (int)rec, ctx->args.state, stage, true, ctx->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, stage, rec * (size_t)T, cudaMemcpyDeviceToHost, ctx->stream);
  out += rec * (size_t)T;
  if (e == cudaSuccess) {
    plfbs::launch_records(ctx->perm, L.C, (int)rec, ctx->args.t1, stage, true, ctx->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, stage, rec * (size_t)L.C, cudaMemcpyDeviceToHost, ctx->stream);
  scratch_free(ctx, stage);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess)
    return set_err(ctx, PLFBS_ERR_CUDA, std::string("checkpoint read-back: ") + cudaGetErrorString(e));
  out += rec * (size_t)L.C;
  if (ctx->N > 0) {
    const size_t n = 3 * (size_t)ctx->N * sizeof(double);
    CK(cudaMemcpyAsync(out, ctx->args.node_x, n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(out + n, ctx->args.node_vel, n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(out + 2 * n, ctx->args.node_force, n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return PLFBS_OK;
}

int plfbs_load_checkpoint(plfbs_ctx* ctx, const void* buf, int64_t bytes) {
  NvtxRange range("plfbs_load_checkpoint");
  TRY(check_ctx(ctx));
  if (!buf || bytes < (int64_t)sizeof(CheckpointHeader))
    return set_err(ctx, PLFBS_ERR_ARG, "checkpoint buffer too small");
  CheckpointHeader h;
  std::memcpy(&h, buf, sizeof h);
  const Layout& L = ctx->L;
  if (std::memcmp(h.magic, kMagic, sizeof kMagic) != 0 || h.version != 1)
    return set_err(ctx, PLFBS_ERR_ARG, "not a plfbs checkpoint (magic/version)");
  if (h.precision != ctx->cfg.precision)
    return set_err(ctx, PLFBS_ERR_ARG, "checkpoint precision differs from the context's");
  if (h.n_cells != L.C || h.n_boundary != L.B || h.n_nodes != ctx->N || h.n_faces != L.F ||
      h.fingerprint != ctx->fingerprint)
    return set_err(ctx, PLFBS_ERR_MESH, "checkpoint was written for another mesh or node set");
  if (bytes < checkpoint_size(ctx))
    return set_err(ctx, PLFBS_ERR_ARG, "checkpoint buffer truncated");
  const size_t rec = ctx->cfg.precision == PLFBS_FP32_DEVIATION ? 16 : 32;
  const int64_t T = (int64_t)L.C + L.B;
  const char* in = static_cast<const char*>(buf) + sizeof h;
  // scattered from the caller's order on the device; at a step boundary t0
  // equals t1
  void* stage = nullptr;
  TRY(scratch_alloc(ctx, &stage, rec * (size_t)T));
  cudaError_t e = cudaMemcpyAsync(stage, in, rec * (size_t)T, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    plfbs::launch_records(ctx->perm, T, (int)rec, stage, ctx->args.state, false, ctx->stream);
    e = cudaGetLastError();
  }
  in += rec * (size_t)T;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(stage, in, rec * (size_t)L.C, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    plfbs::launch_records(ctx->perm, L.C, (int)rec, stage, ctx->args.t1, false, ctx->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->args.t0, ctx->args.t1, rec * (size_t)L.C, cudaMemcpyDeviceToDevice,
                        ctx->stream);
  scratch_free(ctx, stage);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess)
    return set_err(ctx, PLFBS_ERR_CUDA, std::string("checkpoint upload: ") + cudaGetErrorString(e));
  in += rec * (size_t)L.C;
  if (ctx->N > 0) {
    const size_t n = 3 * (size_t)ctx->N * sizeof(double);
    CK(cudaMemcpyAsync(ctx->args.node_x, in, n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->args.node_x0, in, n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->args.node_vel, in + n, n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->args.node_force, in + 2 * n, n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  DevStats& st = *ctx->stats_host;  // pinned host copy of the status header
  std::memset(&st, 0, offsetof(DevStats, history));
  st.halt = h.halt;
  st.converged = h.converged;
  st.diverged = h.diverged;
  st.steps = h.steps;
  st.converged_step = h.converged_step;
  for (int c = 0; c < 6; c++) st.last[c] = h.last[c];
  CK(cudaMemsetAsync(ctx->args.stats, 0, sizeof(DevStats), ctx->stream));
  CK(cudaMemcpyAsync(ctx->args.stats, &st, offsetof(DevStats, history), cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  TRY(reset_force(ctx));
  ctx->stages_done = 0;
  ctx->have_state = true;
  return PLFBS_OK;
}

int plfbs_run(plfbs_ctx* ctx, int64_t max_steps, plfbs_stats* stats, double* history) {
  NvtxRange range("plfbs_run");
  TRY(check_ctx(ctx));
  if (!ctx->have_state) return set_err(ctx, PLFBS_ERR_STATE, "run before set_state");
  if (ctx->stages_done != 0)
    return set_err(ctx, PLFBS_ERR_STATE, "run in the middle of a step (after run_stages)");
  if (max_steps < 0) return set_err(ctx, PLFBS_ERR_ARG, "negative step count");
  TRY(read_stats(ctx));
  const long long start = ctx->stats_host->steps;
  long long done = 0;
  float ms_total = 0.f;
  const long long batch = plfbs::kHistoryCap / 2;
  bool halt = ctx->stats_host->halt != 0;
  while (done < max_steps && !halt) {
    const long long n = std::min<long long>(batch, max_steps - done);
    NvtxRange r("step batch");
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    for (long long k = 0; k < n; k++) CK(cudaGraphLaunch(ctx->step_exec, ctx->stream));
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    TRY(wait_steps(ctx, ctx->timeout_s));
    TRY(read_stats(ctx));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ms_total += ms;
    const long long now = ctx->stats_host->steps;
    if (history) {
      // the batch's records sit in the device ring buffer: at most two spans
      long long t = start + done;
      while (t < now) {
        const long long slot = t % plfbs::kHistoryCap;
        const long long span = std::min(now - t, (long long)plfbs::kHistoryCap - slot);
        CK(cudaMemcpyAsync(history + 6 * (t - start), ctx->args.stats->history[slot],
                           6 * sizeof(double) * span, cudaMemcpyDeviceToHost, ctx->stream));
        t += span;
      }
      CK(cudaStreamSynchronize(ctx->stream));
    }
    halt = ctx->stats_host->halt != 0;
    if (now - start == done && !halt)  // a batch that advanced nothing: never wait again
      return set_err(ctx, PLFBS_ERR_STATE, "the step graph made no progress");
    done = now - start;
  }
  CK(cudaGetLastError());
  if (stats) {
    const DevStats* s = ctx->stats_host;
    stats->steps_done = s->steps;
    stats->converged = s->converged;
    stats->status = s->diverged ? PLFBS_ERR_DIVERGED : PLFBS_OK;
    stats->max_error = s->last[1];
    stats->rho_rms = s->last[2];
    stats->u_rms = s->last[3];
    stats->v_rms = s->last[4];
    stats->w_rms = s->last[5];
    stats->kernel_ms = ms_total;
    stats->steps_run = s->steps - start;
  }
  TRY(check_fault(ctx));
  if (ctx->stats_host->diverged)
    return set_err(ctx, PLFBS_ERR_DIVERGED, "residual is NaN or rho exceeded 1000");
  return PLFBS_OK;
}

int plfbs_set_timeout(plfbs_ctx* ctx, double seconds) {
  TRY(check_ctx(ctx));
  if (!(seconds >= 0) || !std::isfinite(seconds))
    return set_err(ctx, PLFBS_ERR_ARG, "timeout is a finite number of seconds >= 0");
  ctx->timeout_s = seconds;
  return PLFBS_OK;
}

int plfbs_wait(plfbs_ctx* ctx, double seconds) {
  if (!ctx) return set_err(nullptr, PLFBS_ERR_ARG, "null context");
  if (!(seconds >= 0) || !std::isfinite(seconds))
    return set_err(ctx, PLFBS_ERR_ARG, "wait is a finite number of seconds >= 0");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess)
    return set_err(ctx, PLFBS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  if (!ctx->busy) return PLFBS_OK;
  return wait_steps(ctx, seconds > 0 ? seconds : 1e-9);  // 0: just ask
}

int plfbs_set_layout_compression(plfbs_ctx* ctx, int32_t on) {
  TRY(check_ctx(ctx));
  if (on != 0 && on != 1) return set_err(ctx, PLFBS_ERR_ARG, "compression is 0 or 1");
  if (ctx->stages_done != 0)
    return set_err(ctx, PLFBS_ERR_STATE, "layout change in the middle of a step");
  if (on && !ctx->compact_faces && !ctx->compact_cells)
    return set_err(ctx, PLFBS_ERR_ARG, "this mesh's records do not repeat enough for the compact layout");
  ctx->args.compact = on;
  return capture_step(ctx);
}

int plfbs_set_flux_kernel(plfbs_ctx* ctx, int32_t kind) {
  TRY(check_ctx(ctx));
  if (kind != 0 && kind != 1) return set_err(ctx, PLFBS_ERR_ARG, "flux kernel kind is 0 or 1");
  if (ctx->stages_done != 0)
    return set_err(ctx, PLFBS_ERR_STATE, "flux kernel change in the middle of a step");
  if (kind == 1 && (!ctx->flux_maps_ok || ctx->cfg.flavour != PLFBS_FLAVOUR_GPU))
    return set_err(ctx, PLFBS_ERR_ARG,
                   "the TMA-staged flux kernel needs an FP64 GPU-flavour context and "
                   "tensor-map support");
  if (kind == 1) plfbs::prepare_flux_tma();
  CK(cudaGetLastError());
  ctx->args.flux_maps = kind == 1 ? &ctx->flux_maps : nullptr;
  return capture_step(ctx);
}

int plfbs_get_state(plfbs_ctx* ctx, double* rho, double* u, double* v, double* w,
                    int64_t n_total) {
  NvtxRange range("plfbs_get_state");
  TRY(check_ctx(ctx));
  const Layout& L = ctx->L;
  const int64_t T = (int64_t)L.C + L.B;
  if (!rho || !u || !v || !w || n_total != T)
    return set_err(ctx, PLFBS_ERR_ARG, "get_state needs 4 arrays of n_cells + n_boundary values");
  void* buf = nullptr;
  TRY(scratch_alloc(ctx, &buf, 4 * sizeof(double) * (size_t)T));
  double* d = static_cast<double*>(buf);
  plfbs::launch_state_out(ctx->perm, T, ctx->args.state, ctx->cfg.precision,
                          ctx->cfg.max_velocity, ctx->cfg.ref_rho, d, d + T, d + 2 * T, d + 3 * T,
                          ctx->stream);
  cudaError_t e = cudaGetLastError();
  double* dst[4] = {rho, u, v, w};
  for (int k = 0; k < 4 && e == cudaSuccess; k++)
    e = cudaMemcpyAsync(dst[k], d + k * T, sizeof(double) * (size_t)T, cudaMemcpyDeviceToHost,
                        ctx->stream);
  scratch_free(ctx, buf);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess)
    return set_err(ctx, PLFBS_ERR_CUDA, std::string("state read-back: ") + cudaGetErrorString(e));
  return PLFBS_OK;
}

int plfbs_get_nodes(plfbs_ctx* ctx, double* x, double* vel, double* force, int32_t n_nodes) {
  TRY(check_ctx(ctx));
  if (n_nodes != ctx->N) return set_err(ctx, PLFBS_ERR_ARG, "node count mismatch");
  if (ctx->N == 0) return PLFBS_OK;
  const size_t n = 3 * (size_t)ctx->N * sizeof(double);
  if (x) CK(cudaMemcpyAsync(x, ctx->args.node_x, n, cudaMemcpyDeviceToHost, ctx->stream));
  if (vel) CK(cudaMemcpyAsync(vel, ctx->args.node_vel, n, cudaMemcpyDeviceToHost, ctx->stream));
  if (force) CK(cudaMemcpyAsync(force, ctx->args.node_force, n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PLFBS_OK;
}

int plfbs_get_body_force(plfbs_ctx* ctx, double frontal_area, double* cd, double* cl) {
  TRY(check_ctx(ctx));
  if (ctx->N == 0) return set_err(ctx, PLFBS_ERR_STATE, "no immersed body");
  if (!(frontal_area > 0) || !cd || !cl) return set_err(ctx, PLFBS_ERR_ARG, "bad argument");
  std::vector<double> f(3 * (size_t)ctx->N);
  CK(cudaMemcpyAsync(f.data(), ctx->args.node_force, f.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  double sx = 0.0, sy = 0.0;
  for (int n = 0; n < ctx->N; n++) {
    sx += f[3 * n];
    sy += f[3 * n + 1];
  }
  const double q = 0.5 * ctx->cfg.ref_rho * ctx->cfg.max_velocity * ctx->cfg.max_velocity * frontal_area;
  *cd = -sx / q;
  *cl = -sy / q;
  return PLFBS_OK;
}

int plfbs_set_debug(plfbs_ctx* ctx, int enable) {
  TRY(check_ctx(ctx));
  if ((enable != 0) == ctx->debug) return PLFBS_OK;
  if (enable) {
    void* p = nullptr;
    TRY(dev_alloc(ctx, &p, (size_t)ctx->L.C * (ctx->cfg.precision == PLFBS_FP32_DEVIATION ? 16 : 32)));
    ctx->args.res_debug = p;
  } else {
    ctx->args.res_debug = nullptr;
  }
  ctx->debug = enable != 0;
  return capture_step(ctx);
}

int plfbs_run_stages(plfbs_ctx* ctx, int64_t n_stages) {
  TRY(check_ctx(ctx));
  if (!ctx->have_state) return set_err(ctx, PLFBS_ERR_STATE, "run_stages before set_state");
  for (int64_t g = 0; g < n_stages; g++) {
    const int rk = (int)(ctx->stages_done % 4);
    if (rk == 0) plfbs::launch_ibm(ctx->args, ctx->cfg.precision, ctx->stream);
    plfbs::launch_gradient(ctx->args, ctx->cfg.precision, ctx->stream);
    plfbs::launch_flux(ctx->args, ctx->cfg.precision, ctx->stream);
    plfbs::launch_update(ctx->args, ctx->cfg.precision, rk, ctx->stream);
    CK(cudaGetLastError());
    ctx->stages_done = (ctx->stages_done + 1) % 4;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  TRY(read_stats(ctx));
  return check_fault(ctx);
}

int plfbs_get_gradients(plfbs_ctx* ctx, double* grad, int32_t n_cells) {
  TRY(check_ctx(ctx));
  const Layout& L = ctx->L;
  if (!grad || n_cells != L.C) return set_err(ctx, PLFBS_ERR_ARG, "gradients: need 12 n_cells");
  std::vector<double> g(12 * (size_t)L.C);
  if (ctx->cfg.precision == PLFBS_FP32_DEVIATION) {
    std::vector<float> f(g.size());
    CK(cudaMemcpyAsync(f.data(), ctx->args.grad, f.size() * sizeof(float), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double U = ctx->cfg.max_velocity;  // velocity gradients are stored / U
    for (size_t i = 0; i < g.size(); i++) g[i] = (i % 12 < 3 ? 1.0 : U) * f[i];
  } else {
    CK(cudaMemcpyAsync(g.data(), ctx->args.grad, g.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  for (int o = 0; o < L.C; o++)
    std::memcpy(grad + 12 * (size_t)o, &g[12 * (size_t)L.cell_new_of_old[o]], 12 * sizeof(double));
  return PLFBS_OK;
}

int plfbs_get_face_flux(plfbs_ctx* ctx, double* flux, int32_t n_faces) {
  TRY(check_ctx(ctx));
  const Layout& L = ctx->L;
  if (!flux || n_faces != L.F) return set_err(ctx, PLFBS_ERR_ARG, "face flux: need 4 n_faces");
  std::vector<double> g;
  TRY(download4(ctx, ctx->args.flux, (size_t)L.F, g, true));
  std::vector<int32_t> order(L.F);
  CK(cudaMemcpyAsync(order.data(), ctx->face_order, 4 * (size_t)L.F, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->cfg.precision == PLFBS_FP32_DEVIATION) {
    // add back the constant rho0/3 n A the deviation form leaves out (from the
    // FP32 face records: debug output, rounding of n A is ~6e-8 relative)
    std::vector<float> f0(4 * (size_t)L.F);
    CK(cudaMemcpyAsync(f0.data(), ctx->args.face0, f0.size() * sizeof(float),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double p3 = ctx->cfg.ref_rho / 3.0;
    for (int k = 0; k < L.F; k++)
      for (int c = 0; c < 3; c++)
        g[4 * (size_t)k + c] += p3 * (double)f0[4 * (size_t)k + c] * (double)f0[4 * (size_t)k + 3];
  }
  for (int k = 0; k < L.F; k++)
    std::memcpy(flux + 4 * (size_t)order[k], &g[4 * (size_t)k], 4 * sizeof(double));
  return PLFBS_OK;
}

int plfbs_get_layout(plfbs_ctx* ctx, int32_t* sizes, int32_t* cell_order, int32_t* face_order,
                     int32_t* stencil_nbr, double* stencil_w, int32_t* gather) {
  TRY(check_ctx(ctx));
  const Layout& L = ctx->L;
  const KernelArgs& a = ctx->args;
  if (!sizes) return set_err(ctx, PLFBS_ERR_ARG, "layout: null sizes");
  sizes[0] = L.K;
  sizes[1] = L.K2;
  sizes[2] = ctx->args.compact ? ctx->compact_faces : 0;
  sizes[3] = ctx->args.compact ? ctx->compact_cells : 0;
  const size_t C = L.C, KC = (size_t)L.K * C;
  if (cell_order) std::memcpy(cell_order, L.cell_old_of_new.data(), 4 * C);
  if (face_order)
    CK(cudaMemcpyAsync(face_order, ctx->face_order, 4 * (size_t)L.F, cudaMemcpyDeviceToHost,
                       ctx->stream));
  if (stencil_nbr)
    CK(cudaMemcpyAsync(stencil_nbr, a.st_nbr, 4 * KC, cudaMemcpyDeviceToHost, ctx->stream));
  if (gather)
    CK(cudaMemcpyAsync(gather, a.gather, 4 * (size_t)L.K2 * C, cudaMemcpyDeviceToHost,
                       ctx->stream));
  if (stencil_w) {
    const void* w[3] = {a.st_wx, a.st_wy, a.st_wz};
    for (int c = 0; c < 3; c++) {
      double* out = stencil_w + c * KC;
      if (ctx->cfg.precision == PLFBS_FP32_DEVIATION) {
        std::vector<float> f(KC);
        CK(cudaMemcpyAsync(f.data(), w[c], 4 * KC, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (size_t i = 0; i < KC; i++) out[i] = f[i];
      } else {
        CK(cudaMemcpyAsync(out, w[c], 8 * KC, cudaMemcpyDeviceToHost, ctx->stream));
      }
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return PLFBS_OK;
}

int plfbs_get_residual(plfbs_ctx* ctx, double* res, int32_t n_cells) {
  TRY(check_ctx(ctx));
  const Layout& L = ctx->L;
  if (!ctx->args.res_debug) return set_err(ctx, PLFBS_ERR_STATE, "enable plfbs_set_debug first");
  if (!res || n_cells != L.C) return set_err(ctx, PLFBS_ERR_ARG, "residual: need 4 n_cells");
  std::vector<double> g;
  TRY(download4(ctx, ctx->args.res_debug, (size_t)L.C, g, true));
  for (int o = 0; o < L.C; o++)
    std::memcpy(res + 4 * (size_t)o, &g[4 * (size_t)L.cell_new_of_old[o]], 4 * sizeof(double));
  return PLFBS_OK;
}

int plfbs_profile_steps(plfbs_ctx* ctx, int64_t n_steps, double* ms) {
  TRY(check_ctx(ctx));
  if (!ms) return set_err(ctx, PLFBS_ERR_ARG, "null output");
  if (!ctx->have_state || ctx->stages_done != 0)
    return set_err(ctx, PLFBS_ERR_STATE, "profile needs a state at a step boundary");
  for (int k = 0; k < 4; k++) ms[k] = 0.0;
  // ev[0] before the IBM kernel, ev[1] after it, ev[2 + 3 rk + j] after kernel j
  // (gradient, flux, update) of stage rk: 14 events in all
  cudaEvent_t ev[14];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  const KernelArgs& a = ctx->args;
  const int prec = ctx->cfg.precision;
  for (int64_t t = 0; t < n_steps; t++) {
    CK(cudaEventRecord(ev[0], ctx->stream));
    plfbs::launch_ibm(a, prec, ctx->stream);
    CK(cudaEventRecord(ev[1], ctx->stream));
    for (int rk = 0; rk < 4; rk++) {
      plfbs::launch_gradient(a, prec, ctx->stream);
      CK(cudaEventRecord(ev[2 + 3 * rk], ctx->stream));
      plfbs::launch_flux(a, prec, ctx->stream);
      CK(cudaEventRecord(ev[3 + 3 * rk], ctx->stream));
      plfbs::launch_update(a, prec, rk, ctx->stream);
      CK(cudaEventRecord(ev[4 + 3 * rk], ctx->stream));
    }
    CK(cudaEventSynchronize(ev[13]));
    float x = 0.f;
    CK(cudaEventElapsedTime(&x, ev[0], ev[1]));
    ms[0] += x;
    for (int rk = 0; rk < 4; rk++) {
      cudaEvent_t prev = ev[1 + 3 * rk];
      CK(cudaEventElapsedTime(&x, prev, ev[2 + 3 * rk]));
      ms[1] += x;
      CK(cudaEventElapsedTime(&x, ev[2 + 3 * rk], ev[3 + 3 * rk]));
      ms[2] += x;
      CK(cudaEventElapsedTime(&x, ev[3 + 3 * rk], ev[4 + 3 * rk]));
      ms[3] += x;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  CK(cudaGetLastError());
  TRY(read_stats(ctx));
  return check_fault(ctx);
}

int plfbs_profile_kernels(plfbs_ctx* ctx, int64_t launches, double* ms) {
  NvtxRange range("plfbs_profile_kernels");
  TRY(check_ctx(ctx));
  if (!ms || launches <= 0) return set_err(ctx, PLFBS_ERR_ARG, "need launches > 0 and an output");
  if (!ctx->have_state || ctx->stages_done != 0)
    return set_err(ctx, PLFBS_ERR_STATE, "profile needs a state at a step boundary");
  TRY(read_stats(ctx));
  if (ctx->stats_host->halt)
    return set_err(ctx, PLFBS_ERR_STATE, "the run has halted: its kernels return at entry");
  for (int k = 0; k < 5; k++) ms[k] = 0.0;
  // everything the launches write that a later step reads, copied aside on
  // the device and put back afterwards (flux, gradients and partial sums are
  // recomputed by the next step before they are read)
  const KernelArgs& a = ctx->args;
  const Layout& L = ctx->L;
  const int prec = ctx->cfg.precision;
  const size_t e4 = prec == PLFBS_FP32_DEVIATION ? 16 : 32, es = e4 / 4;
  const size_t T = (size_t)L.C + L.B, C = L.C, n3 = 3 * (size_t)ctx->N * sizeof(double);
  std::vector<std::pair<void*, size_t>> keep = {
      {a.state, e4 * T}, {a.t0, e4 * C}, {a.t1, e4 * C}, {a.stats, sizeof(DevStats)}};
  for (void* f : {(void*)a.force_x, (void*)a.force_y, (void*)a.force_z, (void*)a.fforce_x,
                  (void*)a.fforce_y, (void*)a.fforce_z})
    if (f) keep.emplace_back(f, es * C);
  if (ctx->N > 0)
    for (void* f : {(void*)a.node_x, (void*)a.node_x0, (void*)a.node_vel, (void*)a.node_force})
      keep.emplace_back(f, n3);
  size_t total = 0;
  for (auto& k : keep) total += (k.second + 255) / 256 * 256;
  void* snap = nullptr;
  TRY(scratch_alloc(ctx, &snap, total));
  char* q = static_cast<char*>(snap);
  cudaError_t e = cudaSuccess;
  for (auto& k : keep) {
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(q, k.first, k.second, cudaMemcpyDeviceToDevice, ctx->stream);
    q += (k.second + 255) / 256 * 256;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  // mean device time per launch of `launches` back-to-back launches
  auto timed = [&](auto&& launch) -> double {
    if (e != cudaSuccess) return 0.0;
    cudaEventRecord(e0, ctx->stream);
    for (int64_t i = 0; i < launches; i++) launch();
    cudaEventRecord(e1, ctx->stream);
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    float x = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&x, e0, e1);
    return (double)x / (double)launches;
  };
  if (ctx->N > 0) ms[0] = timed([&] { plfbs::launch_ibm(a, prec, ctx->stream); });
  ms[1] = timed([&] { plfbs::launch_gradient(a, prec, ctx->stream); });
  ms[2] = timed([&] { plfbs::launch_flux(a, prec, ctx->stream); });
  for (int rk = 0; rk < 4; rk++)
    ms[3] += 0.25 * timed([&] { plfbs::launch_update(a, prec, rk, ctx->stream, false); });
  ms[4] = timed([&] { plfbs::launch_finish(a, prec, ctx->stream); });
  q = static_cast<char*>(snap);
  for (auto& k : keep) {  // put back even after a failed launch
    cudaMemcpyAsync(k.first, q, k.second, cudaMemcpyDeviceToDevice, ctx->stream);
    q += (k.second + 255) / 256 * 256;
  }
  scratch_free(ctx, snap);
  const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess)
    return set_err(ctx, PLFBS_ERR_CUDA, std::string("profile_kernels: ") + cudaGetErrorString(e));
  TRY(read_stats(ctx));
  return check_fault(ctx);
}

int plfbs_memory_bytes(plfbs_ctx* ctx, int64_t* bytes) {
  if (!ctx || !bytes) return set_err(ctx, PLFBS_ERR_ARG, "null argument");
  *bytes = ctx->bytes;
  return PLFBS_OK;
}

}  // extern "C"
