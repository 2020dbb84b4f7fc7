// The device layout builders of plfbs_create (the face order, records,
// stencil and gather built from the caller's mesh arrays, and the compact
// layout) and the polyMesh geometry entry point, plfbs_polymesh_geometry.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "capi_internal.hpp"

using plfbs::KernelArgs;
using plfbs::Layout;

namespace plfbs_capi {

// Device memory that lives only while the layout is built: returned to the
// pool (stream-ordered) when the builder returns, on every path.
struct ScratchList {
  plfbs_ctx* ctx;
  std::vector<void*> v;
  explicit ScratchList(plfbs_ctx* c) : ctx(c) {}
  ~ScratchList() {
    for (void* p : v) cudaFreeAsync(p, ctx->stream);
  }
  template <typename T>
  int alloc(T** dst, size_t bytes, bool zero) {
    cudaMemPool_t pool = device_pool(ctx->device);
    if (!pool) return set_err(ctx, PLFBS_ERR_CUDA, "device memory pool creation failed");
    void* p = nullptr;
    CK(cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 16), pool, ctx->stream));
    v.push_back(p);
    if (zero) CK(cudaMemsetAsync(p, 0, std::max<size_t>(bytes, 16), ctx->stream));
    *dst = static_cast<T*>(p);
    return PLFBS_OK;
  }
  template <typename T>
  int upload(const T** dst, const T* src, size_t count) {
    T* p = nullptr;
    TRY(alloc(&p, count * sizeof(T), false));
    if (count) CK(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    *dst = p;
    return PLFBS_OK;
  }
};

int stage_mesh(plfbs_ctx* ctx, const plfbs_mesh_view& m) {
  auto& g = ctx->stage;
  g.ok = false;
  const long long C = m.n_cells, F = m.n_faces, Fi = m.n_internal;
  if (C <= 0 || F <= 0 || Fi < 0 || Fi > F || 2 * F >= (1LL << 31) || !m.owner ||
      !m.neighbour || !m.face_area || !m.face_normal || !m.face_centroid || !m.streaming_dt ||
      !m.cell_volume || !m.cell_centroid)
    return PLFBS_OK;  // validation reports it
  const long long T = C + (F - Fi);
  cudaMemPool_t pool = device_pool(ctx->device);
  if (!pool) return set_err(ctx, PLFBS_ERR_CUDA, "device memory pool creation failed");
  auto up = [&](const void* src, size_t bytes, const void** dst) -> int {
    void* p = nullptr;
    CK(cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 16), pool, ctx->stream));
    g.bufs.push_back(p);
    CK(cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    *dst = p;
    return PLFBS_OK;
  };
  const void* q = nullptr;
  TRY(up(m.owner, 4 * (size_t)F, &q));
  g.owner = static_cast<const int32_t*>(q);
  TRY(up(m.neighbour, 4 * (size_t)F, &q));
  g.neighbour = static_cast<const int32_t*>(q);
  TRY(up(m.face_area, 8 * (size_t)F, &q));
  g.area = static_cast<const double*>(q);
  TRY(up(m.face_normal, 24 * (size_t)F, &q));
  g.normal = static_cast<const double*>(q);
  TRY(up(m.face_centroid, 24 * (size_t)F, &q));
  g.fcen = static_cast<const double*>(q);
  TRY(up(m.streaming_dt, 8 * (size_t)F, &q));
  g.sdt = static_cast<const double*>(q);
  TRY(up(m.cell_volume, 8 * (size_t)C, &q));
  g.vol = static_cast<const double*>(q);
  TRY(up(m.cell_centroid, 24 * (size_t)T, &q));
  g.ccen = static_cast<const double*>(q);
  g.C = (int)C;
  g.F = (int)F;
  g.Fi = (int)Fi;
  g.ok = true;
  // the stencil, when its size reads sanely (else the host checks and the
  // layout uploads it)
  if (m.stencil_offsets && m.stencil_cells && m.stencil_faces && m.stencil_offsets[0] == 0 &&
      m.stencil_offsets[C] >= 0) {
    const long long nnz = m.stencil_offsets[C];
    TRY(up(m.stencil_offsets, 4 * (size_t)(C + 1), &q));
    g.st_off = static_cast<const int32_t*>(q);
    TRY(up(m.stencil_cells, 4 * (size_t)nnz, &q));
    g.st_cells = static_cast<const int32_t*>(q);
    TRY(up(m.stencil_faces, 4 * (size_t)nnz, &q));
    g.st_faces = static_cast<const int32_t*>(q);
    void* p = nullptr;
    CK(cudaMallocFromPoolAsync(&p, sizeof(plfbs::MeshScan), pool, ctx->stream));
    g.bufs.push_back(p);
    g.scan = static_cast<plfbs::MeshScan*>(p);
    g.nnz = nnz;
    g.stencil = true;
  }
  return PLFBS_OK;
}

int scan_mesh(plfbs_ctx* ctx, plfbs::MeshScan* out, bool* launched) {
  const auto& g = ctx->stage;
  *launched = false;
  if (!g.ok || !g.stencil) return PLFBS_OK;
  plfbs::launch_mesh_scan(g.owner, g.neighbour, g.area, g.sdt, g.normal, g.vol, g.st_off,
                          g.st_cells, g.st_faces, g.C, g.F, g.Fi, g.nnz, g.scan, ctx->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, g.scan, sizeof *out, cudaMemcpyDeviceToHost, ctx->stream));
  *launched = true;
  return PLFBS_OK;
}

void free_stage(plfbs_ctx* ctx) {
  for (void* p : ctx->stage.bufs) cudaFreeAsync(p, ctx->stream);
  ctx->stage.bufs.clear();
  ctx->stage.ok = false;
  ctx->stage.stencil = false;
}

// The face, stencil and gather arrays of a context, built on the device from
// the caller's mesh arrays (layout.cu); sets args' layout pointers, L.K2 and
// the mesh fingerprint.
int build_device_layout(plfbs_ctx* ctx, const plfbs_mesh_view& m) {
  Layout& L = ctx->L;
  KernelArgs& a = ctx->args;
  const bool fp32 = ctx->cfg.precision == PLFBS_FP32_DEVIATION;
  const size_t C = L.C, F = L.F, Fi = L.Fi, B = L.B, T = C + B;
  const size_t nnz = (size_t)m.stencil_offsets[C];
  const size_t nwin = (C + plfbs::kFaceWindow - 1) / plfbs::kFaceWindow;
  const size_t es = fp32 ? sizeof(float) : sizeof(double);
  ScratchList S(ctx);
  plfbs::DevMesh d{};
  d.C = L.C;
  d.F = L.F;
  d.Fi = L.Fi;
  d.B = L.B;
  if (ctx->stage.ok) {  // copied at the start of plfbs_create
    const auto& g = ctx->stage;
    d.owner = g.owner;
    d.neighbour = g.neighbour;
    d.area = g.area;
    d.normal = g.normal;
    d.fcen = g.fcen;
    d.sdt = g.sdt;
    d.vol = g.vol;
    d.ccen = g.ccen;
  } else {
    TRY(S.upload(&d.owner, m.owner, F));
    TRY(S.upload(&d.neighbour, m.neighbour, F));
    TRY(S.upload(&d.area, m.face_area, F));
    TRY(S.upload(&d.normal, m.face_normal, 3 * F));
    TRY(S.upload(&d.fcen, m.face_centroid, 3 * F));
    TRY(S.upload(&d.sdt, m.streaming_dt, F));
    TRY(S.upload(&d.vol, m.cell_volume, C));
    TRY(S.upload(&d.ccen, m.cell_centroid, 3 * T));
  }
  if (ctx->stage.ok && ctx->stage.stencil) {
    d.st_off = ctx->stage.st_off;
    d.st_cells = ctx->stage.st_cells;
    d.st_faces = ctx->stage.st_faces;
  } else {
    TRY(S.upload(&d.st_off, m.stencil_offsets, C + 1));
    TRY(S.upload(&d.st_cells, m.stencil_cells, nnz));
    TRY(S.upload(&d.st_faces, m.stencil_faces, nnz));
  }
  void* p = nullptr;
  if (ctx->pre.cell_new) {  // copied while the mesh copies ran
    d.bc_new = static_cast<const int32_t*>(ctx->pre.bc_new);
    d.bc_old = static_cast<const int32_t*>(ctx->pre.bc_old);
    d.cell_new = static_cast<const int32_t*>(ctx->pre.cell_new);
  } else {
    TRY(S.upload(&d.bc_new, L.bc_new_of_old.data(), B));
    TRY(S.upload(&d.bc_old, L.bc_old_of_new.data(), B));
    TRY(dev_upload(ctx, &p, L.cell_new_of_old));  // kept: the IBM kernels map caller cells with it
    d.cell_new = static_cast<const int32_t*>(p);
  }
  // caller index -> device index, cells then ghosts (state transfer)
  TRY(pool_alloc(ctx, &p, 4 * T));
  ctx->perm = static_cast<int32_t*>(p);
  plfbs::launch_perm(d.cell_new, d.bc_new, L.C, L.B, ctx->perm, ctx->stream);
  CK(cudaGetLastError());
  plfbs::LayoutScratch s{};
  TRY(S.alloc(&s.own_cnt, 4 * C, true));
  TRY(S.alloc(&s.own_off, 4 * C, false));
  TRY(S.alloc(&s.cursor, 4 * C, true));
  TRY(S.alloc(&s.deg, 4 * C, true));
  TRY(S.alloc(&s.gcnt, 4 * C, true));
  TRY(S.alloc(&s.wsum, 4 * nwin, false));
  TRY(S.alloc(&s.wbase, 4 * (nwin + 1), false));
  TRY(S.alloc(&s.seg, 4 * Fi, false));
  TRY(S.alloc(&s.sig, 2 * Fi, false));
  TRY(S.alloc(&s.info, 4 * sizeof(int32_t), false));
  TRY(S.alloc(&s.fingerprint, sizeof(unsigned long long), true));
  const int32_t info0[4] = {L.C, 0, 0, 0};
  CK(cudaMemcpyAsync(s.info, info0, sizeof info0, cudaMemcpyHostToDevice, ctx->stream));

  TRY(pool_alloc(ctx, &p, 4 * F));
  ctx->face_order = static_cast<int32_t*>(p);
  TRY(pool_alloc(ctx, &p, 8 * F));
  int32_t* face_ids = static_cast<int32_t*>(p);
  void* face[3];
  for (void*& f : face) TRY(pool_alloc(ctx, &f, 4 * es * F));
  TRY(pool_alloc(ctx, &p, 4 * (size_t)L.K * C));
  int32_t* st_nbr = static_cast<int32_t*>(p);
  CK(cudaMemsetAsync(st_nbr, 0xff, 4 * (size_t)L.K * C, ctx->stream));
  void* w[3];
  for (void*& x : w) TRY(dev_alloc(ctx, &x, es * L.K * C));
  void* inv_volume = nullptr;
  TRY(pool_alloc(ctx, &inv_volume, es * C));

  plfbs::launch_layout_order(d, s, ctx->face_order, ctx->stream);
  plfbs::launch_layout_records(d, s, ctx->cfg.precision, ctx->cfg.gradient_mode,
                               ctx->cfg.visc * 3, 1.0 / ctx->cfg.gamma, ctx->face_order, face_ids,
                               face[0], face[1], face[2], st_nbr, w[0], w[1], w[2], inv_volume,
                               ctx->stream);
  CK(cudaGetLastError());
  struct {
    int32_t info[4];
    unsigned long long fp;
  } back;
  CK(cudaMemcpyAsync(back.info, s.info, sizeof back.info, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&back.fp, s.fingerprint, sizeof back.fp, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (back.info[0] < L.C) {
    std::ostringstream e;
    e << "singular least-squares matrix for cell (index " << back.info[0] << ", value 0)";
    return set_err(ctx, PLFBS_ERR_MESH, e.str());
  }
  L.K2 = back.info[1];
  if (fp32 && L.K2 > 16)
    return set_err(ctx, PLFBS_ERR_MESH, "the FP32 form handles cells with at most 16 faces");
  TRY(pool_alloc(ctx, &p, 4 * (size_t)L.K2 * C));
  int32_t* gather = static_cast<int32_t*>(p);
  CK(cudaMemsetAsync(gather, 0xff, 4 * (size_t)L.K2 * C, ctx->stream));
  plfbs::launch_layout_gather(d, s, face_ids, gather, ctx->stream);
  CK(cudaGetLastError());
  // sizes folded into the device's sum over the arrays
  uint64_t h = back.fp;
  for (int64_t v : {(int64_t)L.C, (int64_t)L.F, (int64_t)L.Fi}) h = (h ^ (uint64_t)v) * 1099511628211ull;
  ctx->fingerprint = h;
  a.K2 = L.K2;
  a.face_ids = face_ids;
  a.face0 = face[0];
  a.face1 = face[1];
  a.face2 = face[2];
  a.st_nbr = st_nbr;
  a.st_wx = w[0];
  a.st_wy = w[1];
  a.st_wz = w[2];
  a.gather = gather;
  a.inv_volume = inv_volume;
  a.ibm_map = d.cell_new;
  return PLFBS_OK;
}

// The device order pays a few launches and one read-back (tens of
// microseconds) per component and per breadth-first level, the host order
// about 50 ns per cell. A mesh in more pieces (beyond the cells without
// internal faces), or with more levels than max(256, C / 512) (a long thin
// mesh, whose levels hold few cells each), takes the host order, the same
// order: the device's share then costs about as much as the host order.
constexpr int kMaxDeviceComponents = 256;
inline int max_device_levels(int C) { return std::max(256, C / 512); }

int device_cell_order(plfbs_ctx* ctx, const plfbs_mesh_view& m, std::vector<int32_t>& order) {
  const int C = ctx->L.C, Fi = ctx->L.Fi;
  const size_t nwin = (C + plfbs::kFaceWindow - 1) / plfbs::kFaceWindow;
  ScratchList S(ctx);
  plfbs::RcmDev r{};
  r.C = C;
  r.Fi = Fi;
  TRY(S.upload(&r.owner, m.owner, Fi));
  TRY(S.upload(&r.neighbour, m.neighbour, Fi));
  TRY(S.alloc(&r.deg, 4 * (size_t)C, true));
  TRY(S.alloc(&r.cursor, 4 * (size_t)C, true));
  TRY(S.alloc(&r.cnt, 4 * (size_t)C, false));
  TRY(S.alloc(&r.win_off, 4 * (size_t)C, false));
  TRY(S.alloc(&r.wsum, 4 * nwin, false));
  TRY(S.alloc(&r.wbase, 4 * (nwin + 1), false));
  TRY(S.alloc(&r.off, 4 * ((size_t)C + 1), false));
  TRY(S.alloc(&r.adj_key, 16 * (size_t)Fi, false));
  TRY(S.alloc(&r.adj, 8 * (size_t)Fi, false));
  TRY(S.alloc(&r.pos, 4 * (size_t)C, false));
  TRY(S.alloc(&r.key, 8 * (size_t)C, false));
  TRY(S.alloc(&r.order, 4 * (size_t)C, true));
  TRY(S.alloc(&r.start, 8, false));
  TRY(S.alloc(&r.info, 16, true));
  CK(cudaMemsetAsync(r.pos, 0xff, 4 * (size_t)C, ctx->stream));
  CK(cudaMemsetAsync(r.key, 0xff, 8 * (size_t)C, ctx->stream));
  CK(cudaMemsetAsync(r.start, 0xff, 8, ctx->stream));
  // the total of the last window scan over n items
  auto scan_total = [&](int n, int& v) -> int {
    const size_t w = (n + plfbs::kFaceWindow - 1) / plfbs::kFaceWindow;
    CK(cudaMemcpyAsync(&v, r.wbase + w, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PLFBS_OK;
  };
  plfbs::launch_rcm_graph(r, ctx->stream);
  CK(cudaGetLastError());
  int hi = 0;  // cells placed so far
  TRY(scan_total(C, hi));
  if (hi < 0 || hi > C) return set_err(ctx, PLFBS_ERR_CUDA, "device cell order: bad count");
  int levels = 0;
  const int max_levels = max_device_levels(C);
  for (int comp = 0; hi < C; comp++) {
    if (comp == kMaxDeviceComponents || levels > max_levels) {
      order = plfbs::cell_order(C, Fi, m.owner, m.neighbour, 1);
      return PLFBS_OK;
    }
    plfbs::launch_rcm_start(r, hi, ctx->stream);
    int lo = hi++;
    while (lo < hi) {  // one level per pass; every pass places cells or ends the piece
      if (++levels > max_levels) break;  // the host order, above
      plfbs::launch_rcm_level(r, lo, hi, ctx->stream);
      CK(cudaGetLastError());
      int n = 0;
      TRY(scan_total(hi - lo, n));
      if (n < 0 || n > C - hi)
        return set_err(ctx, PLFBS_ERR_CUDA, "device cell order: level size out of range");
      lo = hi;
      hi += n;
    }
  }
  int32_t info[4];
  order.resize(C);
  CK(cudaMemcpyAsync(order.data(), r.order, 4 * (size_t)C, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(info, r.info, sizeof info, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (info[2] != 0)
    return set_err(ctx, PLFBS_ERR_CUDA, "device cell order: placements out of range");
  std::reverse(order.begin(), order.end());
  std::vector<char> seen(C, 0);  // a permutation before anything is indexed with it
  for (int c : order) {
    if (c < 0 || c >= C || seen[c])
      return set_err(ctx, PLFBS_ERR_CUDA, "device cell order is not a permutation");
    seen[c] = 1;
  }
  return PLFBS_OK;
}

// The compact layout: face records and cells' weight sets that are
// bitwise equal are stored once (layout.cu, dedupe), each item keeping an
// index. Used where a table holds at most 1/8 of the items (structured
// regions of a mesh repeat their geometry); otherwise the kernels read the
// per-item arrays. The per-item arrays stay for the other readers.
int build_compact_layout(plfbs_ctx* ctx) {
  Layout& L = ctx->L;
  KernelArgs& a = ctx->args;
  ctx->compact_faces = ctx->compact_cells = 0;
  const int fp32 = ctx->cfg.precision == PLFBS_FP32_DEVIATION;
  const size_t es = fp32 ? 4 : 8;
  ScratchList S(ctx);
  plfbs::RecordSource src[2];
  src[0] = {0, L.F, 0, fp32, a.face0, a.face1, a.face2};
  src[1] = {1, L.C, L.K, fp32, a.st_wx, a.st_wy, a.st_wz};
  plfbs::DedupeScratch d[2];
  int nwin[2];
  for (int k = 0; k < 2; k++) {
    const size_t n = (size_t)src[k].n;
    int P = 1;
    while ((size_t)P < 2 * n && P < (1 << 30)) P <<= 1;
    nwin[k] = (int)((n + plfbs::kFaceWindow - 1) / plfbs::kFaceWindow);
    d[k].P = P;
    TRY(S.alloc(&d[k].slot_hash, 8 * (size_t)P, true));
    TRY(S.alloc(&d[k].slot_rep, 4 * (size_t)P, false));
    CK(cudaMemsetAsync(d[k].slot_rep, 0x7f, 4 * (size_t)P, ctx->stream));
    TRY(S.alloc(&d[k].item_slot, 4 * n, false));
    TRY(S.alloc(&d[k].rep_of, 4 * n, false));
    TRY(S.alloc(&d[k].is_rep, 4 * n, false));
    TRY(S.alloc(&d[k].off, 4 * n, false));
    TRY(S.alloc(&d[k].wsum, 4 * (size_t)nwin[k], false));
    TRY(S.alloc(&d[k].wbase, 4 * (size_t)(nwin[k] + 1), false));
    TRY(S.alloc(&d[k].info, 16, true));
    plfbs::launch_dedupe_scan(src[k], d[k], ctx->stream);
  }
  CK(cudaGetLastError());
  int32_t unique[2], overflow[2];
  for (int k = 0; k < 2; k++) {
    CK(cudaMemcpyAsync(&unique[k], d[k].wbase + nwin[k], 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&overflow[k], d[k].info, 4, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  void* p = nullptr;
  for (int k = 0; k < 2; k++) {
    const int n = src[k].n, U = unique[k];
    if (overflow[k] || U <= 0 || U > n / 8) continue;
    TRY(pool_alloc(ctx, &p, 4 * (size_t)n));
    int32_t* index = static_cast<int32_t*>(p);
    if (k == 0) {
      void* t[3];
      for (void*& x : t) TRY(pool_alloc(ctx, &x, 4 * es * (size_t)U));
      plfbs::launch_dedupe_emit(src[k], d[k], index, t[0], t[1], t[2], ctx->stream);
      a.face_rec = index;
      a.frec0 = t[0];
      a.frec1 = t[1];
      a.frec2 = t[2];
      ctx->compact_faces = U;
      if (!fp32) {
        TRY(pool_alloc(ctx, &p, 4 * (size_t)U));
        void* relax = nullptr;
        TRY(pool_alloc(ctx, &relax, 16 * (size_t)U));
        plfbs::launch_record_sides(t[0], t[1], t[2], U, ctx->cfg.flavour,
                                   static_cast<int32_t*>(p), static_cast<double*>(relax),
                                   ctx->stream);
        a.frec_sides = static_cast<const int32_t*>(p);
        a.frec_relax = static_cast<const double*>(relax);
      }
    } else {
      TRY(pool_alloc(ctx, &p, 3 * es * (size_t)U * L.K));
      plfbs::launch_dedupe_emit(src[k], d[k], index, p, nullptr, nullptr, ctx->stream);
      a.cell_wset = index;
      a.wtab = p;
      ctx->compact_cells = U;
    }
  }
  CK(cudaGetLastError());
  a.compact = (ctx->compact_faces || ctx->compact_cells) ? 1 : 0;
  return PLFBS_OK;
}

}  // namespace plfbs_capi

namespace {

using namespace plfbs_capi;

int polymesh_geometry(plfbs_ctx* ctx, const plfbs_polymesh_view& pm, double ref_dt,
                      plfbs_mesh_arrays& out) {
  const size_t P = pm.n_points, F = pm.n_faces, Fi = pm.n_internal, C = pm.n_cells;
  const size_t B = F - Fi, T = C + B, nnz = 2 * Fi + B;
  const size_t nwin = (C + plfbs::kFaceWindow - 1) / plfbs::kFaceWindow;
  ScratchList S(ctx);
  plfbs::DevPolyMesh d{};
  d.P = pm.n_points;
  d.F = pm.n_faces;
  d.Fi = pm.n_internal;
  d.C = pm.n_cells;
  TRY(S.upload(&d.points, pm.points, 3 * P));
  TRY(S.upload(&d.face_offsets, pm.face_offsets, F + 1));
  TRY(S.upload(&d.face_points, pm.face_points, (size_t)pm.face_offsets[F]));
  TRY(S.upload(&d.owner, pm.owner, F));
  TRY(S.upload(&d.neighbour, pm.neighbour, Fi));
  plfbs::GeometryOut o{};
  TRY(S.alloc(&o.area, 8 * F, false));
  TRY(S.alloc(&o.normal, 24 * F, false));
  TRY(S.alloc(&o.fcen, 24 * F, false));
  TRY(S.alloc(&o.sdt, 8 * F, false));
  TRY(S.alloc(&o.vol, 8 * T, false));
  TRY(S.alloc(&o.ccen, 24 * T, false));
  TRY(S.alloc(&o.st_off, 4 * (C + 1), false));
  TRY(S.alloc(&o.st_cells, 4 * nnz, false));
  TRY(S.alloc(&o.st_faces, 4 * nnz, false));
  plfbs::GeometryScratch g{};
  TRY(S.alloc(&g.fcsum, 24 * F, false));
  TRY(S.alloc(&g.cnt, 4 * C, true));
  TRY(S.alloc(&g.cursor, 4 * C, true));
  TRY(S.alloc(&g.own_off, 4 * C, false));
  TRY(S.alloc(&g.wsum, 4 * nwin, false));
  TRY(S.alloc(&g.wbase, 4 * (nwin + 1), false));
  TRY(S.alloc(&g.info, 16, true));
  plfbs::launch_polymesh_geometry(d, ref_dt, o, g, ctx->stream);
  CK(cudaGetLastError());
  auto down = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  };
  CK(down(out.face_area, o.area, 8 * F));
  CK(down(out.face_normal, o.normal, 24 * F));
  CK(down(out.face_centroid, o.fcen, 24 * F));
  CK(down(out.streaming_dt, o.sdt, 8 * F));
  CK(down(out.cell_volume, o.vol, 8 * T));
  CK(down(out.cell_centroid, o.ccen, 24 * T));
  CK(down(out.stencil_offsets, o.st_off, 4 * (C + 1)));
  CK(down(out.stencil_cells, o.st_cells, 4 * nnz));
  CK(down(out.stencil_faces, o.st_faces, 4 * nnz));
  CK(cudaStreamSynchronize(ctx->stream));
  std::memcpy(out.owner, pm.owner, 4 * F);
  if (Fi) std::memcpy(out.neighbour, pm.neighbour, 4 * Fi);
  for (size_t f = Fi; f < F; f++) out.neighbour[f] = (int32_t)(C + f - Fi);
  return PLFBS_OK;
}

}  // namespace

extern "C" {

int plfbs_polymesh_geometry(const plfbs_polymesh_view* mesh, double visc, double gamma,
                            double fneq_min, int32_t device, plfbs_mesh_arrays* out) {
  plfbs_capi::NvtxRange range("plfbs_polymesh_geometry");
  if (!mesh || !out || !out->owner || !out->neighbour || !out->face_area || !out->face_normal ||
      !out->face_centroid || !out->streaming_dt || !out->cell_volume || !out->cell_centroid ||
      !out->stencil_offsets || !out->stencil_cells || !out->stencil_faces)
    return set_err(nullptr, PLFBS_ERR_ARG, "null argument");
  if (!std::isfinite(visc) || !(gamma > 0) || !std::isfinite(fneq_min))
    return set_err(nullptr, PLFBS_ERR_ARG, "geometry needs finite visc, fneq_min and gamma > 0");
  std::string err;
  int rc = plfbs::validate_polymesh(*mesh, err);
  if (rc) return set_err(nullptr, rc, err);
  if ((rc = check_device(device))) return rc;
  // calc_face_delta_t: the cap 3 nu / (gamma fneq_min) (none when fneq_min is 0)
  const double ref_dt = fneq_min != 0 ? visc * 3 / gamma / fneq_min : HUGE_VAL;
  plfbs_ctx tmp;
  tmp.device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking) != cudaSuccess)
    return set_err(nullptr, PLFBS_ERR_CUDA, "stream creation failed");
  rc = polymesh_geometry(&tmp, *mesh, ref_dt, *out);
  cudaStreamSynchronize(tmp.stream);  // the scratch frees are stream-ordered
  cudaStreamDestroy(tmp.stream);
  if (rc) plfbs::set_global_error(tmp.err);
  return rc;
}

}  // extern "C"
