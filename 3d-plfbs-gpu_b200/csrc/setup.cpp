// Host-side preparation of a case for the device: validation, locality
// renumbering, boundary order and records, and the host-only least-squares
// weights export. The O(faces) layout is built on the device (layout.cu).
#include <algorithm>
#include <functional>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <queue>
#include <sstream>
#include <thread>

#include "plfbs_internal.hpp"

namespace plfbs {
namespace {

std::string msg(const char* what, long long i, long long v) {
  std::ostringstream s;
  s << what << " (index " << i << ", value " << v << ")";
  return s.str();
}

inline bool finite(double x) { return std::isfinite(x); }

// Reverse Cuthill-McKee over the interior-cell graph of the internal faces:
// start cells by ascending degree (stable), breadth-first, the unvisited
// neighbours of each cell appended by ascending degree (stable, in face
// order), the whole order reversed.
std::vector<int32_t> rcm_order(int C, int Fi, const int32_t* owner, const int32_t* nb) {
  std::vector<int32_t> deg(C, 0);
  for (int f = 0; f < Fi; f++) {
    deg[owner[f]]++;
    deg[nb[f]]++;
  }
  std::vector<int64_t> off(C + 1, 0);
  int dmax = 0;
  for (int i = 0; i < C; i++) {
    off[i + 1] = off[i] + deg[i];
    dmax = std::max(dmax, deg[i]);
  }
  std::vector<int32_t> adj(off[C]);
  {
    std::vector<int64_t> pos(off.begin(), off.end() - 1);
    for (int f = 0; f < Fi; f++) {
      adj[pos[owner[f]]++] = nb[f];
      adj[pos[nb[f]]++] = owner[f];
    }
  }
  // counting sort of the cells by degree (stable)
  std::vector<int32_t> dstart(dmax + 2, 0), by_degree(C);
  for (int i = 0; i < C; i++) dstart[deg[i] + 1]++;
  for (int d = 0; d <= dmax; d++) dstart[d + 1] += dstart[d];
  for (int i = 0; i < C; i++) by_degree[dstart[deg[i]]++] = i;
  std::vector<char> seen(C, 0);
  std::vector<int32_t> order;
  order.reserve(C);
  size_t head = 0;
  for (int s : by_degree) {
    if (seen[s]) continue;
    seen[s] = 1;
    order.push_back(s);
    while (head < order.size()) {
      const int v = order[head++];
      const size_t first = order.size();
      for (int64_t e = off[v]; e < off[v + 1]; e++) {
        const int w = adj[e];
        if (seen[w]) continue;
        seen[w] = 1;
        // insert by degree after equal degrees (stable insertion sort)
        order.push_back(w);
        size_t j = order.size() - 1;
        while (j > first && deg[order[j - 1]] > deg[w]) {
          order[j] = order[j - 1];
          j--;
        }
        order[j] = w;
      }
    }
  }
  std::reverse(order.begin(), order.end());
  return order;  // order[new] = old
}

// body(i) for i in [0, n) on up to 16 host threads in contiguous chunks (the
// per-cell and per-face loops of the layout are independent); serial for
// small n or when no thread can be started.
template <typename Body>
void parallel_for(int n, const Body& body, int serial_below = 32768) {
  const unsigned hw = std::thread::hardware_concurrency();
  const int nt = (int)std::min(16u, hw ? hw : 1u);
  if (nt <= 1 || n < serial_below) {
    for (int i = 0; i < n; i++) body(i);
    return;
  }
  const int chunk = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  int lo = 0;
  for (; lo < n; lo += chunk) {
    const int hi = std::min(n, lo + chunk);
    try {
      th.emplace_back([lo, hi, &body] {
        for (int i = lo; i < hi; i++) body(i);
      });
    } catch (...) {
      break;  // run what is left on this thread
    }
  }
  for (int i = lo; i < n; i++) body(i);
  for (auto& t : th) t.join();
}

// Sorts distinct keys: chunks sorted on the host threads, then merged
// pairwise (in parallel within a round); std::sort below 64 K keys.
void parallel_sort(std::vector<uint64_t>& v) {
  const size_t n = v.size();
  const unsigned hw = std::thread::hardware_concurrency();
  const size_t nt = std::min<size_t>(16, hw ? hw : 1);
  if (nt <= 1 || n < 65536) {
    std::sort(v.begin(), v.end());
    return;
  }
  std::vector<size_t> cut(nt + 1);
  for (size_t k = 0; k <= nt; k++) cut[k] = n * k / nt;
  // a job per thread where a thread can be started, else on this one
  auto run_all = [](std::vector<std::function<void()>>& jobs) {
    std::vector<std::thread> th;
    size_t k = 0;
    for (; k < jobs.size(); k++) {
      try {
        th.emplace_back(jobs[k]);
      } catch (...) {
        break;
      }
    }
    for (; k < jobs.size(); k++) jobs[k]();
    for (auto& t : th) t.join();
  };
  {
    std::vector<std::function<void()>> jobs;
    for (size_t k = 0; k < nt; k++)
      jobs.emplace_back([&, k] { std::sort(v.begin() + cut[k], v.begin() + cut[k + 1]); });
    run_all(jobs);
  }
  std::vector<uint64_t> tmp(n);
  std::vector<uint64_t>*src = &v, *dst = &tmp;
  for (size_t width = 1; width < nt; width *= 2) {
    std::vector<std::function<void()>> jobs;
    for (size_t k = 0; k < nt; k += 2 * width) {
      const size_t a = cut[k], m = cut[std::min(nt, k + width)], b = cut[std::min(nt, k + 2 * width)];
      jobs.emplace_back([=] {
        std::merge(src->begin() + a, src->begin() + m, src->begin() + m, src->begin() + b,
                   dst->begin() + a);
      });
    }
    run_all(jobs);
    std::swap(src, dst);
  }
  if (src != &v) v.swap(tmp);
}

}  // namespace

// gradients::pre_fill_LHS_and_RHS_matrix (gradients.cpp:214-313) with
// add_non_macrovariable_contributions (gradients.cpp:149-210): the blend
// factor beta from the cell aspect ratio (hybrid) or fixed (LS = 1, GG = 0),
// LHS = sum w d d^T beta + 2 (1 - beta) V I, RHS_e = beta w d + (1 - beta) n A
// (sign by ownership), then the cofactor inverse with the reference's
// determinant, which reads (yx zz - yz - zx) in its second term
// (gradients.cpp:282-284); on meshes whose LHS has zero xy/yx terms (axis
// aligned hexes) that term vanishes and the inverse is exact.
int ls_weights(const plfbs_mesh_view& m, int mode, double* lhs_inv, double* rhs,
               std::string& err) {
  const int C = m.n_cells;
  std::atomic<int> bad(C);  // first cell with a singular matrix
  parallel_for(C, [&](int i) {
    double L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double* ci = m.cell_centroid + 3 * (size_t)i;
    double max_area = 0.0, max_disp = 0.0;
    const int e0 = m.stencil_offsets[i], e1 = m.stencil_offsets[i + 1];
    for (int e = e0; e < e1; e++) {
      const int i1 = m.stencil_cells[e], f = m.stencil_faces[e];
      max_area = std::max(max_area, m.face_area[f]);
      const double* c1 = m.cell_centroid + 3 * (size_t)i1;
      const double dx = c1[0] - ci[0], dy = c1[1] - ci[1], dz = c1[2] - ci[2];
      max_disp = std::max(std::sqrt(dx * dx + dy * dy + dz * dz), max_disp);
    }
    const double aspect = 2 * std::fabs(max_disp) * max_area / m.cell_volume[i];
    const int base = mode & 0xff;
    const double beta = base == PLFBS_GRAD_HYBRID ? std::min(1.0, 2 / aspect)
                        : base == PLFBS_GRAD_LS  ? 1.0
                                                 : 0.0;
    L[0] = L[0] + 2 * (1 - beta) * m.cell_volume[i];
    L[4] = L[4] + 2 * (1 - beta) * m.cell_volume[i];
    L[8] = L[8] + 2 * (1 - beta) * m.cell_volume[i];
    for (int e = e0; e < e1; e++) {
      const int i1 = m.stencil_cells[e], f = m.stencil_faces[e];
      const double* xf = m.face_centroid + 3 * (size_t)f;
      const double* n = m.face_normal + 3 * (size_t)f;
      double dx = xf[0] - ci[0], dy = xf[1] - ci[1], dz = xf[2] - ci[2];
      const double l_norm = dx * n[0] + dy * n[1] + dz * n[2];
      const double* c1 = m.cell_centroid + 3 * (size_t)i1;
      dx = c1[0] - ci[0];
      dy = c1[1] - ci[1];
      dz = c1[2] - ci[2];
      const double len = std::sqrt(std::pow(dx, 2.0) + std::pow(dy, 2.0) + std::pow(dz, 2.0));
      const double s = m.face_area[f];
      const double L_norm = dx * n[0] + dy * n[1] + dz * n[2];
      const double w = std::pow(2 * l_norm / L_norm, 2.0) * s / len;
      const double d[3] = {dx, dy, dz};
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) L[3 * r + c] = L[3 * r + c] + w * d[r] * d[c] * beta;
      const double sgn = (m.owner[f] == i) ? 1.0 : -1.0;
      for (int c = 0; c < 3; c++)
        rhs[3 * (size_t)e + c] = sgn > 0 ? beta * w * d[c] + 2 * (1 - beta) * 0.5 * n[c] * s
                                         : beta * w * d[c] + 2 * (1 - beta) * 0.5 * n[c] * -1 * s;
    }
    const double a = L[0], b = L[1], c = L[2], dd = L[3], e = L[4], f = L[5], g = L[6],
                 h = L[7], k = L[8];
    const double det = (mode & PLFBS_GRAD_EXACT_INVERSE)
                           ? a * (e * k - f * h) - b * (dd * k - f * g) + c * (dd * h - e * g)
                           : a * (e * k - f * h) + b * (dd * k - f - g) + c * (dd * h - e * g);
    double* o = lhs_inv + 9 * (size_t)i;
    o[0] = 1 / det * (e * k - f * h);
    o[1] = 1 / det * (c * h - b * k);
    o[2] = 1 / det * (b * f - c * e);
    o[3] = 1 / det * (f * g - dd * k);
    o[4] = 1 / det * (a * k - c * g);
    o[5] = 1 / det * (c * dd - a * f);
    o[6] = 1 / det * (dd * h - e * g);
    o[7] = 1 / det * (b * g - a * h);
    o[8] = 1 / det * (a * e - b * dd);
    if (!finite(o[0]) || !finite(o[4]) || !finite(o[8])) {
      int cur = bad.load();
      while (i < cur && !bad.compare_exchange_weak(cur, i)) {
      }
    }
  });
  if (bad.load() < C) {
    err = msg("singular least-squares matrix for cell", bad.load(), 0);
    return PLFBS_ERR_MESH;
  }
  return PLFBS_OK;
}

// The first index in [0, n) for which bad(i) holds, or n; bad() runs on up
// to 16 host threads.
template <typename Bad>
int first_bad(int n, const Bad& bad) {
  std::atomic<int> first(n);
  parallel_for(n, [&](int i) {
    if (!bad(i)) return;
    int cur = first.load();
    while (i < cur && !first.compare_exchange_weak(cur, i)) {
    }
  });
  return first.load();
}

int validate_polymesh(const plfbs_polymesh_view& pm, std::string& err) {
  const int P = pm.n_points, F = pm.n_faces, Fi = pm.n_internal, C = pm.n_cells;
  if (P <= 0 || C <= 0 || F <= 0 || Fi < 0 || Fi > F) {
    err = "polyMesh sizes must satisfy n_points, n_cells, n_faces > 0, 0 <= n_internal <= n_faces";
    return PLFBS_ERR_ARG;
  }
  if (!pm.points || !pm.face_offsets || !pm.face_points || !pm.owner || (Fi > 0 && !pm.neighbour)) {
    err = "null polyMesh array";
    return PLFBS_ERR_ARG;
  }
  if ((long long)F * 2 >= (1LL << 31)) {
    err = "too many faces";
    return PLFBS_ERR_MESH;
  }
  if (pm.face_offsets[0] != 0) {
    err = "face_offsets[0] must be 0";
    return PLFBS_ERR_MESH;
  }
  const int bn = first_bad(F, [&](int f) { return pm.face_offsets[f + 1] - pm.face_offsets[f] < 3; });
  if (bn < F) {
    err = msg("face with fewer than 3 vertices (or decreasing offsets)", bn,
              pm.face_offsets[bn + 1] - pm.face_offsets[bn]);
    return PLFBS_ERR_MESH;
  }
  const int bp = first_bad(F, [&](int f) {
    for (int k = pm.face_offsets[f]; k < pm.face_offsets[f + 1]; k++)
      if (pm.face_points[k] < 0 || pm.face_points[k] >= P) return true;
    return false;
  });
  if (bp < F) {
    err = msg("face vertex out of range", bp, 0);
    return PLFBS_ERR_MESH;
  }
  const int bo = first_bad(F, [&](int f) {
    if (pm.owner[f] < 0 || pm.owner[f] >= C) return true;
    return f < Fi && (pm.neighbour[f] < 0 || pm.neighbour[f] >= C || pm.neighbour[f] == pm.owner[f]);
  });
  if (bo < F) {
    err = msg("face owner or neighbour out of range", bo, pm.owner[bo]);
    return PLFBS_ERR_MESH;
  }
  return PLFBS_OK;
}

std::vector<int32_t> cell_order(int C, int Fi, const int32_t* owner, const int32_t* nb,
                                int renumber) {
  if (renumber == 1 || renumber == 2) return rcm_order(C, Fi, owner, nb);
  std::vector<int32_t> order(C);
  parallel_for(C, [&](int i) { order[i] = i; });
  return order;
}

// The checks of a caller's mesh arrays (first failing index in loop order):
// sizes, null arrays, face owners and neighbours, positive finite geometry,
// cell volumes, stencil offsets and entries. Everything that indexes with the
// caller's indices (the layout, the least-squares export) runs after them.
// *K_out receives the largest stencil.
int validate_mesh(const plfbs_mesh_view& m, std::string& err, int* K_out, const MeshScan* scan) {
  const int C = m.n_cells, F = m.n_faces, Fi = m.n_internal;
  if (C <= 0 || F <= 0 || Fi < 0 || Fi > F) {
    err = "mesh sizes must satisfy n_cells > 0, n_faces > 0, 0 <= n_internal <= n_faces";
    return PLFBS_ERR_ARG;
  }
  if (!m.owner || !m.neighbour || !m.face_area || !m.face_normal || !m.face_centroid ||
      !m.streaming_dt || !m.cell_volume || !m.cell_centroid || !m.stencil_offsets ||
      !m.stencil_cells || !m.stencil_faces) {
    err = "null mesh array";
    return PLFBS_ERR_ARG;
  }
  const int B = F - Fi;
  if ((long long)F * 2 >= (1LL << 31)) {
    err = "too many faces for the 31-bit gather encoding";
    return PLFBS_ERR_MESH;
  }
  const long long T = (long long)C + B;
  // --- mesh consistency (first failing index in loop order) ----------------
  auto face_problem = [&](int f) -> int {
    if (m.owner[f] < 0 || m.owner[f] >= C) return 1;
    if (f < Fi) {
      if (m.neighbour[f] < 0 || m.neighbour[f] >= C || m.neighbour[f] == m.owner[f]) return 2;
    } else if (m.neighbour[f] != C + (f - Fi)) {
      return 3;
    }
    if (!(m.face_area[f] > 0) || !finite(m.face_area[f]) || !(m.streaming_dt[f] > 0) ||
        !finite(m.face_normal[3 * (size_t)f]) || !finite(m.face_normal[3 * (size_t)f + 1]) ||
        !finite(m.face_normal[3 * (size_t)f + 2]))
      return 4;
    return 0;
  };
  const int bf = scan ? scan->bad_face : first_bad(F, [&](int f) { return face_problem(f) != 0; });
  if (bf < F) {
    static const char* what[5] = {"", "face owner out of range",
                                  "internal face neighbour out of range",
                                  "boundary face neighbour must be n_cells + face - n_internal",
                                  "face area, streaming dt or normal not positive/finite"};
    const int code = face_problem(bf);
    err = msg(what[code], bf, code == 1 ? m.owner[bf] : code == 4 ? 0 : m.neighbour[bf]);
    return PLFBS_ERR_MESH;
  }
  const int bv = scan ? scan->bad_volume : first_bad(C, [&](int i) {
    return !(m.cell_volume[i] > 0) || !finite(m.cell_volume[i]);
  });
  if (bv < C) {
    err = msg("cell volume not positive", bv, 0);
    return PLFBS_ERR_MESH;
  }
  if (m.stencil_offsets[0] != 0) {
    err = "stencil_offsets[0] must be 0";
    return PLFBS_ERR_MESH;
  }
  const int bo = scan ? scan->bad_offset : first_bad(C, [&](int i) {
    return m.stencil_offsets[i + 1] < m.stencil_offsets[i];
  });
  if (bo < C) {
    err = msg("stencil offsets decrease", bo, m.stencil_offsets[bo + 1]);
    return PLFBS_ERR_MESH;
  }
  // first bad stencil entry of each cell (entries of cell i lie in
  // [offsets[i], offsets[i+1]), so the first failing cell holds the first
  // failing entry)
  auto entry_problem = [&](int e, int i) -> int {
    const int j = m.stencil_cells[e], f = m.stencil_faces[e];
    if (j < 0 || j >= T || f < 0 || f >= F) return 1;
    const bool ok = (m.owner[f] == i && m.neighbour[f] == j) ||
                    (f < Fi && m.neighbour[f] == i && m.owner[f] == j);
    return ok ? 0 : 2;
  };
  const int bs = scan ? scan->bad_stencil : first_bad(C, [&](int i) {
    for (int e = m.stencil_offsets[i]; e < m.stencil_offsets[i + 1]; e++)
      if (entry_problem(e, i)) return true;
    return false;
  });
  if (bs < C) {
    for (int e = m.stencil_offsets[bs]; e < m.stencil_offsets[bs + 1]; e++) {
      const int code = entry_problem(e, bs);
      if (code) {
        err = msg(code == 1 ? "stencil entry out of range" : "stencil entry is not a face neighbour",
                  e, m.stencil_cells[e]);
        return PLFBS_ERR_MESH;
      }
    }
  }
  std::atomic<int> Kmax(scan ? scan->kmax : 0);
  if (!scan)
    parallel_for(C, [&](int i) {
      const int k = m.stencil_offsets[i + 1] - m.stencil_offsets[i];
      int cur = Kmax.load(std::memory_order_relaxed);
      while (k > cur && !Kmax.compare_exchange_weak(cur, k, std::memory_order_relaxed)) {
      }
    });
  const int K = Kmax.load();
  if (K == 0) {
    err = "empty gradient stencil";
    return PLFBS_ERR_MESH;
  }
  if (K_out) *K_out = K;
  return PLFBS_OK;
}

// The boundary arrays: present, and types the flavour defines, finite values.
static int check_bcs(const plfbs_config& cfg, const plfbs_bc_view& bcv, int B, std::string& err) {
  if (B > 0 && (!bcv.rho_type || !bcv.vel_type || !bcv.value)) {
    err = "null boundary array";
    return PLFBS_ERR_ARG;
  }
  const bool cpu = cfg.flavour == PLFBS_FLAVOUR_CPU_SOLVER;
  for (int b = 0; b < B; b++) {
    const int rt = bcv.rho_type[b], vt = bcv.vel_type[b];
    if (cpu ? (rt != 1 && rt != 2 && rt != 6 && rt != 7) : (rt != 1 && rt != 2)) {
      err = msg(cpu ? "boundary rho_type not taken by the CPU-Solver flavour (1, 2, 6, 7)"
                    : "boundary rho_type not defined on the GPU path (LBFS.cu:1252-1260 "
                      "handles 1 dirichlet and 2 neumann)",
                b, rt);
      return PLFBS_ERR_BC;
    }
    if (cpu ? (vt != 1 && vt != 2 && vt != 6 && vt != 8) : (vt != 1 && vt != 2 && vt != 9)) {
      err = msg(cpu ? "boundary vel_type not taken by the CPU-Solver flavour (1, 2, 6, 8)"
                    : "boundary vel_type not defined on the GPU path (LBFS.cu:1262-1294 "
                      "handles 1 dirichlet, 2 neumann, 9 parabolic)",
                b, vt);
      return PLFBS_ERR_BC;
    }
    for (int c = 0; c < 4; c++)
      if (!finite(bcv.value[4 * (size_t)b + c])) {
        err = msg("boundary value not finite", b, c);
        return PLFBS_ERR_BC;
      }
  }
  return PLFBS_OK;
}

int prepare_layout(const plfbs_config& cfg, const plfbs_mesh_view& m, const plfbs_bc_view& bcv,
                   Layout& L, std::string& err, const MeshScan* scan,
                   const std::function<int(MeshScan&)>& wait_scan) {
  const int C = m.n_cells, F = m.n_faces, Fi = m.n_internal, B = F - Fi;
  if (wait_scan && cfg.renumber != 1) {
    // The mesh checks run on the device meanwhile (the caller has checked the
    // sizes and pointers). The boundary checks, the identity order and the
    // boundary order and records (which guard the owners they index with)
    // go first; the errors come out in the order of the path below: the
    // mesh's, then the boundary arrays', then the order's.
    L.C = C;
    L.F = F;
    L.Fi = Fi;
    L.B = B;
    std::string berr, oerr;
    const int brc = check_bcs(cfg, bcv, B, berr);
    int orc = PLFBS_OK;
    if (!brc && cfg.renumber == 0)
      orc = order_layout(cfg, m, bcv, cell_order(C, Fi, m.owner, m.neighbour, 0), L, oerr);
    MeshScan s{};
    if (const int wrc = wait_scan(s)) {
      err = "the device mesh checks failed";
      return wrc;
    }
    int K = 0;
    if (const int vrc = validate_mesh(m, err, &K, &s)) return vrc;
    L.K = K;
    if (brc) {
      err = berr;
      return brc;
    }
    if (orc) err = oerr;
    return orc;
  }
  int K = 0;
  const int vrc = validate_mesh(m, err, &K, scan);
  if (vrc) return vrc;
  L.C = C;
  L.F = F;
  L.Fi = Fi;
  L.B = B;
  L.K = K;
  if (const int brc = check_bcs(cfg, bcv, B, err)) return brc;

  // --- renumbering ---------------------------------------------------------
  // renumber 2: the device builds the order, then plfbs_create calls
  // order_layout with it
  if (cfg.renumber == 2) return PLFBS_OK;
  return order_layout(cfg, m, bcv, cell_order(C, Fi, m.owner, m.neighbour, cfg.renumber), L, err);
}

int order_layout(const plfbs_config& cfg, const plfbs_mesh_view& m, const plfbs_bc_view& bcv,
                 std::vector<int32_t> order, Layout& L, std::string& err) {
  const int C = L.C, Fi = L.Fi, B = L.B;
  const bool cpu = cfg.flavour == PLFBS_FLAVOUR_CPU_SOLVER;
  L.cell_old_of_new = std::move(order);
  L.cell_new_of_old.resize(C);
  parallel_for(C, [&](int i) { L.cell_new_of_old[L.cell_old_of_new[i]] = i; });

  // Boundary faces by new owner, ties in face order (a stable sort by owner):
  // one sort of packed (new owner, boundary index) keys. The internal faces
  // are ordered on the device (layout.cu).
  // An owner out of range (arrays not checked yet: see prepare_layout) sorts
  // last; the checks then report it and this order is dropped.
  std::vector<uint64_t> key(B);
  parallel_for(B, [&](int b) {
    const int o = m.owner[Fi + b];
    const uint32_t no = (o >= 0 && o < C) ? (uint32_t)L.cell_new_of_old[o] : 0xffffffffu;
    key[b] = (uint64_t)no << 32 | (uint32_t)b;
  });
  parallel_sort(key);
  L.bc_old_of_new.resize(B);
  L.bc_new_of_old.resize(B);
  parallel_for(B, [&](int b) {
    const int bo = (int)(uint32_t)key[b];
    L.bc_old_of_new[b] = bo;
    L.bc_new_of_old[bo] = b;
  });
  L.quirk_b = B > 0 ? L.bc_new_of_old[0] : -1;

  // --- boundary records --------------------------------------------------------
  L.bc0.assign(4 * (size_t)B, 0.0);
  L.bc1.assign(4 * (size_t)B, 0.0);
  L.bc2.assign(4 * (size_t)B, 0.0);
  L.bc3.assign(4 * (size_t)B, 0.0);
  const double H = cfg.channel_height, H2 = H * 0.5, H4 = H * H * H * H;
  // records of the boundary faces in the new order, on the host threads; the
  // first face (new order) whose ghost sits on its owner is reported
  const int bad = first_bad(B, [&](int bn) {
    const int bo = L.bc_old_of_new[bn];
    const int f = Fi + bo;
    const int own = std::min(std::max(m.owner[f], 0), C - 1);  // in range once checked
    const double* val = bcv.value + 4 * (size_t)bo;
    const double* cg = m.cell_centroid + 3 * ((size_t)C + bo);
    const double* cn = m.cell_centroid + 3 * (size_t)own;
    const double* n = m.face_normal + 3 * (size_t)f;
    for (int c = 0; c < 4; c++) L.bc0[4 * (size_t)bn + c] = val[c];
    for (int c = 0; c < 4; c++) L.bc1[4 * (size_t)bn + c] = val[c];
    if (!cpu && bcv.vel_type[bo] == 9) {  // parabolic inlet target, LBFS.cu:1286
      L.bc1[4 * (size_t)bn] =
          16 * val[0] * (H2 + cg[1]) * (H2 - cg[1]) * (H2 + cg[2]) * (H2 - cg[2]) / H4;
    }
    const double dx = cg[0] - cn[0], dy = cg[1] - cn[1], dz = cg[2] - cn[2];
    const double dmag = std::sqrt(std::pow(dx, 2.0) + std::pow(dy, 2.0) + std::pow(dz, 2.0));
    // Dirichlet ghost-gradient direction and Neumann factors: the unit
    // owner->ghost vector and 1 - |n| (LBFS.cu:1306-1416), or for the CPU
    // Solver the face normal and 1 - n (gradients.cpp:412-414,612-645)
    double* d = &L.bc2[4 * (size_t)bn];
    d[0] = cpu ? n[0] : dx / dmag;
    d[1] = cpu ? n[1] : dy / dmag;
    d[2] = cpu ? n[2] : dz / dmag;
    d[3] = dmag;
    double* t = &L.bc3[4 * (size_t)bn];
    t[0] = cpu ? 1 - n[0] : 1 - std::fabs(n[0]);
    t[1] = cpu ? 1 - n[1] : 1 - std::fabs(n[1]);
    t[2] = cpu ? 1 - n[2] : 1 - std::fabs(n[2]);
    t[3] = (double)(bcv.rho_type[bo] | (bcv.vel_type[bo] << 8));
    return !(dmag > 0);
  });
  if (bad < B) {
    const int bo = L.bc_old_of_new[bad];
    err = msg("ghost centroid coincides with its owner's", bo, m.owner[Fi + bo]);
    return PLFBS_ERR_MESH;
  }
  return PLFBS_OK;
}

}  // namespace plfbs

namespace plfbs {

void boundary_records32(const Layout& L, double rho0, double uref, BoundaryRecords32& o) {
  const size_t B = L.B;
  auto cast = [](const std::vector<double>& v) {
    std::vector<float> r(v.size());
    for (size_t i = 0; i < v.size(); i++) r[i] = (float)v[i];
    return r;
  };
  // boundary values as deviations: velocity / U, rho - rho0
  auto dev = [&](const std::vector<double>& v) {
    std::vector<float> r(v.size());
    for (size_t b = 0; b < B; b++) {
      for (int c = 0; c < 3; c++) r[4 * b + c] = (float)(v[4 * b + c] / uref);
      r[4 * b + 3] = (float)(v[4 * b + 3] - rho0);
    }
    return r;
  };
  o.bc0 = dev(L.bc0);
  o.bc1 = dev(L.bc1);
  o.bc2 = cast(L.bc2);
  o.bc3 = cast(L.bc3);  // the type code (< 2^24) is exact in float
}

}  // namespace plfbs
