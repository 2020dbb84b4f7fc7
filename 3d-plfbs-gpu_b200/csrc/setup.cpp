// Host-side preparation of a case for the device: validation, least-squares
// weights, locality renumbering and the packed face / boundary / stencil /
// gather records the kernels read.
#include <algorithm>
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

// Reverse Cuthill-McKee over the interior-cell graph of the internal faces.
std::vector<int32_t> rcm_order(int C, int Fi, const int32_t* owner, const int32_t* nb) {
  std::vector<int32_t> deg(C, 0);
  for (int f = 0; f < Fi; f++) {
    deg[owner[f]]++;
    deg[nb[f]]++;
  }
  std::vector<int64_t> off(C + 1, 0);
  for (int i = 0; i < C; i++) off[i + 1] = off[i] + deg[i];
  std::vector<int32_t> adj(off[C]);
  std::vector<int64_t> pos(off.begin(), off.end() - 1);
  for (int f = 0; f < Fi; f++) {
    adj[pos[owner[f]]++] = nb[f];
    adj[pos[nb[f]]++] = owner[f];
  }
  std::vector<int32_t> by_degree(C);
  std::iota(by_degree.begin(), by_degree.end(), 0);
  std::stable_sort(by_degree.begin(), by_degree.end(),
                   [&](int a, int b) { return deg[a] < deg[b]; });
  std::vector<char> seen(C, 0);
  std::vector<int32_t> order;
  order.reserve(C);
  std::vector<int32_t> nbrs;
  for (int s : by_degree) {
    if (seen[s]) continue;
    std::queue<int32_t> q;
    q.push(s);
    seen[s] = 1;
    while (!q.empty()) {
      int v = q.front();
      q.pop();
      order.push_back(v);
      nbrs.assign(adj.begin() + off[v], adj.begin() + off[v + 1]);
      std::stable_sort(nbrs.begin(), nbrs.end(), [&](int a, int b) { return deg[a] < deg[b]; });
      for (int w : nbrs)
        if (!seen[w]) {
          seen[w] = 1;
          q.push(w);
        }
    }
  }
  std::reverse(order.begin(), order.end());
  return order;  // order[new] = old
}

// For each of the 7 opposite lattice pairs of D3Q15 (first members e = x, y,
// z, (1,1,1), (1,1,-1), (1,-1,1), (-1,1,1)) the branch the flux kernel takes:
// 1 if e.n > 0.001 dt, 2 if e.n < -0.001 dt, 0 in the dead band
// (LBFS.cu:353-354); packed base 3.
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

int upwind_signature(const double* n, double dt) {
  static const int E[7][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 1},
                              {1, 1, -1}, {1, -1, 1}, {-1, 1, 1}};
  const double d1 = 0.001 * dt;
  int sig = 0, p3 = 1;
  for (int p = 0; p < 7; p++, p3 *= 3) {
    const double s = E[p][0] * n[0] + E[p][1] * n[1] + E[p][2] * n[2];
    sig += p3 * (s > d1 ? 1 : (s < -d1 ? 2 : 0));
  }
  return sig;
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

int build_layout(const plfbs_config& cfg, const plfbs_mesh_view& m, const plfbs_bc_view& bcv,
                 Layout& L, std::string& err) {
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
  if (B > 0 && (!bcv.rho_type || !bcv.vel_type || !bcv.value)) {
    err = "null boundary array";
    return PLFBS_ERR_ARG;
  }
  L.C = C;
  L.F = F;
  L.Fi = Fi;
  L.B = B;
  const long long T = (long long)C + B;
  // --- mesh consistency ---------------------------------------------------
  for (int f = 0; f < F; f++) {
    if (m.owner[f] < 0 || m.owner[f] >= C) {
      err = msg("face owner out of range", f, m.owner[f]);
      return PLFBS_ERR_MESH;
    }
    if (f < Fi) {
      if (m.neighbour[f] < 0 || m.neighbour[f] >= C || m.neighbour[f] == m.owner[f]) {
        err = msg("internal face neighbour out of range", f, m.neighbour[f]);
        return PLFBS_ERR_MESH;
      }
    } else if (m.neighbour[f] != C + (f - Fi)) {
      err = msg("boundary face neighbour must be n_cells + face - n_internal", f, m.neighbour[f]);
      return PLFBS_ERR_MESH;
    }
    if (!(m.face_area[f] > 0) || !finite(m.face_area[f]) || !(m.streaming_dt[f] > 0) ||
        !finite(m.face_normal[3 * (size_t)f]) || !finite(m.face_normal[3 * (size_t)f + 1]) ||
        !finite(m.face_normal[3 * (size_t)f + 2])) {
      err = msg("face area, streaming dt or normal not positive/finite", f, 0);
      return PLFBS_ERR_MESH;
    }
  }
  for (int i = 0; i < C; i++)
    if (!(m.cell_volume[i] > 0) || !finite(m.cell_volume[i])) {
      err = msg("cell volume not positive", i, 0);
      return PLFBS_ERR_MESH;
    }
  if (m.stencil_offsets[0] != 0) {
    err = "stencil_offsets[0] must be 0";
    return PLFBS_ERR_MESH;
  }
  int K = 0;
  for (int i = 0; i < C; i++) {
    const int e0 = m.stencil_offsets[i], e1 = m.stencil_offsets[i + 1];
    if (e1 < e0) {
      err = msg("stencil offsets decrease", i, e1);
      return PLFBS_ERR_MESH;
    }
    K = std::max(K, e1 - e0);
    for (int e = e0; e < e1; e++) {
      const int j = m.stencil_cells[e], f = m.stencil_faces[e];
      if (j < 0 || j >= T || f < 0 || f >= F) {
        err = msg("stencil entry out of range", e, j);
        return PLFBS_ERR_MESH;
      }
      const bool ok = (m.owner[f] == i && m.neighbour[f] == j) ||
                      (f < Fi && m.neighbour[f] == i && m.owner[f] == j);
      if (!ok) {
        err = msg("stencil entry is not a face neighbour", e, j);
        return PLFBS_ERR_MESH;
      }
    }
  }
  if (K == 0) {
    err = "empty gradient stencil";
    return PLFBS_ERR_MESH;
  }
  for (int b = 0; b < B; b++) {
    const int rt = bcv.rho_type[b], vt = bcv.vel_type[b];
    if (rt != 1 && rt != 2) {
      err = msg("boundary rho_type not defined on the GPU path (LBFS.cu:1252-1260 "
                "handles 1 dirichlet and 2 neumann)", b, rt);
      return PLFBS_ERR_BC;
    }
    if (vt != 1 && vt != 2 && vt != 9) {
      err = msg("boundary vel_type not defined on the GPU path (LBFS.cu:1262-1294 "
                "handles 1 dirichlet, 2 neumann, 9 parabolic)", b, vt);
      return PLFBS_ERR_BC;
    }
    for (int c = 0; c < 4; c++)
      if (!finite(bcv.value[4 * (size_t)b + c])) {
        err = msg("boundary value not finite", b, c);
        return PLFBS_ERR_BC;
      }
  }

  // --- least-squares weights (caller numbering) ------------------------------
  const int nnz = m.stencil_offsets[C];
  std::vector<double> lhs(9 * (size_t)C), rhs(3 * (size_t)nnz);
  int rc = ls_weights(m, cfg.gradient_mode, lhs.data(), rhs.data(), err);
  if (rc) return rc;

  // --- renumbering ---------------------------------------------------------
  L.cell_old_of_new.resize(C);
  L.cell_new_of_old.resize(C);
  if (cfg.renumber == 1) {
    L.cell_old_of_new = rcm_order(C, Fi, m.owner, m.neighbour);
  } else {
    std::iota(L.cell_old_of_new.begin(), L.cell_old_of_new.end(), 0);
  }
  for (int i = 0; i < C; i++) L.cell_new_of_old[L.cell_old_of_new[i]] = i;
  auto newc = [&](int old) { return L.cell_new_of_old[old]; };

  // Internal faces by (owner window, upwind signature, new owner, new
  // neighbour): within each window of kFaceWindow owners, faces with the same
  // signature take the same branches in the flux kernel (and on structured
  // meshes form a stream of owner/neighbour pairs at a fixed offset), while
  // the window keeps the cells they read resident in L2 across the classes.
  // Boundary faces by new owner.
  std::vector<int32_t> fint(Fi), fbnd(B);
  std::iota(fint.begin(), fint.end(), 0);
  std::iota(fbnd.begin(), fbnd.end(), Fi);
  constexpr int kFaceWindow = 4096;
  // one 64-bit key per face: window (high bits), signature (< 3^7, 12 bits),
  // owner within the window (12 bits); then the new neighbour and the face.
  struct FaceKey {
    uint64_t key;
    int32_t nb, f;
  };
  std::vector<FaceKey> keys(Fi);
  parallel_for(Fi, [&](int f) {
    const uint64_t o = (uint64_t)newc(m.owner[f]);
    const uint64_t sig =
        (uint64_t)upwind_signature(m.face_normal + 3 * (size_t)f, m.streaming_dt[f]);
    keys[f] = FaceKey{((o / kFaceWindow) << 24) | (sig << 12) | (o % kFaceWindow),
                      newc(m.neighbour[f]), f};
  });
  // the window is the leading key: bucket by window, then sort the windows
  // side by side
  const int nwin = (C + kFaceWindow - 1) / kFaceWindow;
  std::vector<int> woff(nwin + 1, 0);
  for (const FaceKey& k : keys) woff[(k.key >> 24) + 1]++;
  for (int w = 0; w < nwin; w++) woff[w + 1] += woff[w];
  std::vector<FaceKey> sorted(Fi);
  {
    std::vector<int> pos(woff.begin(), woff.end() - 1);
    for (const FaceKey& k : keys) sorted[pos[k.key >> 24]++] = k;
  }
  parallel_for(
      nwin,
      [&](int w) {
        std::sort(sorted.begin() + woff[w], sorted.begin() + woff[w + 1],
                  [](const FaceKey& a, const FaceKey& b) {
                    if (a.key != b.key) return a.key < b.key;
                    if (a.nb != b.nb) return a.nb < b.nb;
                    return a.f < b.f;
                  });
      },
      2);
  for (int k = 0; k < Fi; k++) fint[k] = sorted[k].f;
  std::stable_sort(fbnd.begin(), fbnd.end(),
                   [&](int a, int b) { return newc(m.owner[a]) < newc(m.owner[b]); });
  L.face_old_of_new.resize(F);
  L.face_new_of_old.resize(F);
  for (int k = 0; k < Fi; k++) L.face_old_of_new[k] = fint[k];
  for (int k = 0; k < B; k++) L.face_old_of_new[Fi + k] = fbnd[k];
  for (int k = 0; k < F; k++) L.face_new_of_old[L.face_old_of_new[k]] = k;
  L.bc_old_of_new.resize(B);
  L.bc_new_of_old.resize(B);
  for (int b = 0; b < B; b++) {
    L.bc_old_of_new[b] = fbnd[b] - Fi;
    L.bc_new_of_old[fbnd[b] - Fi] = b;
  }
  // any old cell index (interior or ghost) -> new
  auto newcell = [&](int old) { return old < C ? L.cell_new_of_old[old] : C + L.bc_new_of_old[old - C]; };
  L.quirk_b = B > 0 ? L.bc_new_of_old[0] : -1;

  L.centroid.resize(3 * (size_t)T);
  for (long long o = 0; o < T; o++) {
    const long long n = newcell((int)o);
    for (int c = 0; c < 3; c++) L.centroid[3 * n + c] = m.cell_centroid[3 * o + c];
  }

  // --- face records ----------------------------------------------------------
  L.face0.assign(4 * (size_t)F, 0.0);
  L.face1.assign(4 * (size_t)F, 0.0);
  L.face2.assign(4 * (size_t)F, 0.0);
  L.face_ids.assign(2 * (size_t)F, 0);
  const double visc3 = cfg.visc * 3, pg = 1.0 / cfg.gamma;
  parallel_for(F, [&](int k) {
    const int f = L.face_old_of_new[k];
    const int o = m.owner[f], nbo = m.neighbour[f];
    const double* n = m.face_normal + 3 * (size_t)f;
    const double* xf = m.face_centroid + 3 * (size_t)f;
    const double* c1 = m.cell_centroid + 3 * (size_t)o;
    const double* c2 = m.cell_centroid + 3 * (size_t)nbo;
    double* a = &L.face0[4 * (size_t)k];
    a[0] = n[0];
    a[1] = n[1];
    a[2] = n[2];
    a[3] = m.face_area[f];
    double* b = &L.face1[4 * (size_t)k];
    b[0] = m.streaming_dt[f];
    b[1] = c1[0] - xf[0];  // cell_1 - interface_node, LBFS.cu:343
    b[2] = c1[1] - xf[1];
    b[3] = c1[2] - xf[2];
    double* c = &L.face2[4 * (size_t)k];
    c[0] = c2[0] - xf[0];  // cell_2 - interface_node, LBFS.cu:344
    c[1] = c2[1] - xf[1];
    c[2] = c2[2] - xf[2];
    // relaxation factor 3 nu / (dt_s gamma) (calculate_flux_at_interface, LBFS.cu:1042-1223)
    c[3] = visc3 / m.streaming_dt[f] * pg;
    L.face_ids[2 * (size_t)k] = newc(o);
    L.face_ids[2 * (size_t)k + 1] = newcell(nbo);
  });

  // --- boundary records --------------------------------------------------------
  L.bc0.assign(4 * (size_t)B, 0.0);
  L.bc1.assign(4 * (size_t)B, 0.0);
  L.bc2.assign(4 * (size_t)B, 0.0);
  L.bc3.assign(4 * (size_t)B, 0.0);
  const double H = cfg.channel_height, H2 = H * 0.5, H4 = H * H * H * H;
  for (int bn = 0; bn < B; bn++) {
    const int bo = L.bc_old_of_new[bn];
    const int f = Fi + bo;
    const int own = m.owner[f];
    const double* val = bcv.value + 4 * (size_t)bo;
    const double* cg = m.cell_centroid + 3 * ((size_t)C + bo);
    const double* cn = m.cell_centroid + 3 * (size_t)own;
    const double* n = m.face_normal + 3 * (size_t)f;
    for (int c = 0; c < 4; c++) L.bc0[4 * (size_t)bn + c] = val[c];
    for (int c = 0; c < 4; c++) L.bc1[4 * (size_t)bn + c] = val[c];
    if (bcv.vel_type[bo] == 9) {  // parabolic inlet target, LBFS.cu:1286
      L.bc1[4 * (size_t)bn] =
          16 * val[0] * (H2 + cg[1]) * (H2 - cg[1]) * (H2 + cg[2]) * (H2 - cg[2]) / H4;
    }
    const double dx = cg[0] - cn[0], dy = cg[1] - cn[1], dz = cg[2] - cn[2];
    const double dmag = std::sqrt(std::pow(dx, 2.0) + std::pow(dy, 2.0) + std::pow(dz, 2.0));
    double* d = &L.bc2[4 * (size_t)bn];
    d[0] = dx / dmag;
    d[1] = dy / dmag;
    d[2] = dz / dmag;
    d[3] = dmag;
    double* t = &L.bc3[4 * (size_t)bn];
    t[0] = 1 - std::fabs(n[0]);
    t[1] = 1 - std::fabs(n[1]);
    t[2] = 1 - std::fabs(n[2]);
    t[3] = (double)(bcv.rho_type[bo] | (bcv.vel_type[bo] << 8));
    if (!(dmag > 0)) {
      err = msg("ghost centroid coincides with its owner's", bo, own);
      return PLFBS_ERR_MESH;
    }
  }

  // --- gradient stencil (ELL, precombined weights) ---------------------------
  L.K = K;
  L.st_nbr.assign((size_t)K * C, -1);
  L.st_wx.assign((size_t)K * C, 0.0);
  L.st_wy.assign((size_t)K * C, 0.0);
  L.st_wz.assign((size_t)K * C, 0.0);
  parallel_for(C, [&](int io) {
    const int in = newc(io);
    const double* Li = &lhs[9 * (size_t)io];
    int slot = 0;
    for (int e = m.stencil_offsets[io]; e < m.stencil_offsets[io + 1]; e++, slot++) {
      const double* r = &rhs[3 * (size_t)e];
      const size_t s = (size_t)slot * C + in;
      L.st_nbr[s] = newcell(m.stencil_cells[e]);
      L.st_wx[s] = Li[0] * r[0] + Li[1] * r[1] + Li[2] * r[2];
      L.st_wy[s] = Li[3] * r[0] + Li[4] * r[1] + Li[5] * r[2];
      L.st_wz[s] = Li[6] * r[0] + Li[7] * r[1] + Li[8] * r[2];
    }
  });

  // --- face -> cell gather ------------------------------------------------------
  std::vector<int32_t> nf(C, 0);
  for (int k = 0; k < F; k++) {
    const int f = L.face_old_of_new[k];
    nf[newc(m.owner[f])]++;
    if (f < Fi) nf[newc(m.neighbour[f])]++;
  }
  int K2 = 0;
  for (int i = 0; i < C; i++) K2 = std::max(K2, nf[i]);
  L.K2 = K2;
  L.gather.assign((size_t)K2 * C, -1);
  std::fill(nf.begin(), nf.end(), 0);
  for (int k = 0; k < F; k++) {
    const int f = L.face_old_of_new[k];
    const int o = newc(m.owner[f]);
    L.gather[(size_t)(nf[o]++) * C + o] = (k << 1);
    if (f < Fi) {
      const int nn = newc(m.neighbour[f]);
      L.gather[(size_t)(nf[nn]++) * C + nn] = (k << 1) | 1;
    }
  }
  if ((long long)F * 2 >= (1LL << 31)) {
    err = "too many faces for the 31-bit gather encoding";
    return PLFBS_ERR_MESH;
  }
  L.inv_volume.resize(C);
  for (int io = 0; io < C; io++) L.inv_volume[newc(io)] = 1.0 / m.cell_volume[io];
  return PLFBS_OK;
}

}  // namespace plfbs

namespace plfbs {

void build_layout32(const Layout& L, double rho0, double uref, Layout32& o) {
  const size_t F = L.F, B = L.B;
  auto cast = [](const std::vector<double>& v) {
    std::vector<float> r(v.size());
    for (size_t i = 0; i < v.size(); i++) r[i] = (float)v[i];
    return r;
  };
  o.face0 = cast(L.face0);
  o.face1 = cast(L.face1);
  o.face2 = cast(L.face2);  // (t2, relaxation factor)
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
  o.st_wx = cast(L.st_wx);
  o.st_wy = cast(L.st_wy);
  o.st_wz = cast(L.st_wz);
  o.inv_volume = cast(L.inv_volume);
}

}  // namespace plfbs
