// Test infrastructure: the library's host-side setup (csrc/setup.cpp: the
// checks of the caller's mesh and boundary arrays, the cell order, the
// least-squares weights and the boundary records) built with AddressSanitizer
// and run on the meshes tests/test_asan_host.py writes, valid and corrupt.
// Every array is a heap block of exactly the size the C ABI promises, so any
// access past what the caller handed over ends the run with a sanitizer
// report. Prints one line per case: the status of each call.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "plfbs_internal.hpp"

namespace {

// The device mesh checks' results (csrc/mesh_scan.cu) computed here: the
// smallest failing index of each check, the largest stencil.
plfbs::MeshScan host_scan(const plfbs_mesh_view& m) {
  const int C = m.n_cells, F = m.n_faces, Fi = m.n_internal;
  const long long T = (long long)C + (F - Fi), nnz = m.stencil_offsets[C];
  plfbs::MeshScan s{F, C, C, C, 0};
  auto pf = [](double x) { return x > 0.0 && std::isfinite(x); };
  for (int f = 0; f < F && s.bad_face == F; f++) {
    const int o = m.owner[f], n = m.neighbour[f];
    bool bad = o < 0 || o >= C;
    bad = bad || (f < Fi ? (n < 0 || n >= C || n == o) : n != C + (f - Fi));
    bad = bad || !pf(m.face_area[f]) || !(m.streaming_dt[f] > 0.0);
    for (int c = 0; c < 3; c++) bad = bad || !std::isfinite(m.face_normal[3 * (size_t)f + c]);
    if (bad) s.bad_face = f;
  }
  for (int i = 0; i < C; i++) {
    if (s.bad_volume == C && !pf(m.cell_volume[i])) s.bad_volume = i;
    const int k = m.stencil_offsets[i + 1] - m.stencil_offsets[i];
    if (s.bad_offset == C && k < 0) s.bad_offset = i;
    s.kmax = std::max(s.kmax, k);
  }
  for (int i = 0; i < C && s.bad_stencil == C; i++) {
    const int e0 = m.stencil_offsets[i], e1 = m.stencil_offsets[i + 1];
    if (e0 < 0 || e1 < e0 || e1 > nnz) continue;
    for (int e = e0; e < e1; e++) {
      const int j = m.stencil_cells[e], f = m.stencil_faces[e];
      const bool bad = j < 0 || j >= T || f < 0 || f >= F ||
                       !((m.owner[f] == i && m.neighbour[f] == j) ||
                         (f < Fi && m.neighbour[f] == i && m.owner[f] == j));
      if (bad) {
        s.bad_stencil = i;
        break;
      }
    }
  }
  return s;
}

template <typename T>
std::vector<T> load(const std::string& dir, const char* name, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(dir + "/" + name, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T)));
  return v;
}

}  // namespace

int main(int argc, char** argv) {
  for (int a = 1; a < argc; a++) {
    const std::string dir = argv[a];
    long long C = 0, F = 0, Fi = 0, nnz = 0;
    {
      std::ifstream m(dir + "/meta.txt");
      m >> C >> F >> Fi >> nnz;
    }
    const long long B = F - Fi, T = C + B;
    auto owner = load<int32_t>(dir, "owner", F);
    auto nb = load<int32_t>(dir, "neighbour", F);
    auto area = load<double>(dir, "face_area", F);
    auto normal = load<double>(dir, "face_normal", 3 * F);
    auto fcen = load<double>(dir, "face_centroid", 3 * F);
    auto sdt = load<double>(dir, "streaming_dt", F);
    auto vol = load<double>(dir, "cell_volume", T);
    auto ccen = load<double>(dir, "cell_centroid", 3 * T);
    auto off = load<int32_t>(dir, "stencil_offsets", C + 1);
    auto sc = load<int32_t>(dir, "stencil_cells", nnz);
    auto sf = load<int32_t>(dir, "stencil_faces", nnz);
    auto rt = load<int32_t>(dir, "rho_type", B);
    auto vt = load<int32_t>(dir, "vel_type", B);
    auto bv = load<double>(dir, "bc_value", 4 * B);
    plfbs_mesh_view m{};
    m.n_cells = (int32_t)C;
    m.n_faces = (int32_t)F;
    m.n_internal = (int32_t)Fi;
    m.owner = owner.data();
    m.neighbour = nb.data();
    m.face_area = area.data();
    m.face_normal = normal.data();
    m.face_centroid = fcen.data();
    m.streaming_dt = sdt.data();
    m.cell_volume = vol.data();
    m.cell_centroid = ccen.data();
    m.stencil_offsets = off.data();
    m.stencil_cells = sc.data();
    m.stencil_faces = sf.data();
    plfbs_bc_view b{rt.data(), vt.data(), bv.data()};
    std::printf("%s", dir.c_str());
    const int flavours[2] = {PLFBS_FLAVOUR_GPU, PLFBS_FLAVOUR_CPU_SOLVER};
    for (int flavour : flavours)
      for (int renumber = 0; renumber <= 2; renumber++) {
        plfbs_config cfg{};
        cfg.visc = 0.01;
        cfg.gamma = 1.0;
        cfg.time_marching_step = 0.1;
        cfg.max_velocity = 0.1;
        cfg.ref_rho = 1.0;
        cfg.channel_height = 4.0;
        cfg.renumber = renumber;
        cfg.flavour = flavour;
        plfbs::Layout L;
        std::string err;
        int rc = plfbs::prepare_layout(cfg, m, b, L, err);
        if (renumber != 1) {
          // the path plfbs_create takes when the device checks the mesh: the
          // host's share first on unchecked arrays, then the checks' results
          plfbs::Layout L2;
          std::string err2;
          const int rc2 = plfbs::prepare_layout(cfg, m, b, L2, err2, nullptr,
                                                [&](plfbs::MeshScan& out) {
                                                  out = host_scan(m);
                                                  return PLFBS_OK;
                                                });
          bool same = rc2 == rc && err2 == err;
          if (same && rc == PLFBS_OK && renumber == 0)
            same = L2.bc_old_of_new == L.bc_old_of_new && L2.bc0 == L.bc0 && L2.bc1 == L.bc1 &&
                   L2.bc2 == L.bc2 && L2.bc3 == L.bc3 && L2.quirk_b == L.quirk_b &&
                   L2.K == L.K && L2.cell_new_of_old == L.cell_new_of_old;
          std::printf(" deferred%d%d=%d", flavour, renumber, same ? 1 : 0);
        }
        if (rc == PLFBS_OK && renumber == 2)  // the device order is the host RCM
          rc = plfbs::order_layout(cfg, m, b, plfbs::cell_order(m.n_cells, m.n_internal,
                                                                m.owner, m.neighbour, 1),
                                   L, err);
        std::printf(" layout%d%d=%d", flavour, renumber, rc);
      }
    // the host-only least-squares export, checked as plfbs_ls_weights checks it
    const int modes[4] = {PLFBS_GRAD_LS, PLFBS_GRAD_HYBRID, PLFBS_GRAD_GREEN_GAUSS,
                          PLFBS_GRAD_LS | PLFBS_GRAD_EXACT_INVERSE};
    for (int mode : modes) {
      std::vector<double> lhs(9 * (size_t)C), rhs(3 * (size_t)nnz);
      std::string err;
      int rc = plfbs::validate_mesh(m, err, nullptr);
      if (rc == PLFBS_OK) rc = plfbs::ls_weights(m, mode, lhs.data(), rhs.data(), err);
      std::printf(" ls%d=%d", mode, rc);
    }
    std::printf("\n");
  }
  return 0;
}
