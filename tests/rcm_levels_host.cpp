// Test infrastructure: the device cell order of renumber 2 evaluated serially
// on the host. It runs the same per-thread steps (csrc/rcm_levels.hpp) in the
// same sequence as the kernels and the host driver (layout.cu,
// capi_layout.cpp device_cell_order), with the scatter done in reverse face
// order and the frontier threads run last to first, so the per-cell sort and
// the order independence of the claims are exercised. tests/test_rcm_levels.py
// builds it with g++ and compares it with the sequential order.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "rcm_levels.hpp"

namespace rcm = plfbs::rcm;

extern "C" int rcm_by_levels(int C, int Fi, const int32_t* owner, const int32_t* nb,
                             int32_t* out) {
  std::vector<int32_t> deg(C, 0), off(C + 1, 0), cursor(C, 0), adj(2 * (size_t)Fi);
  std::vector<unsigned long long> adj_key(2 * (size_t)Fi);
  for (int f = 0; f < Fi; f++) {
    deg[owner[f]]++;
    deg[nb[f]]++;
  }
  for (int c = 0; c < C; c++) off[c + 1] = off[c] + deg[c];
  for (int f = Fi - 1; f >= 0; f--) {
    adj_key[off[owner[f]] + cursor[owner[f]]++] = rcm::adj_entry(f, nb[f]);
    adj_key[off[nb[f]] + cursor[nb[f]]++] = rcm::adj_entry(f, owner[f]);
  }
  for (int c = 0; c < C; c++) {
    rcm::sort_entries(&adj_key[off[c]], deg[c]);
    for (int e = off[c]; e < off[c + 1]; e++) adj[e] = (int32_t)(adj_key[e] & 0xffffffffu);
  }
  const rcm::Graph g{C, off.data(), adj.data(), deg.data()};
  std::vector<int32_t> pos(C, -1), order(C, 0), cnt(C, 0);
  std::vector<unsigned long long> key(C, rcm::kUnclaimed);
  int hi = 0;
  for (int c = 0; c < C; c++)  // cells without internal faces, by index
    if (deg[c] == 0) {
      order[hi] = c;
      pos[c] = hi++;
    }
  int bad = 0;
  while (hi < C) {
    unsigned long long s = rcm::kUnclaimed;
    for (int c = 0; c < C; c++)
      if (pos[c] < 0) s = std::min(s, rcm::start_key(deg[c], c));
    const int s_cell = (int)(s & 0xffffffffu);
    order[hi] = s_cell;
    pos[s_cell] = hi;
    int lo = hi++;
    while (lo < hi) {
      for (int p = hi - 1; p >= lo; p--)
        rcm::claim(g, pos.data(), key.data(), p, order[p],
                   [](unsigned long long* a, unsigned long long v) { *a = std::min(*a, v); });
      for (int p = lo; p < hi; p++) cnt[p - lo] = rcm::count_children(g, key.data(), p, order[p]);
      long long first = hi;
      for (int p = lo; p < hi; p++) {
        bad += rcm::emit_children(g, key.data(), p, order[p], first, order.data(), pos.data());
        first += cnt[p - lo];
      }
      lo = hi;
      hi = (int)first;
    }
  }
  for (int i = 0; i < C; i++) out[i] = order[C - 1 - i];
  return bad;
}
