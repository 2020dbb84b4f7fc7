// Reverse Cuthill-McKee by breadth-first levels: the per-thread steps of the
// device cell order (renumber 2, layout.cu), shared with a serial host
// evaluation so the same code can be checked without a GPU.
//
// The sequential order (setup.cpp rcm_order) runs a queue: start cells by
// ascending degree (stable), and each dequeued cell appends its unvisited
// neighbours by ascending degree, ties in the order of its internal faces.
// A cell of level L+1 is appended by the first cell of level L (in queue
// order) that touches it, so the level is rebuilt in parallel from the level
// before it:
//   claim  every frontier position p offers each unvisited neighbour the key
//          (p << 32 | j), j the neighbour's slot in p's face-ordered
//          adjacency; the neighbour keeps the smallest key, i.e. its parent
//          and the parent's first face to it;
//   count  p's children are the entries whose neighbour holds p's key for
//          that slot (repeated neighbours count once, at the first slot);
//   emit   after an exclusive scan of the counts, each child goes to
//          hi + (children of earlier positions) + (its rank among p's
//          children by (degree, slot)).
// Positions are unique across levels, so keys left on visited cells never
// match a later parent and need no reset.
#ifndef PLFBS_RCM_LEVELS_HPP
#define PLFBS_RCM_LEVELS_HPP

#include <cstdint>

#if defined(__CUDACC__)
#define PLFBS_RCM_HD __host__ __device__ __forceinline__
#else
#define PLFBS_RCM_HD inline
#endif

namespace plfbs {
namespace rcm {

constexpr unsigned long long kUnclaimed = ~0ull;

// Cell adjacency over the internal faces: the neighbours of cell c are
// adj[off[c] .. off[c + 1]) in face order; deg[c] = off[c + 1] - off[c].
struct Graph {
  int C;
  const int32_t* off;
  const int32_t* adj;
  const int32_t* deg;
};

PLFBS_RCM_HD unsigned long long claim_key(int p, int slot) {
  return ((unsigned long long)(uint32_t)p << 32) | (uint32_t)slot;
}

// Start key of an unvisited cell: the next start is the smallest.
PLFBS_RCM_HD unsigned long long start_key(int deg, int c) {
  return ((unsigned long long)(uint32_t)deg << 32) | (uint32_t)c;
}

// Adjacency entry (face << 32 | neighbour): sorting a cell's entries puts
// them in face order.
PLFBS_RCM_HD unsigned long long adj_entry(int face, int nbr) {
  return ((unsigned long long)(uint32_t)face << 32) | (uint32_t)nbr;
}

// Insertion sort of one cell's entries (a few per cell).
PLFBS_RCM_HD void sort_entries(unsigned long long* k, int n) {
  for (int i = 1; i < n; i++) {
    const unsigned long long x = k[i];
    int j = i - 1;
    while (j >= 0 && k[j] > x) {
      k[j + 1] = k[j];
      j--;
    }
    k[j + 1] = x;
  }
}

// Frontier position p (cell v) offers its unvisited neighbours its keys.
template <typename AtomicMin>
PLFBS_RCM_HD void claim(const Graph& g, const int32_t* pos, unsigned long long* key, int p, int v,
                        AtomicMin amin) {
  const int e0 = g.off[v], e1 = g.off[v + 1];
  for (int e = e0; e < e1; e++) {
    const int w = g.adj[e];
    if (pos[w] < 0) amin(&key[w], claim_key(p, e - e0));
  }
}

PLFBS_RCM_HD bool is_child(const Graph& g, const unsigned long long* key, int p, int v, int e) {
  return key[g.adj[e]] == claim_key(p, e - g.off[v]);
}

PLFBS_RCM_HD int count_children(const Graph& g, const unsigned long long* key, int p, int v) {
  int n = 0;
  for (int e = g.off[v]; e < g.off[v + 1]; e++) n += is_child(g, key, p, v, e) ? 1 : 0;
  return n;
}

// Places p's children at order[first ..]: rank by (degree, slot). Returns the
// number of placements refused because they fell outside [0, C).
PLFBS_RCM_HD int emit_children(const Graph& g, const unsigned long long* key, int p, int v,
                               long long first, int32_t* order, int32_t* pos) {
  const int e0 = g.off[v], e1 = g.off[v + 1];
  int bad = 0;
  for (int e = e0; e < e1; e++) {
    if (!is_child(g, key, p, v, e)) continue;
    const int w = g.adj[e], dw = g.deg[w];
    int rank = 0;
    for (int e2 = e0; e2 < e1; e2++) {
      if (e2 == e || !is_child(g, key, p, v, e2)) continue;
      const int d2 = g.deg[g.adj[e2]];
      rank += (d2 < dw || (d2 == dw && e2 < e)) ? 1 : 0;
    }
    const long long q = first + rank;
    if (q < 0 || q >= g.C) {
      bad++;
      continue;
    }
    order[q] = w;
    pos[w] = (int32_t)q;
  }
  return bad;
}

}  // namespace rcm
}  // namespace plfbs

#endif
