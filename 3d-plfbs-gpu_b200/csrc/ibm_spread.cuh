// Warp-aggregated force spreading of the IBM kernels (the reference spreads
// with 24 CAS atomics per node, immersed_boundary_method.cu:299-375). The
// kernels take their nodes in a spatial order (KernelArgs::ibm_order: by the
// cell of each node's reference position), so the four nodes of a warp lie
// close together and their 2 x 2 x 2 stencils overlap. The lanes whose
// contributions land in one cell (__match_any_sync on the cell) add them in
// lane order and the group's lowest lane issues the cell's three atomics.
#pragma once

#include <cuda_runtime.h>

namespace plfbs {

// `act`: the lanes of the warp that reach this call (all of them must);
// `cell`: the target cell, or -1 for none; f: this lane's contribution.
template <typename T>
__device__ __forceinline__ void spread_aggregated(unsigned act, int cell, const T f[3], T* fx,
                                                  T* fy, T* fz) {
  const unsigned peers = __match_any_sync(act, cell);
  T s0 = T(0), s1 = T(0), s2 = T(0);
  for (unsigned m = peers; m; m &= m - 1) {
    const int l = __ffs(m) - 1;
    s0 += __shfl_sync(peers, f[0], l);
    s1 += __shfl_sync(peers, f[1], l);
    s2 += __shfl_sync(peers, f[2], l);
  }
  const int lane = threadIdx.x & 31;
  if (cell >= 0 && lane == __ffs(peers) - 1) {
    atomicAdd(fx + cell, s0);
    atomicAdd(fy + cell, s1);
    atomicAdd(fz + cell, s2);
  }
}

}  // namespace plfbs
