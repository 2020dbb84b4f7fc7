// sm_100a kernels of the LBFS explicit time step (FP64 path).
//
// One RK stage is three kernels, and a time step is the IBM kernel plus four
// stages, all captured in one CUDA graph by capi.cpp:
//
//   gradient  (thread per cell)  ghost states inline + least-squares gradient
//                                 [get_interior_gradients, update_unstructured_bcs]
//   flux      (thread per face)  D3Q15 reconstruction + interface equilibrium
//                                 + relaxed moment flux, written per face
//                                 [calc_face_flux, get_bc_gradients]
//   update    (thread per cell)  face->cell gather (no atomics) + body force +
//                                 RK stage; last stage also reduces residuals
//                                 and tests convergence on the device
//                                 [add, time_integration, square/total<256>,
//                                  l2_norm_rms_moukallad]
//   ibm       (8 threads/node)   interpolation, advection, spring force and
//                                 spreading with FP64 atomics
//
// All of them are bandwidth kernels (no dense contraction: tensor cores do not
// apply). Memory per cell is laid out for coalesced 32-byte accesses.
#include <cuda_runtime.h>

#include <cstdint>

#include "ibm_spread.cuh"
#include "plfbs_internal.hpp"

namespace plfbs {
namespace {

struct __align__(32) d4 {
  double x, y, z, w;
};

// Records of four doubles move as one 256-bit access (a whole 32-byte
// sector per thread; every record array is 32-byte aligned): half the load
// and store instructions of two 128-bit halves (step 0.541 -> 0.502 ms).
// Read-only data: non-coherent load the compiler may schedule freely.
__device__ __forceinline__ d4 ld4(const void* base, long long i) {
  const double* p = reinterpret_cast<const double*>(base) + 4 * i;
  d4 v;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
      : "l"(p));
  return v;
}
// Coherent load, for data the same kernel also writes (kept in order).
__device__ __forceinline__ d4 ld4rw(const void* base, long long i) {
  const double* p = reinterpret_cast<const double*>(base) + 4 * i;
  d4 v;
  asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
               : "l"(p)
               : "memory");
  return v;
}
__device__ __forceinline__ void st4(void* base, long long i, const d4& v) {
  double* p = reinterpret_cast<double*>(base) + 4 * i;
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v.x), "d"(v.y), "d"(v.z),
               "d"(v.w)
               : "memory");
}

// The same pointer, opaque to the compiler, so that a load through it is not
// merged with an earlier load of the same address (a deliberate re-read).
template <typename T>
__device__ __forceinline__ const T* launder(const T* p) {
  asm("mov.b64 %0, %0;" : "+l"(p));
  return p;
}

// Whether the context has converged or diverged. One thread per block reads
// the flag; every thread of the block must call this (it synchronises).
__device__ __forceinline__ bool halted(const KernelArgs& a) {
  __shared__ int h;
  if (threadIdx.x == 0) h = *(volatile const int*)&a.stats->halt;
  __syncthreads();
  return h != 0;
}

// Ghost state from its owner. FL = 0 (GPU kernels, update_unstructured_bcs
// in LBFS.cu:1228-1301): bc1 holds the Dirichlet target, the raw value or for
// the parabolic inlet (vel type 9) the profile 16 u (H/2+y)(H/2-y)(H/2+z)(H/2-z)/H^4
// in x. FL = 1 (CPU Solver, Solution::update_unstructured_bcs,
// Solution.cpp:759-833): rho 1 mirror, 2 copy, 6 and 7 the value; velocity 1
// mirror, 2 copy, 6 the value, 8 (u, -v, w) of the owner.
template <int FL>
__device__ __forceinline__ d4 ghost_state(const d4& q, const d4& tgt, int types) {
  const int rt = types & 0xff, vt = types >> 8;
  d4 g;
  if (FL == 1) {
    g.w = rt == 1 ? tgt.w - (q.w - tgt.w) : (rt == 2 ? q.w : tgt.w);
    if (vt == 1) {
      g.x = tgt.x - (q.x - tgt.x);
      g.y = tgt.y - (q.y - tgt.y);
      g.z = tgt.z - (q.z - tgt.z);
    } else if (vt == 2) {
      g.x = q.x;
      g.y = q.y;
      g.z = q.z;
    } else if (vt == 8) {
      g.x = q.x;
      g.y = -q.y;
      g.z = q.z;
    } else {
      g.x = tgt.x;
      g.y = tgt.y;
      g.z = tgt.z;
    }
    return g;
  }
  g.w = (rt == 1) ? tgt.w - (q.w - tgt.w) : q.w;
  if (vt == 2) {
    g.x = q.x;
    g.y = q.y;
    g.z = q.z;
  } else {
    g.x = tgt.x - (q.x - tgt.x);
    g.y = tgt.y - (q.y - tgt.y);
    g.z = tgt.z - (q.z - tgt.z);
  }
  return g;
}

// ---------------------------------------------------------------------------
// gradient: grad_i = sum_e G_e (q_e - q_i), G_e = LHS_i^-1 RHS_e precombined.
// Gradient layout: 3 x d4 per cell = (rx, ry, rz, ux), (uy, uz, vx, vy),
// (vz, wx, wy, wz).
// ---------------------------------------------------------------------------
// One thread per cell. The neighbour ids of up to kStencilUnroll slots are
// loaded first, then every slot's weights and neighbour state, so a cell waits
// for two rounds of loads rather than two per slot; wider stencils fall back
// to walking the slots.
template <bool GHOSTS, int FL, bool CW>
__device__ __forceinline__ void gradient_slot(const KernelArgs& a, int i, long long s, int j,
                                              const d4& qi, double g[12], const double* wrow) {
  d4 qj;
  if (!GHOSTS || j < a.C) {
    qj = ld4(a.state, j);
  } else {
    const int b = j - a.C;
    const d4 tgt = ld4(a.bc1, b);
    const int types = (int)__ldg(reinterpret_cast<const double*>(a.bc3) + 4LL * b + 3);
    qj = ghost_state<FL>(qi, tgt, types);
    st4(a.state, j, qj);  // the ghost's only reader in this kernel is its owner
  }
  // CW: the cell's weight set from the compact table (wrow = its slot's triple)
  const double w[3] = {CW ? __ldg(wrow) : __ldg(static_cast<const double*>(a.st_wx) + s),
                       CW ? __ldg(wrow + 1) : __ldg(static_cast<const double*>(a.st_wy) + s),
                       CW ? __ldg(wrow + 2) : __ldg(static_cast<const double*>(a.st_wz) + s)};
  const double d[4] = {qj.w - qi.w, qj.x - qi.x, qj.y - qi.y, qj.z - qi.z};
#pragma unroll
  for (int f = 0; f < 4; f++)
#pragma unroll
    for (int c = 0; c < 3; c++) g[3 * f + c] = fma(w[c], d[f], g[3 * f + c]);
}

constexpr int kStencilUnroll = 8;

template <int FL, bool CW>
__global__ void __launch_bounds__(kBlock) k_gradient(const KernelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (halted(a)) return;
  if (i >= a.C) return;
  const d4 qi = ld4(a.state, i);
  const double* wset =
      CW ? static_cast<const double*>(a.wtab) + (size_t)__ldg(a.cell_wset + i) * a.K * 3 : nullptr;
  double g[12];
#pragma unroll
  for (int k = 0; k < 12; k++) g[k] = 0.0;
  if (a.K <= kStencilUnroll) {
    int jj[kStencilUnroll];
#pragma unroll
    for (int k = 0; k < kStencilUnroll; k++)
      jj[k] = k < a.K ? __ldg(a.st_nbr + (long long)k * a.C + i) : -1;
#pragma unroll
    for (int k = 0; k < kStencilUnroll; k++)
      if (jj[k] >= 0)
        gradient_slot<true, FL, CW>(a, i, (long long)k * a.C + i, jj[k], qi, g,
                                    CW ? wset + 3 * k : nullptr);
  } else {
    for (int k = 0; k < a.K; k++) {
      const long long s = (long long)k * a.C + i;
      const int j = __ldg(a.st_nbr + s);
      if (j < 0) break;
      gradient_slot<true, FL, CW>(a, i, s, j, qi, g, CW ? wset + 3 * k : nullptr);
    }
  }
  st4(a.grad, 3LL * i + 0, d4{g[0], g[1], g[2], g[3]});
  st4(a.grad, 3LL * i + 1, d4{g[4], g[5], g[6], g[7]});
  st4(a.grad, 3LL * i + 2, d4{g[8], g[9], g[10], g[11]});
}

// ---------------------------------------------------------------------------
// flux
// ---------------------------------------------------------------------------
// Gradients as 12 doubles: rho, u, v, w, each (x, y, z).
__device__ __forceinline__ void load_grad(const void* base, int c, double g[12]) {
  const d4 a0 = ld4(base, 3LL * c), a1 = ld4(base, 3LL * c + 1), a2 = ld4(base, 3LL * c + 2);
  g[0] = a0.x; g[1] = a0.y; g[2] = a0.z; g[3] = a0.w;
  g[4] = a1.x; g[5] = a1.y; g[6] = a1.z; g[7] = a1.w;
  g[8] = a2.x; g[9] = a2.y; g[10] = a2.z; g[11] = a2.w;
}

// Ghost gradient. FL = 0 (get_bc_gradients, LBFS.cu:1306-1416): Dirichlet
// 2 (bc - q_owner) / |d| * d_hat from the raw boundary value (bc2 = (d_hat,
// |d|)); Neumann the owner's gradient times (1 - |n|) componentwise (bc3).
// FL = 1 (gradients::Get_LS_Gradients and get_ghost_grads,
// gradients.cpp:395-506,592-648): Dirichlet (rho 1, velocity 1 and 8) along
// the face normal (bc2 = (n, |d|)), Neumann times (1 - n) (bc3), types 6 zero,
// rho 7 the owner's gradient.
template <int FL>
__device__ __forceinline__ void ghost_grad(const d4& q, const double go[12], const d4& bv,
                                           const d4& dd, const d4& nm, int types,
                                           double g[12]) {
  const int rt = types & 0xff, vt = types >> 8;
  const double dir[3] = {dd.x, dd.y, dd.z}, m[3] = {nm.x, nm.y, nm.z};
  const double dq[4] = {2 * (bv.w - q.w), 2 * (bv.x - q.x), 2 * (bv.y - q.y), 2 * (bv.z - q.z)};
  if constexpr (FL == 1) {
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const int t = f == 0 ? rt : vt;
#pragma unroll
      for (int c = 0; c < 3; c++)
        g[3 * f + c] = (t == 1 || (f > 0 && t == 8)) ? dq[f] / dd.w * dir[c]
                       : t == 2                      ? go[3 * f + c] * m[c]
                       : t == 7                      ? go[3 * f + c]
                                                     : 0.0;
    }
  } else {
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const bool dirichlet = (f == 0) ? (rt == 1) : (vt != 2);
#pragma unroll
      for (int c = 0; c < 3; c++)
        g[3 * f + c] = dirichlet ? dq[f] / dd.w * dir[c] : go[3 * f + c] * m[c];
    }
  }
}

// A cell value at the face, q - t . g (t the offset from the face centroid
// to the cell centroid), as three fused multiply-adds.
__device__ __forceinline__ double reconstruct(double q, const double t[3], const double* g) {
  return fma(-t[2], g[2], fma(-t[1], g[1], fma(-t[0], g[0], q)));
}

template <int EX, int EY, int EZ>
__device__ __forceinline__ double edot(const double* g) {
  // e . g for a lattice direction with components in {-1, 0, 1}
  double s = 0.0;
  if (EX) s = EX > 0 ? g[0] : -g[0];
  if (EY) s = EY > 0 ? s + g[1] : s - g[1];
  if (EZ) s = EZ > 0 ? s + g[2] : s - g[2];
  return s;
}

// e . g of a gradient inside lattice_pair. The diagonal pairs (all of e's
// components nonzero) come after the axis pairs and see each gradient as
// (gx + gy, gx - gy, gz); every diagonal e . g is then one addition, and
// rounds exactly as edot's (gx +- gy) +- gz.
template <int EX, int EY, int EZ>
__device__ __forceinline__ double gdot(const double* g) {
  if (EX == 0 || EY == 0 || EZ == 0) return edot<EX, EY, EZ>(g);
  static_assert(!(EX && EY && EZ) || EX == 1 || (EY == 1 && EZ == 1), "diagonal set");
  if (EX == 1 && EY == 1) return EZ > 0 ? g[0] + g[2] : g[0] - g[2];
  if (EX == 1) return g[1] + g[2];  // (1, -1, 1)
  return g[2] - g[1];               // (-1, 1, 1)
}

// Branch of a lattice pair from s = e . n (see lattice_pair), as two bits.
// FL = 1 (the CPU Solver, Solver.cpp:840-1274) has no dead band: s == 0 takes
// both nodes from the owner side (3).
template <int EX, int EY, int EZ, int FL>
__device__ __forceinline__ unsigned pair_side(const double n[3], double d1) {
  const double s = (EX ? (EX > 0 ? n[0] : -n[0]) : 0.0) + (EY ? (EY > 0 ? n[1] : -n[1]) : 0.0) +
                   (EZ ? (EZ > 0 ? n[2] : -n[2]) : 0.0);
  if (FL == 1) return s > 0.0 ? 1u : (s < 0.0 ? 2u : 3u);
  return s > d1 ? 1u : (s < -d1 ? 2u : 0u);
}

// One opposite pair (k, k') of D3Q15 lattice nodes, e_k' = -e_k = -e, node k
// at x_f - e dt_s (populate_lattice_macros, LBFS.cu:330-938). With s = e . n:
// s > d1 takes node k from the owner side and k' from the neighbour side,
// s < -d1 the reverse, otherwise both from the face average with averaged
// gradients (the +-0.001 dt dead band, LBFS.cu:353-354). Their equilibria
// (populate_feq, LBFS.cu:942-1038) are accumulated into the moments
// rho_I, m = sum e f and P = sum e e^T f (xx, yy, zz, xy, xz, yz). A diagonal
// pair adds the same f_k + f_k' to rho_I, P_xx, P_yy and P_zz: those pairs sum
// it once into D, which the caller adds to the four.
template <int EX, int EY, int EZ, int FL>
__device__ __forceinline__ void lattice_pair(const double si[4], const double sn[4],
                                             const double sc[4], const double g1[12],
                                             const double g2[12], int side, double dt,
                                             const double K[4], double& rhoI, double m[3],
                                             double P[6], double& D) {
  constexpr bool diag = EX != 0 && EY != 0 && EZ != 0;
  // side (pair_side): 1 if s > d1, 2 if s < -d1, 0 in the dead band. Faces are
  // sorted by their branch signature, so these branches are uniform across
  // almost every warp; each computes only its own values.
  double qa[4], qb[4];
  if (side == 1) {
#pragma unroll
    for (int f = 0; f < 4; f++) {
      qa[f] = fma(-gdot<EX, EY, EZ>(g1 + 3 * f), dt, si[f]);
      qb[f] = fma(gdot<EX, EY, EZ>(g2 + 3 * f), dt, sn[f]);
    }
  } else if (side == 2) {
#pragma unroll
    for (int f = 0; f < 4; f++) {
      qa[f] = fma(-gdot<EX, EY, EZ>(g2 + 3 * f), dt, sn[f]);
      qb[f] = fma(gdot<EX, EY, EZ>(g1 + 3 * f), dt, si[f]);
    }
  } else if (FL == 1) {  // side 3: both nodes from the owner side
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const double e = gdot<EX, EY, EZ>(g1 + 3 * f);
      qa[f] = fma(-e, dt, si[f]);
      qb[f] = fma(e, dt, si[f]);
    }
  } else {
    const double hdt = 0.5 * dt;  // e . (g1 + g2) / 2 dt
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const double e = gdot<EX, EY, EZ>(g1 + 3 * f) + gdot<EX, EY, EZ>(g2 + 3 * f);
      qa[f] = fma(-e, hdt, sc[f]);
      qb[f] = fma(e, hdt, sc[f]);
    }
  }
  // w rho (1 + 3 e.u + 4.5 (e.u)^2 / gamma - 1.5 u^2 / gamma) as
  // rho (w + 3w e.u + w c45 (e.u)^2 - w c15 u^2), K = (w, 3w, w c45, w c15)
  // with c45 = 4.5 / gamma and c15 = 1.5 / gamma (kernel constants)
  const double eua = edot<EX, EY, EZ>(qa + 1), eub = -edot<EX, EY, EZ>(qb + 1);
  const double u2a = fma(qa[3], qa[3], fma(qa[2], qa[2], qa[1] * qa[1]));
  const double u2b = fma(qb[3], qb[3], fma(qb[2], qb[2], qb[1] * qb[1]));
  const double fa = qa[0] * fma(-K[3], u2a, fma(K[2] * eua, eua, fma(K[1], eua, K[0])));
  const double fb = qb[0] * fma(-K[3], u2b, fma(K[2] * eub, eub, fma(K[1], eub, K[0])));
  const double sum = fa + fb, dif = fa - fb;
  // The axis pairs come first and each is the first to write its m and P
  // component; (1, 1, 1) is the first diagonal pair: those writes assign.
  constexpr bool first_diag = EX == 1 && EY == 1 && EZ == 1;
  if (diag) {
    if (EX) m[0] += EX > 0 ? dif : -dif;
    if (EY) m[1] += EY > 0 ? dif : -dif;
    if (EZ) m[2] += EZ > 0 ? dif : -dif;
    const double p3 = (EX * EY > 0) ? sum : -sum, p4 = (EX * EZ > 0) ? sum : -sum,
                 p5 = (EY * EZ > 0) ? sum : -sum;
    if (first_diag) {
      D = sum;
      P[3] = p3;
      P[4] = p4;
      P[5] = p5;
    } else {
      D += sum;
      P[3] += p3;
      P[4] += p4;
      P[5] += p5;
    }
  } else {
    rhoI += sum;
    if (EX) m[0] = EX > 0 ? dif : -dif;
    if (EY) m[1] = EY > 0 ? dif : -dif;
    if (EZ) m[2] = EZ > 0 ? dif : -dif;
    if (EX) P[0] = sum;
    if (EY) P[1] = sum;
    if (EZ) P[2] = sum;
  }
}

// Flux of one face (calc_face_flux, LBFS.cu:1592-1710 and
// calculate_flux_at_interface, LBFS.cu:1042-1223), in closed form:
//   rho_I = sum_k feq_k(lattice), m = sum_k e_k feq_k(lattice), u_I = m / rho_I
//   f_k = feq_k(rho_I, u_I) - tau (feq_k(rho_I, u_I) - feq_k(lattice)),
//   tau = 3 nu / (dt_s gamma)
// whose moments are, exactly (D3Q15 equilibrium moments are isotropic):
//   sum e f = m
//   sum e e^T f = (1 - tau) (rho_I / 3 I + m m^T / (rho_I gamma)) + tau P_lattice
// The face flux is (momentum, mass) = ((sum e e^T f) n, (sum e f) . n) A.
// A boundary face (neighbour > n_cells in the reference) takes both sides from
// the boundary value and all gradients from the ghost (LBFS.cu:356-401).
// The face's moments and flux from its reconstructed values (si owner side,
// sn neighbour side, sc their mean, each (rho, u, v, w)) and gradients g1, g2
// (12 doubles each; transformed in place), n the unit normal and dt the
// streaming dt.
template <int FL, bool CR>
__device__ __forceinline__ void face_flux_out(const KernelArgs& a, const int f, const int r,
                                              const double n[3],
                                              const double dt, const double si[4],
                                              const double sn[4], const double sc[4],
                                              double g1[12], double g2[12]) {
  const double pg = a.pg;
  // the seven branch decisions up front: n is not needed again until the end;
  // with the compact layout they come precomputed per record (record_sides)
  unsigned sides;
  if (CR) {  // FP64 compact layouts always carry the record sides
    sides = (unsigned)__ldg(a.frec_sides + r);
  } else {
    const double d1 = 0.001 * dt;
    sides = pair_side<1, 0, 0, FL>(n, d1) | pair_side<0, 1, 0, FL>(n, d1) << 2 |
            pair_side<0, 0, 1, FL>(n, d1) << 4 | pair_side<1, 1, 1, FL>(n, d1) << 6 |
            pair_side<1, 1, -1, FL>(n, d1) << 8 | pair_side<1, -1, 1, FL>(n, d1) << 10 |
            pair_side<-1, 1, 1, FL>(n, d1) << 12;
  }
  // centre node (k = 0): e = 0
  const double u2c = fma(sc[3], sc[3], fma(sc[2], sc[2], sc[1] * sc[1]));
  double rhoI = sc[0] * fma(-a.eq[0][3], u2c, a.eq[0][0]);
  double m[3], P[6], D;  // first written by the pairs below (see lattice_pair)
  lattice_pair<1, 0, 0, FL>(si, sn, sc, g1, g2, sides & 3, dt, a.eq[1], rhoI, m, P, D);
  lattice_pair<0, 1, 0, FL>(si, sn, sc, g1, g2, sides >> 2 & 3, dt, a.eq[1], rhoI, m, P, D);
  lattice_pair<0, 0, 1, FL>(si, sn, sc, g1, g2, sides >> 4 & 3, dt, a.eq[1], rhoI, m, P, D);
#pragma unroll
  for (int k = 0; k < 4; k++) {  // (gx, gy, gz) -> (gx + gy, gx - gy, gz), see gdot
    const double s1 = g1[3 * k] + g1[3 * k + 1], r1 = g1[3 * k] - g1[3 * k + 1];
    const double s2 = g2[3 * k] + g2[3 * k + 1], r2 = g2[3 * k] - g2[3 * k + 1];
    g1[3 * k] = s1;
    g1[3 * k + 1] = r1;
    g2[3 * k] = s2;
    g2[3 * k + 1] = r2;
  }
  lattice_pair<1, 1, 1, FL>(si, sn, sc, g1, g2, sides >> 6 & 3, dt, a.eq[2], rhoI, m, P, D);
  lattice_pair<1, 1, -1, FL>(si, sn, sc, g1, g2, sides >> 8 & 3, dt, a.eq[2], rhoI, m, P, D);
  lattice_pair<1, -1, 1, FL>(si, sn, sc, g1, g2, sides >> 10 & 3, dt, a.eq[2], rhoI, m, P, D);
  lattice_pair<-1, 1, 1, FL>(si, sn, sc, g1, g2, sides >> 12 & 3, dt, a.eq[2], rhoI, m, P, D);
  rhoI += D;
  P[0] += D;
  P[1] += D;
  P[2] += D;

  // n and A, and the relaxation factor tau = 3 nu / (dt_s gamma) as the
  // pair ((1 - tau) A, tau A), are read again here (L1 hits; per record with
  // the compact layout) rather than held in registers through the pairs.
  const d4 g0 = ld4(launder(CR ? a.frec0 : a.face0), r);
  const double nf[3] = {g0.x, g0.y, g0.z};
  const double area = g0.w;
  double omA, tA;
  if (CR) {
    const double2 w = __ldg(reinterpret_cast<const double2*>(a.frec_relax) + r);
    omA = w.x;
    tA = w.y;
  } else {
    const double tau = __ldg(static_cast<const double*>(launder(a.face2)) + 4LL * r + 3);
    omA = (1.0 - tau) * area;
    tA = tau * area;
  }
  const double mn = m[0] * nf[0] + m[1] * nf[1] + m[2] * nf[2];
  const double Pn[3] = {P[0] * nf[0] + P[3] * nf[1] + P[4] * nf[2],
                        P[3] * nf[0] + P[1] * nf[1] + P[5] * nf[2],
                        P[4] * nf[0] + P[5] * nf[1] + P[2] * nf[2]};
  const double p3 = rhoI * (1.0 / 3.0);
  const double mnr = mn / rhoI * pg;
  d4 out;
  out.x = fma(omA, fma(m[0], mnr, p3 * nf[0]), tA * Pn[0]);
  out.y = fma(omA, fma(m[1], mnr, p3 * nf[1]), tA * Pn[1]);
  out.z = fma(omA, fma(m[2], mnr, p3 * nf[2]), tA * Pn[2]);
  out.w = mn * area;
  st4(a.flux, f, out);
}

__device__ __forceinline__ int2 face_ids(const KernelArgs& a, long long f) {
  return __ldg(reinterpret_cast<const int2*>(a.face_ids) + f);
}

// CR: the face's records from the compact tables (rec = its index there).
template <int FL, bool CR>
__device__ __forceinline__ void flux_face(const KernelArgs& a, const int f, const int2 ids,
                                          const int rec) {
  const d4 f0 = CR ? ld4(a.frec0, rec) : ld4(a.face0, f);
  const d4 f1 = CR ? ld4(a.frec1, rec) : ld4(a.face1, f);
  const d4 f2 = CR ? ld4(a.frec2, rec) : ld4(a.face2, f);
  const int o = ids.x, nb = ids.y;
  const double n[3] = {f0.x, f0.y, f0.z};
  const double dt = f1.x;
  const double t1[3] = {f1.y, f1.z, f1.w}, t2[3] = {f2.x, f2.y, f2.z};

  const d4 qo = ld4(a.state, o);
  double g1[12], g2[12], si[4], sn[4], sc[4];
  load_grad(a.grad, o, g1);
  const double qov[4] = {qo.w, qo.x, qo.y, qo.z};
  bool interior = true;
  d4 qn;
  if (nb < a.C) {
    qn = ld4(a.state, nb);
    load_grad(a.grad, nb, g2);
  } else {
    const int b = nb - a.C;
    const d4 bv = ld4(a.bc0, b), tgt = ld4(a.bc1, b), dd = ld4(a.bc2, b), nm = ld4(a.bc3, b);
    const int types = (int)nm.w;
    ghost_grad<FL>(qo, g1, bv, dd, nm, types, g2);
    if (b == a.quirk_b) {
      // The reference tests neighbour > n_cells (LBFS.cu:356), so its first
      // ghost (index n_cells) goes through the interior branch with the ghost
      // state and gradient as the neighbour's.
      qn = ghost_state<FL>(qo, tgt, types);
    } else {
      interior = false;
      const int rt = types & 0xff, vt = types >> 8;
      const double bvv[4] = {bv.w, bv.x, bv.y, bv.z};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        // FL = 1 (populate_lattice_macros, Solver.cpp:862-904): rho 1 and
        // velocity 1 the value, velocity 8 (u, 0, w) of the owner, otherwise
        // extrapolated with the ghost gradient
        const bool dirichlet = (k == 0) ? (rt == 1) : (FL == 1 ? vt == 1 : vt != 2);
        const double ext = reconstruct(qov[k], t1, g2 + 3 * k);
        sc[k] = dirichlet ? bvv[k] : (FL == 1 && k > 0 && vt == 8) ? (k == 2 ? 0.0 : qov[k]) : ext;
        si[k] = sc[k];
        sn[k] = sc[k];
      }
      // FL = 0: the ghost gradient on both sides (LBFS.cu:398-401); FL = 1
      // keeps the owner's on the owner side
      if (FL == 0) {
#pragma unroll
        for (int k = 0; k < 12; k++) g1[k] = g2[k];
      }
    }
  }
  if (interior) {
    const double qnv[4] = {qn.w, qn.x, qn.y, qn.z};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      si[k] = reconstruct(qov[k], t1, g1 + 3 * k);
      sn[k] = reconstruct(qnv[k], t2, g2 + 3 * k);
      sc[k] = (si[k] + sn[k]) * 0.5;
    }
  }

  face_flux_out<FL, CR>(a, f, CR ? rec : f, n, dt, si, sn, sc, g1, g2);
}

// Persistent over the faces [f_begin, f_end) (grid stride): the
// owner/neighbour ids of a thread's next face are loaded before its current
// face is computed, so the next face's cell gathers do not wait behind a load
// of its face record. Four blocks per SM (128 registers, a few doubles spilled
// to L1) measured faster than three without spills (73 vs 75 us) and than
// five or six with more spills (102, 191 us): latency hiding wins until the
// spills take over.
template <int FL, bool CR>
__global__ void __launch_bounds__(kFluxBlock, 4) k_flux(const KernelArgs a, int f_begin,
                                                        int f_end) {
  if (halted(a)) return;
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long f = f_begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= f_end) return;
  int2 ids = face_ids(a, f);
  int rec = CR ? __ldg(a.face_rec + f) : 0;
  for (;;) {
    const long long fn = f + stride;
    const int2 next = fn < f_end ? face_ids(a, fn) : make_int2(0, 0);
    const int next_rec = (CR && fn < f_end) ? __ldg(a.face_rec + fn) : 0;
    flux_face<FL, CR>(a, (int)f, ids, rec);
    if (fn >= f_end) break;
    f = fn;
    ids = next;
    rec = next_rec;
  }
}

// ---------------------------------------------------------------------------
// flux, TMA-staged (internal faces): a producer warp gathers each tile's cell
// rows into shared memory with tile::gather4 bulk tensor copies while four
// consumer warps compute the previous tile. The consumers never wait on a
// global gather; the arithmetic per face is face_flux_out's.
// ---------------------------------------------------------------------------
constexpr int kTmaFaces = 128;  // faces per tile, one per consumer thread
constexpr int kTmaStages = 2;
constexpr int kTmaThreads = kTmaFaces + 32;
// stage layout (bytes): owner state rows, neighbour state rows, owner
// gradient rows, neighbour gradient rows
constexpr int kTmaSo = 0, kTmaSn = kTmaFaces * 32, kTmaGo = 2 * kTmaFaces * 32,
              kTmaGn = kTmaGo + kTmaFaces * 96, kTmaStageBytes = kTmaGn + kTmaFaces * 96;
// + room to align the stages to 128 bytes by hand (bulk tensor copies need it)
constexpr int kTmaSmem = kTmaStages * kTmaStageBytes + 2 * kTmaStages * 8 + 128;
constexpr int kSpinLimit = 1 << 22;  // try_wait rounds before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, int bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
// Waits for the phase of the given parity; false after kSpinLimit tries.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  for (int i = 0; i < kSpinLimit; i++) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// Rows r[0..3] (column 0) of a 2D tensor map into consecutive boxes at dst.
__device__ __forceinline__ void gather4(void* dst, const CUtensorMap* map, const int r[4],
                                        uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]),
      "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void report_fault(const KernelArgs& a) {
  atomicExch(&a.stats->fault, 1);
  atomicExch(&a.stats->halt, 1);
}

__global__ void __launch_bounds__(kTmaThreads, 3)
    k_flux_tma(const KernelArgs a, const __grid_constant__ FluxMaps maps) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  if (halted(a)) return;
  unsigned char* smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kTmaStages * kTmaStageBytes);
  uint64_t* empty = full + kTmaStages;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kTmaStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kTmaFaces / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int ntiles = (a.Fi + kTmaFaces - 1) / kTmaFaces;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == kTmaFaces / 32) {
    // producer: four faces per lane, one gather4 per row kind
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, k++) {
      const int s = k % kTmaStages;
      if (k >= kTmaStages && !mbar_wait(&empty[s], (k / kTmaStages - 1) & 1)) {
        report_fault(a);
        return;
      }
      int own[4], nbr[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int f = t * kTmaFaces + 4 * lane + j;
        const int2 id = f < a.Fi ? face_ids(a, f) : make_int2(0, 0);  // past the end: cell 0
        own[j] = id.x;
        nbr[j] = id.y;
      }
      if (lane == 0) mbar_expect_tx(&full[s], kTmaStageBytes);
      __syncwarp();
      unsigned char* st = smem + s * kTmaStageBytes;
      gather4(st + kTmaSo + 128 * lane, &maps.state, own, &full[s]);
      gather4(st + kTmaSn + 128 * lane, &maps.state, nbr, &full[s]);
      gather4(st + kTmaGo + 384 * lane, &maps.grad, own, &full[s]);
      gather4(st + kTmaGn + 384 * lane, &maps.grad, nbr, &full[s]);
    }
    return;
  }
  // consumers: one face per thread per tile
  const int c = threadIdx.x;
  int k = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, k++) {
    const int s = k % kTmaStages;
    const int f = t * kTmaFaces + c;
    const bool valid = f < a.Fi;
    d4 f0{}, f1{}, f2{};
    if (valid) {  // face records: contiguous, issued before the wait
      f0 = ld4(a.face0, f);
      f1 = ld4(a.face1, f);
      f2 = ld4(a.face2, f);
    }
    if (!mbar_wait(&full[s], (k / kTmaStages) & 1)) {
      report_fault(a);
      mbar_wait(&full[s], (k / kTmaStages) & 1);  // let copies in flight land
      return;
    }
    const unsigned char* st = smem + s * kTmaStageBytes;
    const double* so = reinterpret_cast<const double*>(st + kTmaSo) + 4 * c;
    const double* sn_ = reinterpret_cast<const double*>(st + kTmaSn) + 4 * c;
    const double* go = reinterpret_cast<const double*>(st + kTmaGo) + 12 * c;
    const double* gn = reinterpret_cast<const double*>(st + kTmaGn) + 12 * c;
    // state rows are (u, v, w, rho)
    const double qov[4] = {so[3], so[0], so[1], so[2]}, qnv[4] = {sn_[3], sn_[0], sn_[1], sn_[2]};
    double g1[12], g2[12];
#pragma unroll
    for (int i = 0; i < 12; i++) {
      g1[i] = go[i];
      g2[i] = gn[i];
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (!valid) continue;
    const double n[3] = {f0.x, f0.y, f0.z};
    const double dt = f1.x;
    const double t1[3] = {f1.y, f1.z, f1.w}, t2[3] = {f2.x, f2.y, f2.z};
    double si[4], sn[4], sc[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      si[q] = reconstruct(qov[q], t1, g1 + 3 * q);
      sn[q] = reconstruct(qnv[q], t2, g2 + 3 * q);
      sc[q] = (si[q] + sn[q]) * 0.5;
    }
    face_flux_out<0, false>(a, f, f, n, dt, si, sn, sc, g1, g2);
  }
}

// ---------------------------------------------------------------------------
// update: gather + body force + RK stage (time_integration, LBFS.cu:1457-1521)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// K2MAX: face slots the launch is specialised for (0 = any count, looped).
template <int RK, int K2MAX>
__global__ void __launch_bounds__(kBlock) k_update(const KernelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (halted(a)) return;  // uniform across the launch
  constexpr double alpha = (RK == 0 || RK == 3) ? 1.0 : 0.5;
  constexpr double beta = (RK == 0 || RK == 3) ? (1.0 / 6.0) : (1.0 / 3.0);
  double sq[4] = {0.0, 0.0, 0.0, 0.0};
  bool bad = false;
  if (i < a.C) {
    // The RK accumulators are loaded first, with the gather, so no store of
    // the stage can come between them and the flux loads.
    const d4 t0 = ld4rw(a.t0, i);
    d4 t1 = ld4rw(a.t1, i);
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    if (K2MAX > 0) {
      int e[K2MAX > 0 ? K2MAX : 1];
#pragma unroll
      for (int k = 0; k < K2MAX; k++) e[k] = (k < a.K2) ? __ldg(a.gather + (long long)k * a.C + i) : -1;
      d4 fl[K2MAX > 0 ? K2MAX : 1];
#pragma unroll
      for (int k = 0; k < K2MAX; k++)
        if (e[k] >= 0) fl[k] = ld4(a.flux, e[k] >> 1);
#pragma unroll
      for (int k = 0; k < K2MAX; k++) {
        if (e[k] < 0) continue;
        const double sg = (e[k] & 1) ? 1.0 : -1.0;
        r[0] = fma(sg, fl[k].x, r[0]);
        r[1] = fma(sg, fl[k].y, r[1]);
        r[2] = fma(sg, fl[k].z, r[2]);
        r[3] = fma(sg, fl[k].w, r[3]);
      }
    } else {
      for (int k = 0; k < a.K2; k++) {
        const int e = __ldg(a.gather + (long long)k * a.C + i);
        if (e < 0) break;
        const d4 fl = ld4(a.flux, e >> 1);
        const double sg = (e & 1) ? 1.0 : -1.0;
        r[0] = fma(sg, fl.x, r[0]);
        r[1] = fma(sg, fl.y, r[1]);
        r[2] = fma(sg, fl.z, r[2]);
        r[3] = fma(sg, fl.w, r[3]);
      }
    }
    const double iv = __ldg(static_cast<const double*>(a.inv_volume) + i);
    double R[4] = {r[0] * iv, r[1] * iv, r[2] * iv, r[3] * iv};  // u, v, w, rho
    if (a.force_x) {
      R[0] += a.force_x[i];
      R[1] += a.force_y[i];
      R[2] += a.force_z[i];
    } else {
      R[0] += a.pressure_gradient;
    }
    if (a.res_debug) st4(a.res_debug, i, d4{R[0], R[1], R[2], R[3]});
    const double dt = a.dt;
    double f1 = t0.w + R[3] * dt * alpha;
    double f2 = t0.x + R[0] * dt * alpha;
    double f3 = t0.y + R[1] * dt * alpha;
    double f4 = t0.z + R[2] * dt * alpha;
    t1.w = t1.w + dt * beta * R[3];
    t1.x = t1.x + dt * beta * R[0];
    t1.y = t1.y + dt * beta * R[1];
    t1.z = t1.z + dt * beta * R[2];
    d4 q;
    if (RK == 3) {
      q = d4{t1.x / t1.w, t1.y / t1.w, t1.z / t1.w, t1.w};
      st4(a.t0, i, t1);  // the next step starts from t1 (Solver_gpu.cu:671)
      sq[0] = R[3] * R[3];
      sq[1] = R[0] * R[0];
      sq[2] = R[1] * R[1];
      sq[3] = R[2] * R[2];
      bad = !(t1.w <= 1000.0);  // the CPU solver's divergence test, Solver.cpp:448-493
    } else {
      q = d4{f2 / f1, f3 / f1, f4 / f1, f1};
    }
    st4(a.t1, i, t1);
    st4(a.state, i, q);
    // The last reader of this step's force resets it for the IBM. The stores
    // come after every load of the stage: placed before the t0/t1 loads they
    // would hold those loads back (the pointers may alias).
    if (RK == 3 && a.force_x) {
      a.force_x[i] = a.pressure_gradient;
      a.force_y[i] = 0.0;
      a.force_z[i] = 0.0;
    }
  }
  if (RK != 3) return;

  // Per-block squared-residual sums (warp shuffle, then the block's warps in
  // order); k_finish reduces them.
  __shared__ double red[kBlock / 32][4];
  __shared__ int any_bad;
  if (threadIdx.x == 0) any_bad = 0;
  __syncthreads();
  if (bad) atomicOr(&any_bad, 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const double v = warp_sum(sq[c]);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int w = 0; w < kBlock / 32; w++) v += red[w][threadIdx.x];
    a.partial[4LL * blockIdx.x + threadIdx.x] = v;
  }
  if (threadIdx.x == 0 && any_bad) a.stats->diverged = 1;
}

// One block after the last stage: sums the per-block partials in a fixed
// order, forms the rms norms of l2_norm_rms_moukallad (residuals.cpp:95-113)
// and max_error (:139-147), records the step and tests convergence
// (Solver_gpu.cu:870); a converged or diverged context halts.
__global__ void __launch_bounds__(kFinishBlock) k_finish(const KernelArgs a) {
  if (halted(a)) return;
  __shared__ double red[kFinishBlock / 32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
  for (int b = threadIdx.x; b < a.nblk_update; b += kFinishBlock) {
    const double2 p0 = __ldg(reinterpret_cast<const double2*>(a.partial + 4LL * b));
    const double2 p1 = __ldg(reinterpret_cast<const double2*>(a.partial + 4LL * b) + 1);
    v[0] += p0.x;
    v[1] += p0.y;
    v[2] += p1.x;
    v[3] += p1.y;
  }
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const double w = warp_sum(v[c]);
    if (lane == 0) red[warp][c] = w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[4];
    for (int c = 0; c < 4; c++) {
      tot[c] = 0.0;
      for (int w = 0; w < kFinishBlock / 32; w++) tot[c] += red[w][c];
    }
    DevStats* st = a.stats;
    const double nC = (double)a.C;
    const double rho_rms = sqrt(tot[0] / nC) * a.inv_ref_rho;
    const double u_rms = sqrt(tot[1] / nC) * a.inv_ref_mom;
    const double v_rms = sqrt(tot[2] / nC) * a.inv_ref_mom;
    const double w_rms = sqrt(tot[3] / nC) * a.inv_ref_mom;
    const double me = fmax(fmax(w_rms, u_rms), v_rms);  // residuals::max_error
    const long long t = st->steps;
    double* h = st->history[t % kHistoryCap];
    h[0] = (double)t;
    h[1] = me;
    h[2] = rho_rms;
    h[3] = u_rms;
    h[4] = v_rms;
    h[5] = w_rms;
    for (int c = 0; c < 6; c++) st->last[c] = h[c];
    st->steps = t + 1;
    if (!(me == me) || !(rho_rms == rho_rms)) st->diverged = 1;
    if (me < a.tolerance) {
      st->converged = 1;
      st->converged_step = t;
    }
    if (st->converged || st->diverged) st->halt = 1;
  }
}

// Seeds the RK accumulator from the state (Solver_gpu.cu:664): t0 = t1 = q.
// The reference seeds the velocity state although the stages treat t0/t1 as
// (rho u, rho v, rho w, rho); with conserved = true (warm starts, no reference
// counterpart) the accumulators get the conserved variables instead.
template <bool CONSERVED>
__global__ void k_seed(const KernelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.C) return;
  d4 q = ld4(a.state, i);
  if (CONSERVED) q = d4{q.w * q.x, q.w * q.y, q.w * q.z, q.w};
  st4(a.t0, i, q);
  st4(a.t1, i, q);
}

// ---------------------------------------------------------------------------
// IBM (immersed_boundary_method.cu:13-90, 161-190, 244-295, 299-375), once
// per time step before the RK stages.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void stencil_origin(const KernelArgs& a, const double x[3],
                                               double r[3], int lo[3]) {
  r[0] = (x[0] - a.origin[0]) / a.ibm_dx;
  r[1] = fabs((x[1] - a.origin[1]) / a.ibm_dx);
  r[2] = fabs((x[2] - a.origin[2]) / a.ibm_dx);
#pragma unroll
  for (int c = 0; c < 3; c++) lo[c] = (int)round(r[c]) - 1;
}

// Eight threads per node, one per cell of its 2 x 2 x 2 stencil: each loads
// its cell's state, the node's velocity is the sum over the eight (xor
// butterfly, so every lane holds the same bits), every lane advances the node
// and forms its force, and the warp spreads its lanes' forces with one FP64
// atomic per distinct cell and component (spread_aggregated; nodes in the
// spatial order ibm_order). Lane 0 of a node writes the node's arrays.
__global__ void __launch_bounds__(kIbmBlock) k_ibm(const KernelArgs a) {
  if (halted(a)) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int slot = t >> 3, sub = t & 7;
  const bool active = slot < a.N;
  const int nd = active ? __ldg(a.ibm_order + slot) : 0;
  const int xc = a.ibm_xc, yc = a.ibm_yc;
  double x[3] = {0.0, 0.0, 0.0}, r[3] = {0.0, 0.0, 0.0};
  int lo[3] = {0, 0, 0};
  if (active) {
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = a.node_x[3 * nd + c];
    stencil_origin(a, x, r, lo);
  }
  const int di = sub & 1, dj = (sub >> 1) & 1, dk = sub >> 2;
  double v[3] = {0.0, 0.0, 0.0};
  {
    const int ii = lo[0] + di, jj = lo[1] + dj, kk = lo[2] + dk;
    const long long cell = (long long)ii + (long long)jj * xc + (long long)kk * yc * xc;
    if (active && cell < a.C && cell >= 0) {  // the reference's linear-index check
      const double wx = 1 - fabs(ii + 0.5 - r[0]);
      const double wy = 1 - fabs(jj + 0.5 - r[1]);
      const double wz = 1 - fabs(kk + 0.5 - r[2]);
      const d4 q = ld4(a.state, a.ibm_map[cell]);
      v[0] = q.x * wx * wy * wz * a.ibm_inv_dx3;
      v[1] = q.y * wx * wy * wz * a.ibm_inv_dx3;
      v[2] = q.z * wx * wy * wz * a.ibm_inv_dx3;
    }
  }
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 1; o < 8; o <<= 1)
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] += __shfl_xor_sync(full, v[c], o);
  const unsigned act = __ballot_sync(full, active);
  if (!active) return;
  double fn[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    x[c] = a.node_x0[3 * nd + c] + v[c] * a.dt;
    fn[c] = -a.ibm_area_k * (x[c] - a.node_ref[3 * nd + c]);
  }
  if (sub == 0) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      a.node_x[3 * nd + c] = x[c];
      a.node_x0[3 * nd + c] = x[c];
      a.node_vel[3 * nd + c] = v[c];
      a.node_force[3 * nd + c] = fn[c];
    }
  }
  stencil_origin(a, x, r, lo);
  const int ii = lo[0] + di, jj = lo[1] + dj, kk = lo[2] + dk;
  const long long cell = (long long)ii + (long long)jj * xc + (long long)kk * yc * xc;
  int target = -1;
  double f[3] = {0.0, 0.0, 0.0};
  if (cell < a.C && cell >= 0) {
    const double wx = 1 - fabs(ii + 0.5 - r[0]);
    const double wy = 1 - fabs(jj + 0.5 - r[1]);
    const double wz = 1 - fabs(kk + 0.5 - r[2]);
    target = a.ibm_map[cell];
#pragma unroll
    for (int c = 0; c < 3; c++) f[c] = fn[c] * wx * wy * wz * a.ibm_inv_dx3;
  }
  spread_aggregated(act, target, f, a.force_x, a.force_y, a.force_z);
}

// ---------------------------------------------------------------------------
// Wall forces of post_processing::cylinder_post_processing
// (post_processing.cpp:50-173) over the listed boundary faces (internal bc
// indices), from the current state and gradients (the reference calls it
// after update_unstructured_bcs and Get_LS_Gradients on the host, so the
// ghost gradients follow the host rules of gradients.cpp:441-463 and 592-645:
// Dirichlet velocity 2 (u_b - u_o) / |d| times the face normal, Neumann the
// owner's gradient times (1 - n)). Per face: p = rho_o gamma / 3,
//   drag += ((p - nu gamma du/dx) n_x - nu gamma du/dy n_y) A
//   lift += (nu gamma dv/dx n_x - (p - nu gamma dv/dy) n_y) A.
// One block; the partial sums are added in a fixed order. out[2] = {drag, lift}.
// ---------------------------------------------------------------------------
constexpr int kWallBlock = 1024;

__global__ void __launch_bounds__(kWallBlock) k_wall_forces(const KernelArgs a, const int* walls,
                                                            int n, int fp32, double visc_g,
                                                            double gamma, double* out) {
  __shared__ double red[kWallBlock / 32][2];
  double dr = 0.0, li = 0.0;
  const long long Fi = (long long)a.F - a.B;  // boundary face of bc b: Fi + b
  for (int k = threadIdx.x; k < n; k += kWallBlock) {
    const int b = walls[k];
    const long long f = Fi + b;
    const int o = a.face_ids[2 * f];
    double nx, ny, area, rho, uo, vo, ub, vb, dmag, gux, guy, gvx, gvy;
    int types;
    if (fp32) {  // deviation units: velocity / U, rho - rho0
      const float4 f0 = reinterpret_cast<const float4*>(a.face0)[f];
      const float4 q = reinterpret_cast<const float4*>(a.state)[o];
      const float4 bv = reinterpret_cast<const float4*>(a.bc0)[b];
      const float4 dd = reinterpret_cast<const float4*>(a.bc2)[b];
      const float4 nm = reinterpret_cast<const float4*>(a.bc3)[b];
      const float4 g0 = reinterpret_cast<const float4*>(a.grad)[3LL * o];
      const float4 g1 = reinterpret_cast<const float4*>(a.grad)[3LL * o + 1];
      const double U = a.uref;
      nx = f0.x; ny = f0.y; area = f0.w;
      rho = a.rho0 + q.w;
      uo = U * q.x; vo = U * q.y; ub = U * bv.x; vb = U * bv.y;
      dmag = dd.w;
      types = (int)nm.w;
      gux = U * g0.w; guy = U * g1.x; gvx = U * g1.z; gvy = U * g1.w;
    } else {
      const d4 f0 = ld4(a.face0, f), q = ld4(a.state, o), bv = ld4(a.bc0, b), dd = ld4(a.bc2, b),
               nm = ld4(a.bc3, b), g0 = ld4(a.grad, 3LL * o), g1 = ld4(a.grad, 3LL * o + 1);
      nx = f0.x; ny = f0.y; area = f0.w;
      rho = q.w;
      uo = q.x; vo = q.y; ub = bv.x; vb = bv.y;
      dmag = dd.w;
      types = (int)nm.w;
      gux = g0.w; guy = g1.x; gvx = g1.z; gvy = g1.w;
    }
    double ux, uy, vx, vy;
    if ((types >> 8) == 1) {  // Dirichlet velocity: get_ghost_grads
      const double du = 2 * (ub - uo), dv = 2 * (vb - vo);
      ux = du / dmag * nx;
      uy = du / dmag * ny;
      vx = dv / dmag * nx;
      vy = dv / dmag * ny;
    } else {  // Neumann velocity (the host checked the type)
      ux = gux * (1 - nx);
      uy = guy * (1 - ny);
      vx = gvx * (1 - nx);
      vy = gvy * (1 - ny);
    }
    const double p = rho / 3.0 * gamma;
    dr = dr + ((p - visc_g * ux) * nx - visc_g * uy * ny) * area;
    li = li + (visc_g * vx * nx - (p - visc_g * vy) * ny) * area;
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    dr += __shfl_down_sync(0xffffffffu, dr, s);
    li += __shfl_down_sync(0xffffffffu, li, s);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5][0] = dr;
    red[threadIdx.x >> 5][1] = li;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double d = 0.0, l = 0.0;
    for (int w = 0; w < kWallBlock / 32; w++) {
      d += red[w][0];
      l += red[w][1];
    }
    out[0] = d;
    out[1] = l;
  }
}

inline int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

// The seven branch decisions of each unique face record of the compact
// layout, as face_flux_out computes them.
template <int FL>
__global__ void k_record_sides(const void* frec0, const void* frec1, const void* frec2, int n,
                               int32_t* out, double2* relax) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const d4 f0 = ld4(frec0, r), f1 = ld4(frec1, r), f2 = ld4(frec2, r);
    // the pair face_flux_out forms per face without the compact layout
    relax[r] = make_double2((1.0 - f2.w) * f0.w, f2.w * f0.w);
    const double nv[3] = {f0.x, f0.y, f0.z};
    const double d1 = 0.001 * f1.x;
    out[r] = (int32_t)(pair_side<1, 0, 0, FL>(nv, d1) | pair_side<0, 1, 0, FL>(nv, d1) << 2 |
                       pair_side<0, 0, 1, FL>(nv, d1) << 4 | pair_side<1, 1, 1, FL>(nv, d1) << 6 |
                       pair_side<1, 1, -1, FL>(nv, d1) << 8 |
                       pair_side<1, -1, 1, FL>(nv, d1) << 10 |
                       pair_side<-1, 1, 1, FL>(nv, d1) << 12);
  }
}

}  // namespace

void launch_record_sides(const void* frec0, const void* frec1, const void* frec2, int n,
                         int flavour, int32_t* out, double* relax, cudaStream_t s) {
  if (n <= 0) return;
  const int nb = (int)blocks_for(n, kBlock);
  double2* rl = reinterpret_cast<double2*>(relax);
  if (flavour == PLFBS_FLAVOUR_CPU_SOLVER)
    k_record_sides<1><<<nb, kBlock, 0, s>>>(frec0, frec1, frec2, n, out, rl);
  else
    k_record_sides<0><<<nb, kBlock, 0, s>>>(frec0, frec1, frec2, n, out, rl);
}

void launch_gradient(const KernelArgs& a, int precision, cudaStream_t s) {
  if (precision == PLFBS_FP32_DEVIATION) return launch_gradient32(a, s);
  const int nb = blocks_for(a.C, kBlock);
  const bool cw = a.compact && a.wtab;
  if (a.flavour == PLFBS_FLAVOUR_CPU_SOLVER) {
    if (cw)
      k_gradient<1, true><<<nb, kBlock, 0, s>>>(a);
    else
      k_gradient<1, false><<<nb, kBlock, 0, s>>>(a);
  } else {
    if (cw)
      k_gradient<0, true><<<nb, kBlock, 0, s>>>(a);
    else
      k_gradient<0, false><<<nb, kBlock, 0, s>>>(a);
  }
}
int prepare_flux_tma() {
  static std::atomic<int> tma_resident[kMaxDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = 0;
  int r = tma_resident[dev].load(std::memory_order_relaxed);
  if (r <= 0) {
    int per_sm = 0, sms = 0;
    cudaFuncSetAttribute(k_flux_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaSmem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flux_tma, kTmaThreads, kTmaSmem) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        per_sm <= 0 || sms <= 0) {
      per_sm = 1;
      sms = 148;
    }
    r = per_sm * sms;
    tma_resident[dev].store(r, std::memory_order_relaxed);
  }
  return r;
}

void launch_flux(const KernelArgs& a, int precision, cudaStream_t s) {
  if (precision == PLFBS_FP32_DEVIATION) return launch_flux32(a, s);
  static std::atomic<int> resident[kMaxDevices];
  const bool cr = a.compact && a.face_rec;
  if (a.flavour == PLFBS_FLAVOUR_CPU_SOLVER) {
    static std::atomic<int> cpu_resident[kMaxDevices], cpu_cr_resident[kMaxDevices];
    if (cr)
      k_flux<1, true><<<persistent_blocks(k_flux<1, true>, kFluxBlock, a.F, cpu_cr_resident),
                        kFluxBlock, 0, s>>>(a, 0, a.F);
    else
      k_flux<1, false><<<persistent_blocks(k_flux<1, false>, kFluxBlock, a.F, cpu_resident),
                         kFluxBlock, 0, s>>>(a, 0, a.F);
    return;
  }
  if (!a.flux_maps || a.Fi == 0) {
    static std::atomic<int> cr_resident[kMaxDevices];
    if (cr)
      k_flux<0, true><<<persistent_blocks(k_flux<0, true>, kFluxBlock, a.F, cr_resident),
                        kFluxBlock, 0, s>>>(a, 0, a.F);
    else
      k_flux<0, false><<<persistent_blocks(k_flux<0, false>, kFluxBlock, a.F, resident),
                         kFluxBlock, 0, s>>>(a, 0, a.F);
    return;
  }
  // internal faces through the TMA-staged kernel, boundary faces (the last
  // F - Fi of the face order) through the per-thread one
  const int r = prepare_flux_tma();
  const int tiles = (a.Fi + kTmaFaces - 1) / kTmaFaces;
  k_flux_tma<<<tiles < r ? tiles : r, kTmaThreads, kTmaSmem, s>>>(a, *a.flux_maps);
  if (a.F > a.Fi) {
    static std::atomic<int> bnd_resident[kMaxDevices];
    k_flux<0, false><<<persistent_blocks(k_flux<0, false>, kFluxBlock, a.F - a.Fi, bnd_resident),
                       kFluxBlock, 0, s>>>(a, a.Fi, a.F);
  }
}
template <int RK>
static void launch_update_rk(const KernelArgs& a, int nb, cudaStream_t s) {
  if (a.K2 <= 4)
    k_update<RK, 4><<<nb, kBlock, 0, s>>>(a);
  else if (a.K2 <= 6)
    k_update<RK, 6><<<nb, kBlock, 0, s>>>(a);
  else if (a.K2 <= 8)
    k_update<RK, 8><<<nb, kBlock, 0, s>>>(a);
  else
    k_update<RK, 0><<<nb, kBlock, 0, s>>>(a);
}
void launch_update(const KernelArgs& a, int precision, int rk, cudaStream_t s, bool finish) {
  if (precision == PLFBS_FP32_DEVIATION) return launch_update32(a, rk, s, finish);
  const int nb = blocks_for(a.C, kBlock);
  switch (rk) {
    case 0: launch_update_rk<0>(a, nb, s); break;
    case 1: launch_update_rk<1>(a, nb, s); break;
    case 2: launch_update_rk<2>(a, nb, s); break;
    default:
      launch_update_rk<3>(a, nb, s);
      if (finish) k_finish<<<1, kFinishBlock, 0, s>>>(a);
      break;
  }
}
void launch_finish(const KernelArgs& a, int precision, cudaStream_t s) {
  if (precision == PLFBS_FP32_DEVIATION) return launch_finish32(a, s);
  k_finish<<<1, kFinishBlock, 0, s>>>(a);
}
void launch_seed(const KernelArgs& a, int precision, bool conserved, cudaStream_t s) {
  if (precision == PLFBS_FP32_DEVIATION) return launch_seed32(a, conserved, s);
  if (conserved)
    k_seed<true><<<blocks_for(a.C, kBlock), kBlock, 0, s>>>(a);
  else
    k_seed<false><<<blocks_for(a.C, kBlock), kBlock, 0, s>>>(a);
}
void launch_ibm(const KernelArgs& a, int precision, cudaStream_t s) {
  if (precision == PLFBS_FP32_DEVIATION) return launch_ibm32(a, s);
  if (a.N > 0) k_ibm<<<blocks_for(8LL * a.N, kIbmBlock), kIbmBlock, 0, s>>>(a);
}

void launch_wall_forces(const KernelArgs& a, int precision, const int* walls, int n,
                        double visc_gamma, double gamma, double* out, cudaStream_t s) {
  k_wall_forces<<<1, kWallBlock, 0, s>>>(a, walls, n, precision == PLFBS_FP32_DEVIATION ? 1 : 0,
                                          visc_gamma, gamma, out);
}

}  // namespace plfbs
