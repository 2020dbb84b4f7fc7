// sm_100a kernels of the FP32 deviation form (PLFBS_FP32_DEVIATION).
//
// Same step structure as kernels.cu (gradient -> flux -> gather+RK per stage,
// IBM once per step), with state, gradients, fluxes, geometry and weights in
// FP32 and the variables shifted and scaled so that FP32 keeps the precision
// the residual needs:
//   state  (u/U, v/U, w/U, rho - rho0)
//   t0,t1  the RK accumulators in the same units (momentum / U, rho - rho0)
//   flux   (momentum flux / U, mass flux) with the constant rho0/3 n A part of
//          the momentum flux removed: it telescopes to zero over every closed
//          cell (sum_f n_f A_f = 0), so only deviations are carried.
// The equilibrium at a lattice node is split the same way:
//   feq = w rho0 + w [drho + rho U phi],
//   phi = 3 e.u' + 4.5 U (e.u')^2 / gamma - 1.5 U |u'|^2 / gamma,  u' = u/U,
// and the w rho0 part, whose moments are (rho0, 0, rho0/3 I), is left out of
// every sum. The residual norms are reduced in FP64, the Lagrangian node
// positions and forces stay FP64 (forces are spread as FP32 / U).
#include <cuda_runtime.h>

#include <cstdint>

#include "ibm_spread.cuh"
#include "plfbs_internal.hpp"

namespace plfbs {
namespace {

struct __align__(16) f4 {
  float x, y, z, w;
};

__device__ __forceinline__ f4 ldf(const void* base, long long i) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(base) + i);
  return f4{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ f4 ldf_rw(const void* base, long long i) {
  const float4 v = reinterpret_cast<const float4*>(base)[i];
  return f4{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ void stf(void* base, long long i, const f4& v) {
  reinterpret_cast<float4*>(base)[i] = make_float4(v.x, v.y, v.z, v.w);
}

// Whether the context has converged or diverged. One thread per block reads
// the flag; every thread of the block must call this (it synchronises).
__device__ __forceinline__ bool halted(const KernelArgs& a) {
  __shared__ int h;
  if (threadIdx.x == 0) h = *(volatile const int*)&a.stats->halt;
  __syncthreads();
  return h != 0;
}

// Ghost state in deviation units (the same affine rules as the FP64 path).
__device__ __forceinline__ f4 ghost_state32(const f4& q, const f4& tgt, int types) {
  const int rt = types & 0xff, vt = types >> 8;
  f4 g;
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

// Gradient layout: 3 x float4 per cell: (rx ry rz ux)(uy uz vx vy)(vz wx wy wz).
// Stencil slots as in k_gradient: neighbour ids first, then the slots.
template <bool CW>
__device__ __forceinline__ void gradient_slot32(const KernelArgs& a, long long s, int j,
                                                const f4& qi, float g[12], const float* wrow) {
  f4 qj;
  if (j < a.C) {
    qj = ldf(a.state, j);
  } else {
    const int b = j - a.C;
    const f4 tgt = ldf(a.bc1, b);
    const int types = (int)__ldg(reinterpret_cast<const float*>(a.bc3) + 4LL * b + 3);
    qj = ghost_state32(qi, tgt, types);
    stf(a.state, j, qj);
  }
  // CW: the cell's weight set from the compact table (wrow = its slot's triple)
  const float w[3] = {CW ? __ldg(wrow) : __ldg(static_cast<const float*>(a.st_wx) + s),
                      CW ? __ldg(wrow + 1) : __ldg(static_cast<const float*>(a.st_wy) + s),
                      CW ? __ldg(wrow + 2) : __ldg(static_cast<const float*>(a.st_wz) + s)};
  const float d[4] = {qj.w - qi.w, qj.x - qi.x, qj.y - qi.y, qj.z - qi.z};
#pragma unroll
  for (int f = 0; f < 4; f++)
#pragma unroll
    for (int c = 0; c < 3; c++) g[3 * f + c] = fmaf(w[c], d[f], g[3 * f + c]);
}

template <bool CW>
__global__ void __launch_bounds__(kBlock) k_gradient32(const KernelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (halted(a)) return;
  if (i >= a.C) return;
  const f4 qi = ldf(a.state, i);
  const float* wset =
      CW ? static_cast<const float*>(a.wtab) + (size_t)__ldg(a.cell_wset + i) * a.K * 3 : nullptr;
  float g[12];
#pragma unroll
  for (int k = 0; k < 12; k++) g[k] = 0.0f;
  constexpr int kUnroll = 8;
  if (a.K <= kUnroll) {
    int jj[kUnroll];
#pragma unroll
    for (int k = 0; k < kUnroll; k++) jj[k] = k < a.K ? __ldg(a.st_nbr + (long long)k * a.C + i) : -1;
#pragma unroll
    for (int k = 0; k < kUnroll; k++)
      if (jj[k] >= 0)
        gradient_slot32<CW>(a, (long long)k * a.C + i, jj[k], qi, g, CW ? wset + 3 * k : nullptr);
  } else {
    for (int k = 0; k < a.K; k++) {
      const long long s = (long long)k * a.C + i;
      const int j = __ldg(a.st_nbr + s);
      if (j < 0) break;
      gradient_slot32<CW>(a, s, j, qi, g, CW ? wset + 3 * k : nullptr);
    }
  }
  stf(a.grad, 3LL * i + 0, f4{g[0], g[1], g[2], g[3]});
  stf(a.grad, 3LL * i + 1, f4{g[4], g[5], g[6], g[7]});
  stf(a.grad, 3LL * i + 2, f4{g[8], g[9], g[10], g[11]});
}

__device__ __forceinline__ void load_grad32(const void* base, int c, float g[12]) {
  const f4 a0 = ldf(base, 3LL * c), a1 = ldf(base, 3LL * c + 1), a2 = ldf(base, 3LL * c + 2);
  g[0] = a0.x; g[1] = a0.y; g[2] = a0.z; g[3] = a0.w;
  g[4] = a1.x; g[5] = a1.y; g[6] = a1.z; g[7] = a1.w;
  g[8] = a2.x; g[9] = a2.y; g[10] = a2.z; g[11] = a2.w;
}

__device__ __forceinline__ void ghost_grad32(const f4& q, const float go[12], const f4& bv,
                                             const f4& dd, const f4& nm, int types, float g[12]) {
  const int rt = types & 0xff, vt = types >> 8;
  const float dir[3] = {dd.x, dd.y, dd.z}, m[3] = {nm.x, nm.y, nm.z};
  const float dq[4] = {2.0f * (bv.w - q.w), 2.0f * (bv.x - q.x), 2.0f * (bv.y - q.y),
                       2.0f * (bv.z - q.z)};
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const bool dirichlet = (f == 0) ? (rt == 1) : (vt != 2);
#pragma unroll
    for (int c = 0; c < 3; c++)
      g[3 * f + c] = dirichlet ? dq[f] / dd.w * dir[c] : go[3 * f + c] * m[c];
  }
}

template <int EX, int EY, int EZ>
__device__ __forceinline__ float edotf(const float* g) {
  float s = 0.0f;
  if (EX) s = EX > 0 ? g[0] : -g[0];
  if (EY) s = EY > 0 ? s + g[1] : s - g[1];
  if (EZ) s = EZ > 0 ? s + g[2] : s - g[2];
  return s;
}

// e . g of a gradient; diagonal pairs see (gx + gy, gx - gy, gz) (as gdot in
// kernels.cu).
template <int EX, int EY, int EZ>
__device__ __forceinline__ float gdotf(const float* g) {
  if (EX == 0 || EY == 0 || EZ == 0) return edotf<EX, EY, EZ>(g);
  if (EX == 1 && EY == 1) return EZ > 0 ? g[0] + g[2] : g[0] - g[2];
  if (EX == 1) return g[1] + g[2];  // (1, -1, 1)
  return g[2] - g[1];               // (-1, 1, 1)
}

// Consts shared by the lattice pairs of one face.
struct PairConst {
  float d1, dt, hdt;
  float rho0, U, c45u, c15u;  // c45u = 4.5 U / gamma, c15u = 1.5 U / gamma
  float u3, c45uu, c15uu;     // 3 U, U c45u, U c15u
};

// Deviation part of the equilibrium at one node: w [drho + rho U phi].
__device__ __forceinline__ float feq_dev(const PairConst& k, float wgt, const float q[4],
                                         float eu) {
  const float u2 = fmaf(q[3], q[3], fmaf(q[2], q[2], q[1] * q[1]));
  // U phi = U (3 eu + c45u eu^2 - c15u u2), with U folded into the constants
  const float uphi = fmaf(eu, fmaf(k.c45uu, eu, k.u3), -k.c15uu * u2);
  return wgt * fmaf(k.rho0 + q[0], uphi, q[0]);
}

template <int EX, int EY, int EZ>
__device__ __forceinline__ void lattice_pair32(const float si[4], const float sn[4],
                                               const float sc[4], const float g1[12],
                                               const float g2[12], const float n[3],
                                               const PairConst& k, float wgt, float& drhoI,
                                               float m[3], float P[6], float& D) {
  constexpr bool diag = EX != 0 && EY != 0 && EZ != 0;
  const float s = (EX ? (EX > 0 ? n[0] : -n[0]) : 0.0f) + (EY ? (EY > 0 ? n[1] : -n[1]) : 0.0f) +
                  (EZ ? (EZ > 0 ? n[2] : -n[2]) : 0.0f);
  float qa[4], qb[4];
  if (s > k.d1) {
#pragma unroll
    for (int f = 0; f < 4; f++) {
      qa[f] = fmaf(-gdotf<EX, EY, EZ>(g1 + 3 * f), k.dt, si[f]);
      qb[f] = fmaf(gdotf<EX, EY, EZ>(g2 + 3 * f), k.dt, sn[f]);
    }
  } else if (s < -k.d1) {
#pragma unroll
    for (int f = 0; f < 4; f++) {
      qa[f] = fmaf(-gdotf<EX, EY, EZ>(g2 + 3 * f), k.dt, sn[f]);
      qb[f] = fmaf(gdotf<EX, EY, EZ>(g1 + 3 * f), k.dt, si[f]);
    }
  } else {
#pragma unroll
    for (int f = 0; f < 4; f++) {
      const float e = gdotf<EX, EY, EZ>(g1 + 3 * f) + gdotf<EX, EY, EZ>(g2 + 3 * f);
      qa[f] = fmaf(-e, k.hdt, sc[f]);
      qb[f] = fmaf(e, k.hdt, sc[f]);
    }
  }
  const float fa = feq_dev(k, wgt, qa, edotf<EX, EY, EZ>(qa + 1));
  const float fb = feq_dev(k, wgt, qb, -edotf<EX, EY, EZ>(qb + 1));
  const float sum = fa + fb, dif = fa - fb;
  if (EX) m[0] += EX > 0 ? dif : -dif;
  if (EY) m[1] += EY > 0 ? dif : -dif;
  if (EZ) m[2] += EZ > 0 ? dif : -dif;
  if (diag) {
    D += sum;
  } else {
    drhoI += sum;
    if (EX) P[0] += sum;
    if (EY) P[1] += sum;
    if (EZ) P[2] += sum;
  }
  if (EX && EY) P[3] += (EX * EY > 0) ? sum : -sum;
  if (EX && EZ) P[4] += (EX * EZ > 0) ? sum : -sum;
  if (EY && EZ) P[5] += (EY * EZ > 0) ? sum : -sum;
}

// Face flux in deviation form (see the file comment); the same branches and
// boundary handling as k_flux in kernels.cu.
// CR: the face's records from the compact tables (rec = its index there).
template <bool CR>
__device__ __forceinline__ void flux_face32(const KernelArgs& a, const int f, const int2 ids,
                                            const int rec) {
  const f4 f0 = CR ? ldf(a.frec0, rec) : ldf(a.face0, f);
  const f4 f1 = CR ? ldf(a.frec1, rec) : ldf(a.face1, f);
  const f4 f2 = CR ? ldf(a.frec2, rec) : ldf(a.face2, f);
  const int o = ids.x, nb = ids.y;
  const float n[3] = {f0.x, f0.y, f0.z};
  const float area = f0.w, dt = f1.x;
  const float t1[3] = {f1.y, f1.z, f1.w}, t2[3] = {f2.x, f2.y, f2.z};
  const f4 qo = ldf(a.state, o);
  float g1[12], g2[12], si[4], sn[4], sc[4];
  load_grad32(a.grad, o, g1);
  const float qov[4] = {qo.w, qo.x, qo.y, qo.z};
  bool interior = true;
  f4 qn;
  if (nb < a.C) {
    qn = ldf(a.state, nb);
    load_grad32(a.grad, nb, g2);
  } else {
    const int b = nb - a.C;
    const f4 bv = ldf(a.bc0, b), tgt = ldf(a.bc1, b), dd = ldf(a.bc2, b), nm = ldf(a.bc3, b);
    const int types = (int)nm.w;
    ghost_grad32(qo, g1, bv, dd, nm, types, g2);
    if (b == a.quirk_b) {
      qn = ghost_state32(qo, tgt, types);  // interior branch, LBFS.cu:356
    } else {
      interior = false;
      const int rt = types & 0xff, vt = types >> 8;
      const float bvv[4] = {bv.w, bv.x, bv.y, bv.z};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const bool dirichlet = (k == 0) ? (rt == 1) : (vt != 2);
        sc[k] = dirichlet ? bvv[k]
                          : qov[k] - (t1[0] * g2[3 * k] + t1[1] * g2[3 * k + 1] +
                                      t1[2] * g2[3 * k + 2]);
        si[k] = sc[k];
        sn[k] = sc[k];
      }
#pragma unroll
      for (int k = 0; k < 12; k++) g1[k] = g2[k];
    }
  }
  if (interior) {
    const float qnv[4] = {qn.w, qn.x, qn.y, qn.z};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      si[k] = qov[k] - (t1[0] * g1[3 * k] + t1[1] * g1[3 * k + 1] + t1[2] * g1[3 * k + 2]);
      sn[k] = qnv[k] - (t2[0] * g2[3 * k] + t2[1] * g2[3 * k + 1] + t2[2] * g2[3 * k + 2]);
      sc[k] = (si[k] + sn[k]) * 0.5f;
    }
  }
  PairConst kc;
  kc.d1 = 0.001f * dt;
  kc.dt = dt;
  kc.hdt = 0.5f * dt;
  kc.rho0 = a.rho0f;
  kc.U = (float)a.uref;
  const float pg = (float)a.pg;
  kc.c45u = 4.5f * kc.U * pg;
  kc.c15u = 1.5f * kc.U * pg;
  kc.u3 = 3.0f * kc.U;
  kc.c45uu = kc.U * kc.c45u;
  kc.c15uu = kc.U * kc.c15u;
  const float w0 = 2.0f / 9.0f, w1 = 1.0f / 9.0f, w7 = 1.0f / 72.0f;
  // centre node: e = 0
  const float u2c = fmaf(sc[3], sc[3], fmaf(sc[2], sc[2], sc[1] * sc[1]));
  float drhoI = w0 * fmaf(kc.rho0 + sc[0], kc.U * (-kc.c15u * u2c), sc[0]);
  float m[3] = {0.0f, 0.0f, 0.0f};
  float P[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  float D = 0.0f;
  lattice_pair32<1, 0, 0>(si, sn, sc, g1, g2, n, kc, w1, drhoI, m, P, D);
  lattice_pair32<0, 1, 0>(si, sn, sc, g1, g2, n, kc, w1, drhoI, m, P, D);
  lattice_pair32<0, 0, 1>(si, sn, sc, g1, g2, n, kc, w1, drhoI, m, P, D);
#pragma unroll
  for (int k = 0; k < 4; k++) {  // (gx, gy, gz) -> (gx + gy, gx - gy, gz), see gdotf
    const float s1 = g1[3 * k] + g1[3 * k + 1], r1 = g1[3 * k] - g1[3 * k + 1];
    const float s2 = g2[3 * k] + g2[3 * k + 1], r2 = g2[3 * k] - g2[3 * k + 1];
    g1[3 * k] = s1;
    g1[3 * k + 1] = r1;
    g2[3 * k] = s2;
    g2[3 * k + 1] = r2;
  }
  lattice_pair32<1, 1, 1>(si, sn, sc, g1, g2, n, kc, w7, drhoI, m, P, D);
  lattice_pair32<1, 1, -1>(si, sn, sc, g1, g2, n, kc, w7, drhoI, m, P, D);
  lattice_pair32<1, -1, 1>(si, sn, sc, g1, g2, n, kc, w7, drhoI, m, P, D);
  lattice_pair32<-1, 1, 1>(si, sn, sc, g1, g2, n, kc, w7, drhoI, m, P, D);
  drhoI += D;
  P[0] += D;
  P[1] += D;
  P[2] += D;

  const float tau = f2.w;  // 3 nu / (dt_s gamma), per face from the layout
  const float mn = m[0] * n[0] + m[1] * n[1] + m[2] * n[2];
  const float Pn[3] = {P[0] * n[0] + P[3] * n[1] + P[4] * n[2],
                       P[3] * n[0] + P[1] * n[1] + P[5] * n[2],
                       P[4] * n[0] + P[5] * n[1] + P[2] * n[2]};
  const float mnr = mn / (kc.rho0 + drhoI) * pg;
  const float p3 = drhoI * (1.0f / 3.0f);
  const float sA = area * a.inv_uref_f;  // momentum flux is stored divided by U
  f4 out;
  out.x = ((1.0f - tau) * fmaf(m[0], mnr, p3 * n[0]) + tau * Pn[0]) * sA;
  out.y = ((1.0f - tau) * fmaf(m[1], mnr, p3 * n[1]) + tau * Pn[1]) * sA;
  out.z = ((1.0f - tau) * fmaf(m[2], mnr, p3 * n[2]) + tau * Pn[2]) * sA;
  out.w = mn * area;
  stf(a.flux, f, out);
}

// Persistent over the faces, next face's ids prefetched (as k_flux); six blocks
// per SM (85 registers) measured fastest.
template <bool CR>
__global__ void __launch_bounds__(kFluxBlock, 6) k_flux32(const KernelArgs a) {
  if (halted(a)) return;
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.F) return;
  int2 ids = __ldg(reinterpret_cast<const int2*>(a.face_ids) + f);
  int rec = CR ? __ldg(a.face_rec + f) : 0;
  for (;;) {
    const long long fn = f + stride;
    const int2 next =
        fn < a.F ? __ldg(reinterpret_cast<const int2*>(a.face_ids) + fn) : make_int2(0, 0);
    const int next_rec = (CR && fn < a.F) ? __ldg(a.face_rec + fn) : 0;
    flux_face32<CR>(a, (int)f, ids, rec);
    if (fn >= a.F) break;
    f = fn;
    ids = next;
    rec = next_rec;
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Gather + body force + RK stage in deviation units; the last stage reduces
// the squared residuals in FP64 (momentum residuals are already divided by U,
// so inv_ref_mom is 1 / rho_ref here).
template <int RK, int K2MAX>
__global__ void __launch_bounds__(kBlock) k_update32(const KernelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (halted(a)) return;
  constexpr float alpha = (RK == 0 || RK == 3) ? 1.0f : 0.5f;
  constexpr float beta = (RK == 0 || RK == 3) ? (1.0f / 6.0f) : (1.0f / 3.0f);
  double sq[4] = {0.0, 0.0, 0.0, 0.0};
  bool bad = false;
  if (i < a.C) {
    // The RK accumulators are loaded first, with the gather, so no store of
    // the stage can come between them and the flux loads.
    const f4 t0 = ldf_rw(a.t0, i);
    f4 t1 = ldf_rw(a.t1, i);
    float r[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    int e[K2MAX];
#pragma unroll
    for (int k = 0; k < K2MAX; k++) e[k] = (k < a.K2) ? __ldg(a.gather + (long long)k * a.C + i) : -1;
    f4 fl[K2MAX];
#pragma unroll
    for (int k = 0; k < K2MAX; k++)
      if (e[k] >= 0) fl[k] = ldf(a.flux, e[k] >> 1);
#pragma unroll
    for (int k = 0; k < K2MAX; k++) {
      if (e[k] < 0) continue;
      const float sg = (e[k] & 1) ? 1.0f : -1.0f;
      r[0] = fmaf(sg, fl[k].x, r[0]);
      r[1] = fmaf(sg, fl[k].y, r[1]);
      r[2] = fmaf(sg, fl[k].z, r[2]);
      r[3] = fmaf(sg, fl[k].w, r[3]);
    }
    const float iv = __ldg(static_cast<const float*>(a.inv_volume) + i);
    float R[4] = {r[0] * iv, r[1] * iv, r[2] * iv, r[3] * iv};
    const float pgU = (float)(a.pressure_gradient) * a.inv_uref_f;
    if (a.fforce_x) {
      R[0] += a.fforce_x[i];
      R[1] += a.fforce_y[i];
      R[2] += a.fforce_z[i];
    } else {
      R[0] += pgU;
    }
    if (a.res_debug) stf(a.res_debug, i, f4{R[0], R[1], R[2], R[3]});
    const float dt = (float)a.dt;
    const float f1 = t0.w + R[3] * dt * alpha;
    const float f2 = t0.x + R[0] * dt * alpha;
    const float f3 = t0.y + R[1] * dt * alpha;
    const float f4v = t0.z + R[2] * dt * alpha;
    t1.w = t1.w + dt * beta * R[3];
    t1.x = t1.x + dt * beta * R[0];
    t1.y = t1.y + dt * beta * R[1];
    t1.z = t1.z + dt * beta * R[2];
    f4 q;
    if (RK == 3) {
      const float rho = a.rho0f + t1.w;
      q = f4{t1.x / rho, t1.y / rho, t1.z / rho, t1.w};
      stf(a.t0, i, t1);
      sq[0] = (double)R[3] * R[3];
      sq[1] = (double)R[0] * R[0];
      sq[2] = (double)R[1] * R[1];
      sq[3] = (double)R[2] * R[2];
      bad = !(rho <= 1000.0f);
    } else {
      const float rho = a.rho0f + f1;
      q = f4{f2 / rho, f3 / rho, f4v / rho, f1};
    }
    stf(a.t1, i, t1);
    stf(a.state, i, q);
    if (RK == 3 && a.fforce_x) {  // after every load of the stage (see k_update)
      a.fforce_x[i] = pgU;
      a.fforce_y[i] = 0.0f;
      a.fforce_z[i] = 0.0f;
    }
  }
  if (RK != 3) return;

  // Per-block squared-residual sums (warp shuffle, then the block's warps in
  // order); k_finish32 reduces them.
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
__global__ void __launch_bounds__(kFinishBlock) k_finish32(const KernelArgs a) {
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

// As k_seed; the conserved accumulators in deviation units are
// (rho u / U, rho v / U, rho w / U, rho - rho0).
template <bool CONSERVED>
__global__ void k_seed32(const KernelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.C) return;
  f4 q = ldf(a.state, i);
  if (CONSERVED) {
    const float rho = a.rho0f + q.w;
    q = f4{rho * q.x, rho * q.y, rho * q.z, q.w};
  }
  stf(a.t0, i, q);
  stf(a.t1, i, q);
}

// IBM with FP64 node positions and forces; velocities interpolated from the
// FP32 state (times U) and forces spread as force / U in FP32.
// Eight threads per node, warp-aggregated spreading (as k_ibm). Node quantities stay FP64; the state is
// scaled by U when read and the spread force divided by U when written.
__global__ void __launch_bounds__(kIbmBlock) k_ibm32(const KernelArgs a) {
  if (halted(a)) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int slot = t >> 3, sub = t & 7;
  const bool active = slot < a.N;
  const int nd = active ? __ldg(a.ibm_order + slot) : 0;
  const int xc = a.ibm_xc, yc = a.ibm_yc;
  const double U = a.uref;
  double x[3] = {0.0, 0.0, 0.0}, r[3] = {0.0, 0.0, 0.0};
  int lo[3] = {0, 0, 0};
  auto origin = [&](const double p[3]) {
    r[0] = (p[0] - a.origin[0]) / a.ibm_dx;
    r[1] = fabs((p[1] - a.origin[1]) / a.ibm_dx);
    r[2] = fabs((p[2] - a.origin[2]) / a.ibm_dx);
#pragma unroll
    for (int c = 0; c < 3; c++) lo[c] = (int)round(r[c]) - 1;
  };
  if (active) {
#pragma unroll
    for (int c = 0; c < 3; c++) x[c] = a.node_x[3 * nd + c];
    origin(x);
  }
  const int di = sub & 1, dj = (sub >> 1) & 1, dk = sub >> 2;
  double v[3] = {0.0, 0.0, 0.0};
  {
    const int ii = lo[0] + di, jj = lo[1] + dj, kk = lo[2] + dk;
    const long long cell = (long long)ii + (long long)jj * xc + (long long)kk * yc * xc;
    if (active && cell < a.C && cell >= 0) {
      const double wx = 1 - fabs(ii + 0.5 - r[0]);
      const double wy = 1 - fabs(jj + 0.5 - r[1]);
      const double wz = 1 - fabs(kk + 0.5 - r[2]);
      const f4 q = ldf(a.state, a.ibm_map[cell]);
      v[0] = (U * q.x) * wx * wy * wz * a.ibm_inv_dx3;
      v[1] = (U * q.y) * wx * wy * wz * a.ibm_inv_dx3;
      v[2] = (U * q.z) * wx * wy * wz * a.ibm_inv_dx3;
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
  origin(x);
  const int ii = lo[0] + di, jj = lo[1] + dj, kk = lo[2] + dk;
  const long long cell = (long long)ii + (long long)jj * xc + (long long)kk * yc * xc;
  int target = -1;
  float f[3] = {0.f, 0.f, 0.f};
  if (cell < a.C && cell >= 0) {
    const double wgt = (1 - fabs(ii + 0.5 - r[0])) * (1 - fabs(jj + 0.5 - r[1])) *
                       (1 - fabs(kk + 0.5 - r[2])) * a.ibm_inv_dx3 / U;
    target = a.ibm_map[cell];
#pragma unroll
    for (int c = 0; c < 3; c++) f[c] = (float)(fn[c] * wgt);
  }
  spread_aggregated(act, target, f, a.fforce_x, a.fforce_y, a.fforce_z);
}

inline int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

template <int RK>
void launch_update32_rk(const KernelArgs& a, int nb, cudaStream_t s) {
  if (a.K2 <= 4)
    k_update32<RK, 4><<<nb, kBlock, 0, s>>>(a);
  else if (a.K2 <= 6)
    k_update32<RK, 6><<<nb, kBlock, 0, s>>>(a);
  else if (a.K2 <= 8)
    k_update32<RK, 8><<<nb, kBlock, 0, s>>>(a);
  else
    k_update32<RK, 16><<<nb, kBlock, 0, s>>>(a);
}

}  // namespace

void launch_gradient32(const KernelArgs& a, cudaStream_t s) {
  if (a.compact && a.wtab)
    k_gradient32<true><<<blocks_for(a.C, kBlock), kBlock, 0, s>>>(a);
  else
    k_gradient32<false><<<blocks_for(a.C, kBlock), kBlock, 0, s>>>(a);
}
void launch_flux32(const KernelArgs& a, cudaStream_t s) {
  static std::atomic<int> resident[kMaxDevices], cr_resident[kMaxDevices];
  if (a.compact && a.face_rec)
    k_flux32<true><<<persistent_blocks(k_flux32<true>, kFluxBlock, a.F, cr_resident), kFluxBlock,
                     0, s>>>(a);
  else
    k_flux32<false><<<persistent_blocks(k_flux32<false>, kFluxBlock, a.F, resident), kFluxBlock,
                      0, s>>>(a);
}
void launch_update32(const KernelArgs& a, int rk, cudaStream_t s, bool finish) {
  const int nb = blocks_for(a.C, kBlock);
  switch (rk) {
    case 0: launch_update32_rk<0>(a, nb, s); break;
    case 1: launch_update32_rk<1>(a, nb, s); break;
    case 2: launch_update32_rk<2>(a, nb, s); break;
    default:
      launch_update32_rk<3>(a, nb, s);
      if (finish) k_finish32<<<1, kFinishBlock, 0, s>>>(a);
      break;
  }
}
void launch_finish32(const KernelArgs& a, cudaStream_t s) {
  k_finish32<<<1, kFinishBlock, 0, s>>>(a);
}
void launch_seed32(const KernelArgs& a, bool conserved, cudaStream_t s) {
  if (conserved)
    k_seed32<true><<<blocks_for(a.C, kBlock), kBlock, 0, s>>>(a);
  else
    k_seed32<false><<<blocks_for(a.C, kBlock), kBlock, 0, s>>>(a);
}
void launch_ibm32(const KernelArgs& a, cudaStream_t s) {
  if (a.N > 0) k_ibm32<<<blocks_for(8LL * a.N, kIbmBlock), kIbmBlock, 0, s>>>(a);
}

}  // namespace plfbs
