// Learned warm start: a mesh graph network over the solver's face graph
// (include/plfbs_gnn.h). No counterpart in the reference.
//
// Every MLP of the network is Linear(K1, 64) -> ReLU -> Linear(64, NOUT) over
// rows gathered from the graph. One fused kernel per direction does a whole
// MLP for tiles of 128 rows:
//   forward:  gather X1 (FP32 -> BF16 in shared memory), Z1 = X1 W1 + b1
//             (stored for the backward pass), Y = relu(Z1) W2 + b2 (+ the
//             row's own input for the residual message-passing layers);
//   backward: the same gather plus dY, then dA = dY W2^T, dZ1 = dA relu'(Z1),
//             dX1 = dZ1 W1^T (scattered by segment), and the weight gradients
//             X1^T dZ1, relu(Z1)^T dY and the bias sums accumulated per block
//             across its tiles; a second kernel adds the block partials in a
//             fixed order, so gradients are deterministic.
// The products run on the tensor cores: by default as tcgen05 MMAs (one
// thread issuing 128 x N x 16 BF16 products from shared-memory descriptors,
// FP32 accumulators in tensor memory; the backward's transposed operands read
// through MN-major descriptors), or as mma.sync m16n8k16 BF16 x BF16 -> FP32
// with ldmatrix operands (.trans for the transposed products), one warp per
// 16 rows. Aggregation over edges goes through CSR lists (no atomics). Activations and master weights are FP32; Adam runs on the device.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "plfbs.h"
#include "plfbs_gnn.h"

namespace gnn {

using bf16 = __nv_bfloat16;
constexpr int H = 64;          // hidden width
constexpr int TM = 128;        // rows per tile
constexpr int kThreads = 256;  // 8 warps, 16 rows each
constexpr int FP = 16;         // features and outputs are padded to 16 columns

enum Mode { ENC = 0, EDGE = 1, NODE = 2, DEC = 3 };

// ---------------------------------------------------------------------------
// tensor-core helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned su32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const bf16* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(su32(p))
               : "memory");
}
__device__ __forceinline__ void ldsm_x4_t(unsigned (&r)[4], const bf16* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(su32(p))
               : "memory");
}
__device__ __forceinline__ void ldsm_x2_t(unsigned (&r)[2], const bf16* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0, %1}, [%2];\n"
               : "=r"(r[0]), "=r"(r[1])
               : "r"(su32(p))
               : "memory");
}
// c (16x8, FP32) += a (16x16, BF16, row) * b (16x8, BF16, col)
__device__ __forceinline__ void mma(float (&c)[4], const unsigned (&a)[4], unsigned b0,
                                    unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, "
      "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Fragment layout of the accumulators (per 16x8 tile j): c0, c1 at row
// lane/4, columns 8j + 2(lane%4) + {0, 1}; c2, c3 at row lane/4 + 8.

// acc[j] += A[r0 .. r0+16, 0 .. K) * W[0 .. K, 8j .. 8j+8); A and W row-major
// in shared memory (W as [K][ldw]).
template <int K, int NT>
__device__ __forceinline__ void gemm_a_w(float (&acc)[NT][4], const bf16* A, int lda, int r0,
                                         const bf16* W, int ldw) {
  static_assert(NT % 2 == 0, "pairs of n-tiles");
  const int lane = threadIdx.x & 31, mat = lane >> 3, rr = lane & 7;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    unsigned a[4];
    ldsm_x4(a, A + (r0 + (lane & 15)) * lda + k0 + (lane >> 4) * 8);
#pragma unroll
    for (int j = 0; j < NT; j += 2) {
      unsigned b[4];
      ldsm_x4_t(b, W + (k0 + rr + (mat & 1) * 8) * ldw + 8 * j + (mat >> 1) * 8);
      mma(acc[j], a, b[0], b[1]);
      mma(acc[j + 1], a, b[2], b[3]);
    }
  }
}

// acc[j] += A[r0 .. r0+16, 0 .. K) * W[n0 + 8j .., 0 .. K)^T with W row-major
// [rows][ldw]: the product with a transposed weight matrix.
template <int K, int NT>
__device__ __forceinline__ void gemm_a_wt(float (&acc)[NT][4], const bf16* A, int lda, int r0,
                                          const bf16* W, int ldw, int n0) {
  static_assert(NT % 2 == 0, "pairs of n-tiles");
  const int lane = threadIdx.x & 31, mat = lane >> 3, rr = lane & 7;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    unsigned a[4];
    ldsm_x4(a, A + (r0 + (lane & 15)) * lda + k0 + (lane >> 4) * 8);
#pragma unroll
    for (int j = 0; j < NT; j += 2) {
      unsigned b[4];
      ldsm_x4(b, W + (n0 + 8 * j + rr + (mat >> 1) * 8) * ldw + k0 + (mat & 1) * 8);
      mma(acc[j], a, b[0], b[1]);
      mma(acc[j + 1], a, b[2], b[3]);
    }
  }
}

// acc[i] += X[0 .. 128, p0 + 16i ..)^T * D[0 .. 128, n0 .. n0+8): weight
// gradients, reducing over the tile's rows.
template <int RT>
__device__ __forceinline__ void gemm_xt_d(float (&acc)[RT][4], const bf16* X, int ldx, int p0,
                                          const bf16* D, int ldd, int n0) {
  const int lane = threadIdx.x & 31, mat = lane >> 3, rr = lane & 7;
#pragma unroll 2
  for (int m0 = 0; m0 < TM; m0 += 16) {
    unsigned b[2];
    ldsm_x2_t(b, D + (m0 + rr + (mat & 1) * 8) * ldd + n0);
#pragma unroll
    for (int i = 0; i < RT; i++) {
      unsigned a[4];
      ldsm_x4_t(a, X + (m0 + rr + (mat >> 1) * 8) * ldx + p0 + 16 * i + (mat & 1) * 8);
      mma(acc[i], a, b[0], b[1]);
    }
  }
}

__device__ __forceinline__ float4 ldg4(const float* p) {
  return __ldg(reinterpret_cast<const float4*>(p));
}
__device__ __forceinline__ void st_bf16x4(bf16* p, float4 v) {
  __nv_bfloat162 lo = __floats2bfloat162_rn(v.x, v.y), hi = __floats2bfloat162_rn(v.z, v.w);
  *reinterpret_cast<__nv_bfloat162*>(p) = lo;
  *reinterpret_cast<__nv_bfloat162*>(p + 2) = hi;
}

// ---------------------------------------------------------------------------
// gather of the input rows X1 of one tile
// ---------------------------------------------------------------------------
struct Rows {
  int M;
  const float* x0;      // ENC: features [M][16]; EDGE: e_prev; NODE: h_prev; DEC: h   ([M][64])
  const float* hs;      // EDGE: node states gathered at src and dst [N][64]
  const int* src;       // EDGE
  const int* dst;       // EDGE
  const int* in_off;    // NODE: incoming edges of each node (CSR)
  const int* in_idx;
  const float* eagg;    // NODE: edge states summed over the incoming edges [E][64]
};

template <int MODE, int K1>
__device__ __forceinline__ void load_x(const Rows& a, int row0, bf16* Xs, int lx) {
  constexpr int C4 = K1 / 4;
  for (int q = threadIdx.x; q < TM * C4; q += kThreads) {
    const int r = q / C4, c4 = q - r * C4, m = row0 + r;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (m < a.M) {
      if (MODE == ENC) {
        v = ldg4(a.x0 + (size_t)m * FP + 4 * c4);
      } else if (MODE == DEC) {
        v = ldg4(a.x0 + (size_t)m * H + 4 * c4);
      } else if (MODE == EDGE) {
        const int seg = c4 >> 4, cc = (c4 & 15) * 4;
        const float* p = seg == 0 ? a.x0 + (size_t)m * H
                                  : a.hs + (size_t)(seg == 1 ? a.src[m] : a.dst[m]) * H;
        v = ldg4(p + cc);
      } else {
        const int seg = c4 >> 4, cc = (c4 & 15) * 4;
        if (seg == 0) {
          v = ldg4(a.x0 + (size_t)m * H + cc);
        } else {
          for (int k = a.in_off[m]; k < a.in_off[m + 1]; k++) {
            const float4 e = ldg4(a.eagg + (size_t)a.in_idx[k] * H + cc);
            v.x += e.x;
            v.y += e.y;
            v.z += e.z;
            v.w += e.w;
          }
        }
      }
    }
    st_bf16x4(Xs + r * lx + 4 * c4, v);
  }
}

template <int K1, int NOUT>
__device__ __forceinline__ void load_weights(const bf16* W1, const bf16* W2, bf16* W1s, int lw1,
                                             bf16* W2s, int lw2) {
  for (int i = threadIdx.x; i < K1 * H / 8; i += kThreads) {
    const int r = i / (H / 8), c = (i % (H / 8)) * 8;
    *reinterpret_cast<uint4*>(W1s + r * lw1 + c) = *reinterpret_cast<const uint4*>(W1 + r * H + c);
  }
  for (int i = threadIdx.x; i < H * NOUT / 8; i += kThreads) {
    const int r = i / (NOUT / 8), c = (i % (NOUT / 8)) * 8;
    *reinterpret_cast<uint4*>(W2s + r * lw2 + c) =
        *reinterpret_cast<const uint4*>(W2 + r * NOUT + c);
  }
}

template <int K1, int NOUT>
constexpr size_t fwd_smem() {
  return 2 * (size_t)(TM * (K1 + 8) + TM * (H + 8) + K1 * (H + 8) + H * (NOUT + 8));
}
template <int K1, int NOUT>
constexpr size_t bwd_smem() {
  return 2 * (size_t)(TM * (K1 + 8) + TM * (NOUT + 8) + 2 * TM * (H + 8) + K1 * (H + 8) +
                      H * (NOUT + 8)) +
         4 * (size_t)(TM * (NOUT + 4) + 8 * H + kThreads * 4);
}

// ---------------------------------------------------------------------------
// forward
// ---------------------------------------------------------------------------
struct Fwd {
  Rows x;
  const bf16* W1;   // [K1][64]
  const float* b1;  // [64]
  const bf16* W2;   // [64][NOUT]
  const float* b2;  // [NOUT]
  float* z1;        // [M][64] pre-activations, or null (inference)
  float* y;         // [M][NOUT]
};

template <int MODE, int K1, int NOUT>
__global__ void __launch_bounds__(kThreads, 2) k_mlp_fwd(const Fwd a) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int LX = K1 + 8, LH = H + 8, LW2 = NOUT + 8;
  bf16* Xs = reinterpret_cast<bf16*>(smem);
  bf16* Hs = Xs + TM * LX;
  bf16* W1s = Hs + TM * LH;
  bf16* W2s = W1s + K1 * LH;
  load_weights<K1, NOUT>(a.W1, a.W2, W1s, LH, W2s, LW2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = warp * 16;
  const int ntiles = (a.x.M + TM - 1) / TM;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row0 = tile * TM;
    __syncthreads();  // weights in place; the previous tile's X no longer read
    load_x<MODE, K1>(a.x, row0, Xs, LX);
    __syncthreads();
    float acc[H / 8][4] = {};
    gemm_a_w<K1, H / 8>(acc, Xs, LX, r0, W1s, LH);
#pragma unroll
    for (int j = 0; j < H / 8; j++) {
      const int col = 8 * j + 2 * t;
      const float c0 = a.b1[col], c1 = a.b1[col + 1];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int r = r0 + g + 8 * h, m = row0 + r;
        const float v0 = acc[j][2 * h] + c0, v1 = acc[j][2 * h + 1] + c1;
        if (a.z1 && m < a.x.M) *reinterpret_cast<float2*>(a.z1 + (size_t)m * H + col) = make_float2(v0, v1);
        *reinterpret_cast<__nv_bfloat162*>(Hs + r * LH + col) =
            __floats2bfloat162_rn(fmaxf(v0, 0.f), fmaxf(v1, 0.f));
      }
    }
    __syncwarp();  // a warp's second product reads only its own 16 rows of Hs
    float acc2[NOUT / 8][4] = {};
    gemm_a_w<H, NOUT / 8>(acc2, Hs, LH, r0, W2s, LW2);
#pragma unroll
    for (int j = 0; j < NOUT / 8; j++) {
      const int col = 8 * j + 2 * t;
      const float c0 = a.b2[col], c1 = a.b2[col + 1];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int m = row0 + r0 + g + 8 * h;
        if (m >= a.x.M) continue;
        float v0 = acc2[j][2 * h] + c0, v1 = acc2[j][2 * h + 1] + c1;
        if (MODE == EDGE || MODE == NODE) {  // residual: the row's own previous state
          const float2 p = *reinterpret_cast<const float2*>(a.x.x0 + (size_t)m * H + col);
          v0 += p.x;
          v1 += p.y;
        }
        *reinterpret_cast<float2*>(a.y + (size_t)m * NOUT + col) = make_float2(v0, v1);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// forward on the fifth-generation tensor cores (tcgen05). Operands sit in
// shared memory in the canonical K-major layout without swizzle: 8-row x
// 16-byte core matrices, the K-adjacent ones 128 B apart (leading byte
// offset), 8-row groups K x 16 B apart (stride byte offset). One thread issues
// the MMAs (128 x N x 16 each, BF16 in, FP32 accumulators in tensor memory)
// and commits them to an mbarrier; a warp reads the 32 accumulator rows of
// its lane quarter (warp % 4) with tcgen05.ld, one row per thread, warps w
// and w + 4 taking the two halves of the columns.
// ---------------------------------------------------------------------------
constexpr int kTcThreads = 256;  // 8 warps: warps w and w + 4 share accumulator rows

__device__ __forceinline__ uint32_t canon_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ uint64_t smem_desc(const void* base, int K) {
  const uint64_t addr = su32(base);
  return ((addr & 0x3FFFFull) >> 4) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)((K * 16) >> 4) << 32) | (1ull << 46);
}
// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 and M >> 4.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}
// The same canonical [rows][C] tile read MN-major (the backward's transposed
// operands): its C columns are the M (or N) dimension and its rows the K
// dimension, so the 8-column groups (128 B apart) are the stride byte offset
// and the 8-row groups (C * 16 B apart) the leading byte offset.
__device__ __forceinline__ uint64_t smem_desc_mn(const void* base, int C) {
  const uint64_t addr = su32(base);
  return ((addr & 0x3FFFFull) >> 4) | ((uint64_t)((C * 16) >> 4) << 16) |
         ((uint64_t)(128 >> 4) << 32) | (1ull << 46);
}
// idesc_bf16 with A (bit 15) and B (bit 16) read MN-major.
__host__ __device__ constexpr uint32_t idesc_bf16_mn(int M, int N) {
  return idesc_bf16(M, N) | (1u << 15) | (1u << 16);
}
__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                     int accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   su32(mbar))
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(su32(mbar)), "r"(count)
               : "memory");
}
// Waits for the mbarrier phase of the given parity; gives up (false) after a
// bounded number of tries instead of spinning for ever.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); i++) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(su32(mbar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, int ncols) {  // one whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                   su32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {  // the same warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols)
               : "memory");
}
// 16 consecutive FP32 columns of this thread's row (lane) of the accumulator.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// 256-bit global accesses (one full 32-byte sector per thread); p 32-byte aligned.
__device__ __forceinline__ void ldg8(const float* p, float (&v)[8]) {
  asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]),
                 "=f"(v[6]), "=f"(v[7])
               : "l"(p));
}
__device__ __forceinline__ void stg8(float* p, const float* v) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"l"(p), "f"(v[0]),
               "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}

// As load_x, into the canonical layout. Thread t takes row t % 128 of the tile
// and its 8-element (16-byte) chunks t / 128, t / 128 + 2, ...: a warp's stores
// fill whole core matrices (no bank conflicts) and each thread reads whole
// 32-byte sectors. The row's sources (its node rows for an edge MLP, its CSR
// range for a node MLP) are read once, and the chunks are loaded four at a
// time, so that a thread has four independent gathers in flight rather than
// one (the kernels are bound by the latency of these gathers); a group of
// four chunks covers one 64-column input segment.
template <int MODE, int K1>
__device__ __forceinline__ void load_x_canon(const Rows& a, int row0, unsigned char* As) {
  constexpr int C8 = K1 / 8, NQ = TM * C8 / kTcThreads, G = NQ < 4 ? NQ : 4;
  static_assert(kTcThreads == 2 * TM && (TM * C8) % kTcThreads == 0 && NQ % G == 0,
                "chunks per thread");
  const int r = threadIdx.x % TM, kc0 = threadIdx.x / TM, m = row0 + r;
  const bool valid = m < a.M;
  const float *p0 = nullptr, *p1 = nullptr, *p2 = nullptr;
  int e0 = 0, e1 = 0;
  if (valid) {
    p0 = a.x0 + (size_t)m * (MODE == ENC ? FP : H);
    if (MODE == EDGE) {
      p1 = a.hs + (size_t)a.src[m] * H;
      p2 = a.hs + (size_t)a.dst[m] * H;
    }
    if (MODE == NODE) {
      e0 = a.in_off[m];
      e1 = a.in_off[m + 1];
    }
  }
#pragma unroll
  for (int g0 = 0; g0 < NQ; g0 += G) {
    float v[G][8];
#pragma unroll
    for (int i = 0; i < G; i++) {
      const int c = kc0 + 2 * (g0 + i);  // this chunk: columns 8c .. 8c + 7
#pragma unroll
      for (int j = 0; j < 8; j++) v[i][j] = 0.f;
      if (valid && !(MODE == NODE && c >= 8)) {
        const int seg = MODE == ENC ? 0 : c / 8;
        const float* p = seg == 0 ? p0 : (seg == 1 ? p1 : p2);
        ldg8(p + (MODE == ENC ? 8 * c : 8 * (c % 8)), v[i]);
      }
    }
    if (MODE == NODE && kc0 + 2 * g0 >= 8) {
      // the aggregate segment: the sum of the edge states over the incoming
      // edges, in CSR order
#pragma unroll 2
      for (int e = e0; e < e1; e++) {
        const float* pe = a.eagg + (size_t)a.in_idx[e] * H;
#pragma unroll
        for (int i = 0; i < G; i++) {
          float u[8];
          ldg8(pe + 8 * (kc0 + 2 * (g0 + i) - 8), u);
#pragma unroll
          for (int j = 0; j < 8; j++) v[i][j] += u[j];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < G; i++) {
      const int c = kc0 + 2 * (g0 + i);
      __nv_bfloat162 b[4] = {
          __floats2bfloat162_rn(v[i][0], v[i][1]), __floats2bfloat162_rn(v[i][2], v[i][3]),
          __floats2bfloat162_rn(v[i][4], v[i][5]), __floats2bfloat162_rn(v[i][6], v[i][7])};
      *reinterpret_cast<uint4*>(As + canon_off(r, 8 * c, K1)) =
          *reinterpret_cast<const uint4*>(b);
    }
  }
}

template <int MODE, int K1, int NOUT>
__global__ void __launch_bounds__(kTcThreads) k_mlp_fwd_tc(const Fwd a, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* As = smem;                       // [128][K1]
  unsigned char* Hs = As + TM * K1 * 2;           // [128][64]
  unsigned char* W1t = Hs + TM * H * 2;           // [64][K1]: W1 transposed
  unsigned char* W2t = W1t + H * K1 * 2;          // [NOUT][64]: W2 transposed
  uint64_t* mbar = reinterpret_cast<uint64_t*>(W2t + NOUT * H * 2);
  uint32_t* slot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < K1 * H; i += kTcThreads)
    *reinterpret_cast<bf16*>(W1t + canon_off(i % H, i / H, K1)) = a.W1[i];
  for (int i = tid; i < H * NOUT; i += kTcThreads)
    *reinterpret_cast<bf16*>(W2t + canon_off(i % NOUT, i / NOUT, H)) = a.W2[i];
  if (tid == 0) mbar_init(mbar, 1);
  if (warp == 0) tmem_alloc(slot, 128);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot, d1 = tmem, d2 = tmem + 64;
  const int quarter = warp & 3, half = warp >> 2;
  const uint32_t lanes = (uint32_t)(quarter * 32) << 16;  // this warp's 32 accumulator rows
  const int r = quarter * 32 + lane;                       // this thread's row of the tile
  uint32_t parity = 0;
  bool ok = true;
  const int ntiles = (a.x.M + TM - 1) / TM;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int row0 = tile * TM, m = row0 + r;
    load_x_canon<MODE, K1>(a.x, row0, As);
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int k0 = 0; k0 < K1; k0 += 16)
        umma(d1, smem_desc(As + k0 * 16, K1), smem_desc(W1t + k0 * 16, K1),
             idesc_bf16(TM, H), k0 > 0);
      umma_commit(mbar);
    }
    __syncwarp();
    ok = mbar_wait(mbar, parity);
    parity ^= 1u;
    tc_fence_after();
#pragma unroll
    for (int c0 = 32 * half; c0 < 32 * half + 32; c0 += 16) {
      float v[16];
      tmem_ld16(d1 + lanes + c0, v);
      __align__(16) bf16 hb[16];
#pragma unroll
      for (int i = 0; i < 16; i++) {
        v[i] += a.b1[c0 + i];
        hb[i] = __float2bfloat16_rn(fmaxf(v[i], 0.f));
      }
      if (a.z1 && m < a.x.M) {
        stg8(a.z1 + (size_t)m * H + c0, v);
        stg8(a.z1 + (size_t)m * H + c0 + 8, v + 8);
      }
      *reinterpret_cast<uint4*>(Hs + canon_off(r, c0, H)) = *reinterpret_cast<const uint4*>(hb);
      *reinterpret_cast<uint4*>(Hs + canon_off(r, c0 + 8, H)) =
          *reinterpret_cast<const uint4*>(hb + 8);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int k0 = 0; k0 < H; k0 += 16)
        umma(d2, smem_desc(Hs + k0 * 16, H), smem_desc(W2t + k0 * 16, H), idesc_bf16(TM, NOUT),
             k0 > 0);
      umma_commit(mbar);
    }
    __syncwarp();
    ok = ok && mbar_wait(mbar, parity);
    parity ^= 1u;
    tc_fence_after();
#pragma unroll
    for (int c0 = 32 * half; c0 < 32 * half + 32 && c0 < NOUT; c0 += 16) {
      float v[16];
      tmem_ld16(d2 + lanes + c0, v);
      if (m < a.x.M) {
        if (MODE == EDGE || MODE == NODE) {  // residual: the row's own previous state
          float p0[8], p1[8];
          ldg8(a.x.x0 + (size_t)m * H + c0, p0);
          ldg8(a.x.x0 + (size_t)m * H + c0 + 8, p1);
#pragma unroll
          for (int i = 0; i < 8; i++) {
            v[i] += p0[i];
            v[8 + i] += p1[i];
          }
        }
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] += a.b2[c0 + i];
        stg8(a.y + (size_t)m * NOUT + c0, v);
        stg8(a.y + (size_t)m * NOUT + c0 + 8, v + 8);
      }
    }
    tc_fence_before();
    ok = __syncthreads_and(ok);  // operands and accumulators free for the next tile
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  tc_fence_after();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 128);
}

// Shared memory of a launch: the operands, and at least 60 KB so that no SM
// holds more than three blocks, whose 3 x 128 tensor-memory columns fit in
// the 512 an SM has (tcgen05.alloc would otherwise wait for a block to end).
template <int K1, int NOUT>
constexpr size_t tc_smem() {
  return std::max<size_t>(2 * (size_t)(TM * K1 + TM * H + H * K1 + NOUT * H) + 16, 61440);
}

// ---------------------------------------------------------------------------
// backward
// ---------------------------------------------------------------------------
struct Bwd {
  Rows x;
  const float* dy;    // [M][NOUT], or null (zero)
  const float* dadd;  // EDGE: [N][64] added to dy at dst (the node aggregate's gradient), or null
  const float* z1;    // [M][64]
  const bf16* W1;
  const bf16* W2;
  float* dx0;    // EDGE/NODE: dy + dX1[:, 0:64]; DEC: dX1 ([M][64]); ENC: unused
  float* dseg1;  // EDGE: dX1[:, 64:128] per edge (to src); NODE: dX1[:, 64:128] (aggregate)
  float* dseg2;  // EDGE: dX1[:, 128:192] per edge (to dst)
  float* part;   // [gridDim.x][K1*64 + 64 + 64*NOUT + NOUT]
};

template <int MODE, int K1, int NOUT>
__global__ void __launch_bounds__(kThreads, 1) k_mlp_bwd(const Bwd a) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int LX = K1 + 8, LH = H + 8, LD = NOUT + 8, L32 = NOUT + 4;
  constexpr int RT1 = K1 / 16;        // row tiles of dW1 per warp (its n-tile is the warp)
  constexpr int RT2 = NOUT == H ? 4 : 1;
  bf16* Xs = reinterpret_cast<bf16*>(smem);
  bf16* Ds = Xs + TM * LX;  // dY (BF16)
  bf16* As = Ds + TM * LD;  // relu(Z1)
  bf16* Zs = As + TM * LH;  // dZ1
  bf16* W1s = Zs + TM * LH;
  bf16* W2s = W1s + K1 * LH;
  float* D32 = reinterpret_cast<float*>(W2s + H * LD);  // dY (FP32)
  float* red = D32 + TM * L32;                          // [8][64] + [kThreads][4]
  load_weights<K1, NOUT>(a.W1, a.W2, W1s, LH, W2s, LD);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = warp * 16;
  float gW1[RT1][4] = {}, gW2[RT2][4] = {}, gb1[2 * (H / 8)] = {}, gb2[4] = {};
  const int ntiles = (a.x.M + TM - 1) / TM;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row0 = tile * TM;
    __syncthreads();
    load_x<MODE, K1>(a.x, row0, Xs, LX);
    constexpr int C4 = NOUT / 4;  // kThreads is a multiple: each thread keeps its 4 columns
    for (int q = threadIdx.x; q < TM * C4; q += kThreads) {
      const int r = q / C4, c4 = q - r * C4, m = row0 + r;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (m < a.x.M) {
        if (a.dy) v = ldg4(a.dy + (size_t)m * NOUT + 4 * c4);
        if (MODE == EDGE && a.dadd) {
          const float4 d = ldg4(a.dadd + (size_t)a.x.dst[m] * H + 4 * c4);
          v.x += d.x;
          v.y += d.y;
          v.z += d.z;
          v.w += d.w;
        }
      }
      gb2[0] += v.x;
      gb2[1] += v.y;
      gb2[2] += v.z;
      gb2[3] += v.w;
      *reinterpret_cast<float4*>(D32 + r * L32 + 4 * c4) = v;
      st_bf16x4(Ds + r * LD + 4 * c4, v);
    }
    for (int q = threadIdx.x; q < TM * H / 4; q += kThreads) {
      const int r = q / (H / 4), c4 = q - r * (H / 4), m = row0 + r;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (m < a.x.M) v = ldg4(a.z1 + (size_t)m * H + 4 * c4);
      v = make_float4(fmaxf(v.x, 0.f), fmaxf(v.y, 0.f), fmaxf(v.z, 0.f), fmaxf(v.w, 0.f));
      st_bf16x4(As + r * LH + 4 * c4, v);
    }
    __syncthreads();
    // dA = dY W2^T, dZ1 = dA where Z1 > 0
    {
      float da[H / 8][4] = {};
      gemm_a_wt<NOUT, H / 8>(da, Ds, LD, r0, W2s, LD, 0);
#pragma unroll
      for (int j = 0; j < H / 8; j++) {
        const int col = 8 * j + 2 * t;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int r = r0 + g + 8 * h;
          const __nv_bfloat162 av = *reinterpret_cast<const __nv_bfloat162*>(As + r * LH + col);
          const float v0 = __low2float(av) > 0.f ? da[j][2 * h] : 0.f;
          const float v1 = __high2float(av) > 0.f ? da[j][2 * h + 1] : 0.f;
          gb1[2 * j] += v0;
          gb1[2 * j + 1] += v1;
          *reinterpret_cast<__nv_bfloat162*>(Zs + r * LH + col) = __floats2bfloat162_rn(v0, v1);
        }
      }
    }
    // dW2 += relu(Z1)^T dY
    if (NOUT == H)
      gemm_xt_d<RT2>(gW2, As, LH, 0, Ds, LD, 8 * warp);
    else
      gemm_xt_d<RT2>(gW2, As, LH, 16 * (warp >> 1), Ds, LD, 8 * (warp & 1));
    __syncthreads();  // dZ1 of every row
    gemm_xt_d<RT1>(gW1, Xs, LX, 0, Zs, LH, 8 * warp);
    if (MODE != ENC) {
      // dX1 = dZ1 W1^T, 64 columns (one input segment) at a time
#pragma unroll 1
      for (int seg = 0; seg < K1 / H; seg++) {
        float dx[H / 8][4] = {};
        gemm_a_wt<H, H / 8>(dx, Zs, LH, r0, W1s, LH, H * seg);
        float* out = seg == 0 ? a.dx0 : (seg == 1 ? a.dseg1 : a.dseg2);
#pragma unroll
        for (int j = 0; j < H / 8; j++) {
          const int col = 8 * j + 2 * t;
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int r = r0 + g + 8 * h, m = row0 + r;
            if (m >= a.x.M) continue;
            float v0 = dx[j][2 * h], v1 = dx[j][2 * h + 1];
            if (seg == 0 && MODE != DEC) {  // the residual path passes dY through
              v0 += D32[r * L32 + col];
              v1 += D32[r * L32 + col + 1];
            }
            *reinterpret_cast<float2*>(out + (size_t)m * H + col) = make_float2(v0, v1);
          }
        }
      }
    }
  }
  // block partials: [dW1 K1 x 64][db1 64][dW2 64 x NOUT][db2 NOUT]
  float* P = a.part + (size_t)blockIdx.x * (K1 * H + H + H * NOUT + NOUT);
#pragma unroll
  for (int i = 0; i < RT1; i++) {
    const int p = 16 * i + g, n = 8 * warp + 2 * t;
    P[p * H + n] = gW1[i][0];
    P[p * H + n + 1] = gW1[i][1];
    P[(p + 8) * H + n] = gW1[i][2];
    P[(p + 8) * H + n + 1] = gW1[i][3];
  }
  float* P2 = P + K1 * H + H;
#pragma unroll
  for (int i = 0; i < RT2; i++) {
    const int p = (NOUT == H ? 16 * i : 16 * (warp >> 1)) + g;
    const int n = (NOUT == H ? 8 * warp : 8 * (warp & 1)) + 2 * t;
    P2[p * NOUT + n] = gW2[i][0];
    P2[p * NOUT + n + 1] = gW2[i][1];
    P2[(p + 8) * NOUT + n] = gW2[i][2];
    P2[(p + 8) * NOUT + n + 1] = gW2[i][3];
  }
  // db1: over the 8 row groups of a warp (lanes with equal t), then warps in order
#pragma unroll
  for (int k = 0; k < 2 * (H / 8); k++) {
    float v = gb1[k];
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    gb1[k] = v;
  }
  __syncthreads();
  if (g == 0) {
#pragma unroll
    for (int j = 0; j < H / 8; j++) {
      red[warp * H + 8 * j + 2 * t] = gb1[2 * j];
      red[warp * H + 8 * j + 2 * t + 1] = gb1[2 * j + 1];
    }
  }
  float* red2 = red + 8 * H;
#pragma unroll
  for (int c = 0; c < 4; c++) red2[threadIdx.x * 4 + c] = gb2[c];
  __syncthreads();
  if (threadIdx.x < H) {
    float s = 0.f;
    for (int w = 0; w < 8; w++) s += red[w * H + threadIdx.x];
    P[K1 * H + threadIdx.x] = s;
  }
  if (threadIdx.x < NOUT) {  // column c was kept by the threads with tid % C4 == c / 4
    constexpr int C4 = NOUT / 4;
    const int c = threadIdx.x;
    float s = 0.f;
    for (int th = c / 4; th < kThreads; th += C4) s += red2[th * 4 + (c & 3)];
    P2[H * NOUT + c] = s;
  }
}

// ---------------------------------------------------------------------------
// backward, tcgen05 form. Per 128-row tile, five products on the tensor cores
// with FP32 accumulators in tensor memory:
//   dA   = dY W2^T          A = dY [128][NOUT], B = W2 [64][NOUT]        (K-major)
//   dW2 += relu(Z1)^T dY     A = relu(Z1), B = dY, both read MN-major
//   dZ1  = dA where Z1 > 0   (epilogue: tensor memory -> shared memory)
//   dX1  = dZ1 W1^T          A = dZ1 [128][64], B = W1 [K1][64]          (K-major)
//   dW1 += X1^T dZ1          A = X1 read MN-major (128 features per MMA), B = dZ1 MN-major
// The transposed operands are the K-major tiles themselves, read through
// MN-major descriptors, so nothing is transposed in memory. dW1 and dW2 stay
// in tensor memory over all of the block's tiles and are written once as the
// block's partials, like k_mlp_bwd's; db1 and db2 are per-thread sums added
// in a fixed order. An MMA's rows past a matrix's last feature read the
// operand buffer that follows it and land in accumulator rows nobody reads.
// Tensor memory: dA and then dX1 in columns [0, K1), dW1 in [192, 192 + 64 *
// ceil(K1 / 128)), dW2 after it; 512 columns, one block per SM.
// ---------------------------------------------------------------------------
constexpr int kBwdCols = 512;

template <int K1, int NOUT>
constexpr size_t bwd_tc_smem() {
  // the operands and the mbarrier; at least 116 KB so that an SM holds one
  // block (two blocks' 2 x 512 tensor-memory columns would not fit), which
  // also covers the end-of-kernel bias reduction buffers (66 KB)
  return std::max<size_t>(
      2 * (size_t)(TM * K1 + TM * NOUT + 2 * TM * H + K1 * H + H * NOUT) + 16, 118784);
}

template <int MODE, int K1, int NOUT>
__global__ void __launch_bounds__(kTcThreads, 1) k_mlp_bwd_tc(const Bwd a, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* Xs = smem;                 // X1 [128][K1]
  unsigned char* Ds = Xs + TM * K1 * 2;     // dY [128][NOUT] (BF16)
  unsigned char* As = Ds + TM * NOUT * 2;   // relu(Z1) [128][64]
  unsigned char* Zs = As + TM * H * 2;      // dZ1 [128][64]
  unsigned char* W1c = Zs + TM * H * 2;     // W1 [K1][64]
  unsigned char* W2c = W1c + K1 * H * 2;    // W2 [64][NOUT]
  // the mbarrier and the tensor-memory address at the end, clear of the
  // bias reduction buffers that reuse the operands' space
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + bwd_tc_smem<K1, NOUT>() - 16);
  uint32_t* slot = reinterpret_cast<uint32_t*>(mbar + 1);
  constexpr int MT = (K1 + TM - 1) / TM;    // 128-feature row blocks of dW1
  constexpr uint32_t cX = 0, cW1 = 192, cW2 = cW1 + 64 * MT;
  static_assert(K1 <= 192 && H <= 192 && cW2 + NOUT <= kBwdCols, "tensor-memory columns");
  static_assert(NOUT % 16 == 0 && K1 % 16 == 0, "MMA shapes");
  constexpr int GB2 = (TM * (NOUT / 8) + kTcThreads - 1) / kTcThreads * 8;  // dY columns a thread sums
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < K1 * H; i += kTcThreads)
    *reinterpret_cast<bf16*>(W1c + canon_off(i / H, i % H, H)) = a.W1[i];
  for (int i = tid; i < H * NOUT; i += kTcThreads)
    *reinterpret_cast<bf16*>(W2c + canon_off(i / NOUT, i % NOUT, NOUT)) = a.W2[i];
  if (tid == 0) mbar_init(mbar, 1);
  if (warp == 0) tmem_alloc(slot, kBwdCols);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;
  const int quarter = warp & 3, half = warp >> 2;
  const uint32_t lanes = (uint32_t)(quarter * 32) << 16;  // this warp's 32 accumulator rows
  const int r = quarter * 32 + lane;                       // this thread's row of the tile
  float gb1[32], gb2[GB2];
#pragma unroll
  for (int i = 0; i < 32; i++) gb1[i] = 0.f;
#pragma unroll
  for (int i = 0; i < GB2; i++) gb2[i] = 0.f;
  uint32_t parity = 0;
  bool ok = true, any = false;
  const int ntiles = (a.x.M + TM - 1) / TM;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int row0 = tile * TM, m = row0 + r;
    load_x_canon<MODE, K1>(a.x, row0, Xs);
    // dY (plus the node aggregate's gradient at dst for an edge MLP) as BF16,
    // its column sums (db2) kept per thread: thread tid holds row tid % 128 of
    // the 8-column chunks tid / 128 + 2 j
    const int rr = tid % TM, mm = row0 + rr;  // this thread's row of dY and Z1
    const float* pd = (MODE == EDGE && a.dadd && mm < a.x.M)
                          ? a.dadd + (size_t)a.x.dst[mm] * H : nullptr;
#pragma unroll
    for (int j = 0; j < GB2 / 8; j++) {
      const int k = 8 * (tid / TM + 2 * j);
      float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (mm < a.x.M) {
        if (a.dy) ldg8(a.dy + (size_t)mm * NOUT + k, v);
        if (MODE == EDGE && pd) {
          float d[8];
          ldg8(pd + k, d);
#pragma unroll
          for (int i = 0; i < 8; i++) v[i] += d[i];
        }
      }
#pragma unroll
      for (int i = 0; i < 8; i++) gb2[8 * j + i] += v[i];
      __nv_bfloat162 b[4] = {__floats2bfloat162_rn(v[0], v[1]), __floats2bfloat162_rn(v[2], v[3]),
                             __floats2bfloat162_rn(v[4], v[5]), __floats2bfloat162_rn(v[6], v[7])};
      *reinterpret_cast<uint4*>(Ds + canon_off(rr, k, NOUT)) = *reinterpret_cast<const uint4*>(b);
    }
#pragma unroll
    for (int j = 0; j < TM * (H / 8) / kTcThreads; j++) {
      const int k = 8 * (tid / TM + 2 * j);
      float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (mm < a.x.M) ldg8(a.z1 + (size_t)mm * H + k, v);
      __nv_bfloat162 b[4] = {
          __floats2bfloat162_rn(fmaxf(v[0], 0.f), fmaxf(v[1], 0.f)),
          __floats2bfloat162_rn(fmaxf(v[2], 0.f), fmaxf(v[3], 0.f)),
          __floats2bfloat162_rn(fmaxf(v[4], 0.f), fmaxf(v[5], 0.f)),
          __floats2bfloat162_rn(fmaxf(v[6], 0.f), fmaxf(v[7], 0.f))};
      *reinterpret_cast<uint4*>(As + canon_off(rr, k, H)) = *reinterpret_cast<const uint4*>(b);
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int k0 = 0; k0 < NOUT; k0 += 16)
        umma(tmem + cX, smem_desc(Ds + k0 * 16, NOUT), smem_desc(W2c + k0 * 16, NOUT),
             idesc_bf16(TM, H), k0 > 0);
#pragma unroll
      for (int k0 = 0; k0 < TM; k0 += 16)
        umma(tmem + cW2, smem_desc_mn(As + k0 * H * 2, H), smem_desc_mn(Ds + k0 * NOUT * 2, NOUT),
             idesc_bf16_mn(TM, NOUT), any || k0 > 0);
      umma_commit(mbar);
    }
    __syncwarp();
    ok = mbar_wait(mbar, parity);
    parity ^= 1u;
    tc_fence_after();
    // dZ1 = dA where Z1 > 0, into shared memory; db1 per thread
#pragma unroll
    for (int c = 0; c < 32; c += 16) {
      const int c0 = 32 * half + c;
      float v[16];
      tmem_ld16(tmem + cX + lanes + c0, v);
      __align__(16) bf16 av[16];
      *reinterpret_cast<uint4*>(av) = *reinterpret_cast<const uint4*>(As + canon_off(r, c0, H));
      *reinterpret_cast<uint4*>(av + 8) =
          *reinterpret_cast<const uint4*>(As + canon_off(r, c0 + 8, H));
      __align__(16) bf16 zb[16];
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const float z = __bfloat162float(av[i]) > 0.f ? v[i] : 0.f;
        gb1[c + i] += z;
        zb[i] = __float2bfloat16_rn(z);
      }
      *reinterpret_cast<uint4*>(Zs + canon_off(r, c0, H)) = *reinterpret_cast<const uint4*>(zb);
      *reinterpret_cast<uint4*>(Zs + canon_off(r, c0 + 8, H)) =
          *reinterpret_cast<const uint4*>(zb + 8);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      if (MODE != ENC) {
#pragma unroll
        for (int k0 = 0; k0 < H; k0 += 16)
          umma(tmem + cX, smem_desc(Zs + k0 * 16, H), smem_desc(W1c + k0 * 16, H),
               idesc_bf16(TM, K1), k0 > 0);
      }
#pragma unroll
      for (int t = 0; t < MT; t++)
#pragma unroll
        for (int k0 = 0; k0 < TM; k0 += 16)
          umma(tmem + cW1 + 64 * t, smem_desc_mn(Xs + k0 * K1 * 2 + t * 2048, K1),
               smem_desc_mn(Zs + k0 * H * 2, H), idesc_bf16_mn(TM, H), any || k0 > 0);
      umma_commit(mbar);
    }
    __syncwarp();
    ok = mbar_wait(mbar, parity) && ok;
    parity ^= 1u;
    tc_fence_after();
    any = true;
    if (MODE != ENC) {
      // dX1 by input segment of 64 columns; the residual path passes dY through
      // to segment 0 (not for the decoder)
      constexpr int HALF = K1 / 2;
#pragma unroll
      for (int c0 = HALF * half; c0 < HALF * half + HALF; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + cX + lanes + c0, v);
        const int seg = c0 / H, col = c0 % H;
        if (m < a.x.M) {
          if (seg == 0 && MODE != DEC) {
            float d0[8] = {}, d1[8] = {};
            if (a.dy) {
              ldg8(a.dy + (size_t)m * NOUT + col, d0);
              ldg8(a.dy + (size_t)m * NOUT + col + 8, d1);
            }
            if (MODE == EDGE && a.dadd) {
              float e0[8], e1[8];
              ldg8(a.dadd + (size_t)a.x.dst[m] * H + col, e0);
              ldg8(a.dadd + (size_t)a.x.dst[m] * H + col + 8, e1);
#pragma unroll
              for (int i = 0; i < 8; i++) {
                d0[i] += e0[i];
                d1[i] += e1[i];
              }
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
              v[i] += d0[i];
              v[8 + i] += d1[i];
            }
          }
          float* out = seg == 0 ? a.dx0 : (seg == 1 ? a.dseg1 : a.dseg2);
          stg8(out + (size_t)m * H + col, v);
          stg8(out + (size_t)m * H + col + 8, v + 8);
        }
      }
    }
    tc_fence_before();
    ok = __syncthreads_and(ok);  // operands and accumulators free for the next tile
  }
  tc_fence_after();
  // block partials: [dW1 K1 x 64][db1 64][dW2 64 x NOUT][db2 NOUT]
  float* P = a.part + (size_t)blockIdx.x * (K1 * H + H + H * NOUT + NOUT);
  float* P2 = P + K1 * H + H;
#pragma unroll
  for (int t = 0; t < MT; t++) {
    const int f = TM * t + r;  // feature of this accumulator row
#pragma unroll
    for (int c = 0; c < 32; c += 16) {
      const int c0 = 32 * half + c;
      float v[16];
      if (any) {
        tmem_ld16(tmem + cW1 + 64 * t + lanes + c0, v);
      } else {
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = 0.f;
      }
      if (f < K1) {
        stg8(P + (size_t)f * H + c0, v);
        stg8(P + (size_t)f * H + c0 + 8, v + 8);
      }
    }
  }
  for (int c0 = 16 * half; c0 < NOUT; c0 += 32) {  // dW2: rows are the 64 hidden units
    float v[16];
    if (any) {
      tmem_ld16(tmem + cW2 + lanes + c0, v);
    } else {
#pragma unroll
      for (int i = 0; i < 16; i++) v[i] = 0.f;
    }
    if (r < H) {
      stg8(P2 + (size_t)r * NOUT + c0, v);
      stg8(P2 + (size_t)r * NOUT + c0 + 8, v + 8);
    }
  }
  // db1 and db2: the per-thread sums through shared memory (the operands are
  // no longer read: every MMA has completed), added over rows in order
  float* red = reinterpret_cast<float*>(smem);  // [128][65]
  float* red2 = red + TM * (H + 1);             // [256][GB2 + 1]
#pragma unroll
  for (int i = 0; i < 32; i++) red[r * (H + 1) + 32 * half + i] = gb1[i];
#pragma unroll
  for (int i = 0; i < GB2; i++) red2[tid * (GB2 + 1) + i] = gb2[i];
  __syncthreads();
  if (tid < H) {
    float s = 0.f;
    for (int rr = 0; rr < TM; rr++) s += red[rr * (H + 1) + tid];
    P[K1 * H + tid] = s;
  } else if (tid >= 128 && tid < 128 + NOUT) {
    const int c = tid - 128, ch = c / 8, t0 = (ch % 2) * TM, j = ch / 2;
    float s = 0.f;
    for (int rr = 0; rr < TM; rr++) s += red2[(t0 + rr) * (GB2 + 1) + 8 * j + c % 8];
    P2[H * NOUT + c] = s;
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, kBwdCols);
}

// Sum of the block partials into the flat gradient of one MLP:
// W1 [kin][64], b1 [64], W2 [64][out], b2 [out]. A block takes 32 gradient
// entries (consecutive, so each warp's loads are coalesced) and its 8 warps
// split the partials: warp w sums blocks w, w + 8, ... in order, and the 8 sums
// are added in warp order, a fixed order whatever the launch.
constexpr int kReduceWarps = 8;
__global__ void __launch_bounds__(32 * kReduceWarps)
    k_reduce_parts(const float* part, int nblk, int K1, int NOUT, int kin, int out, float* grad) {
  __shared__ float sums[kReduceWarps][32];
  const int stride = K1 * H + H + H * NOUT + NOUT;
  const int n1 = kin * H, n2 = n1 + H, n3 = n2 + H * out, n4 = n3 + out;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + lane;
  float s = 0.f;
  if (i < n4) {
    int po;
    if (i < n1)
      po = i;
    else if (i < n2)
      po = K1 * H + (i - n1);
    else if (i < n3)
      po = K1 * H + H + ((i - n2) / out) * NOUT + (i - n2) % out;
    else
      po = K1 * H + H + H * NOUT + (i - n3);
#pragma unroll 4
    for (int b = w; b < nblk; b += kReduceWarps) s += part[(size_t)b * stride + po];
  }
  sums[w][lane] = s;
  __syncthreads();
  if (w == 0 && i < n4) {
    float t = sums[0][lane];
#pragma unroll
    for (int k = 1; k < kReduceWarps; k++) t += sums[k][lane];
    grad[i] = t;
  }
}

// Flat FP32 parameters of one MLP -> padded BF16 weights and FP32 biases.
__global__ void k_pack(const float* p, int K1, int NOUT, int kin, int out, bf16* W1, float* b1,
                       bf16* W2, float* b2) {
  const int n = K1 * H + H + H * NOUT + NOUT;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < K1 * H) {
      const int r = i / H, c = i % H;
      W1[i] = __float2bfloat16_rn(r < kin ? p[r * H + c] : 0.f);
    } else if (i < K1 * H + H) {
      b1[i - K1 * H] = p[kin * H + (i - K1 * H)];
    } else if (i < K1 * H + H + H * NOUT) {
      const int k = i - K1 * H - H, r = k / NOUT, c = k % NOUT;
      W2[k] = __float2bfloat16_rn(c < out ? p[kin * H + H + r * out + c] : 0.f);
    } else {
      const int c = i - K1 * H - H - H * NOUT;
      b2[c] = c < out ? p[kin * H + H + H * out + c] : 0.f;
    }
  }
}

__global__ void k_adam(float* p, const float* gr, float* m, float* v, int64_t n, float lr,
                       float c1, float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = gr[i];
    const float mi = 0.9f * m[i] + 0.1f * gi, vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
  }
}

// Mean squared error over the first `out` of FP columns; dy = its gradient.
__global__ void k_loss(const float* y, const float* target, int N, int out, float* dy,
                       double* part) {
  __shared__ double s[kThreads / 32];
  double acc = 0.0;
  const float scale = 2.f / ((float)N * out);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * FP; i += gridDim.x * blockDim.x) {
    const int c = i % FP;
    float d = 0.f;
    if (c < out) d = y[i] - target[i];
    dy[i] = d * scale;
    acc += (double)d * d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < kThreads / 32; w++) v += s[w];
    part[blockIdx.x] = v;
  }
}

// dh[i] += sum of dsrc over the edges leaving i + sum of ddst over the edges
// entering i (the edge MLP's gradients with respect to its gathered states).
__global__ void k_node_grad(int N, const int* out_off, const int* out_idx, const int* in_off,
                            const int* in_idx, const float* dsrc, const float* ddst, float* dh) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x, i = q / (H / 4), c = (q % (H / 4)) * 4;
  if (i >= N) return;
  float4 s = *reinterpret_cast<const float4*>(dh + (size_t)i * H + c);
  for (int k = out_off[i]; k < out_off[i + 1]; k++) {
    const float4 d = ldg4(dsrc + (size_t)out_idx[k] * H + c);
    s.x += d.x;
    s.y += d.y;
    s.z += d.z;
    s.w += d.w;
  }
  for (int k = in_off[i]; k < in_off[i + 1]; k++) {
    const float4 d = ldg4(ddst + (size_t)in_idx[k] * H + c);
    s.x += d.x;
    s.y += d.y;
    s.z += d.z;
    s.w += d.w;
  }
  *reinterpret_cast<float4*>(dh + (size_t)i * H + c) = s;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Mlp {
  int mode, K1, NOUT, kin, out;
  int64_t off, count;  // in the flat parameter array
  bf16* W1 = nullptr;
  float* b1 = nullptr;
  bf16* W2 = nullptr;
  float* b2 = nullptr;
};

}  // namespace gnn

using namespace gnn;

struct plfbs_gnn {
  plfbs_gnn_shape s{};
  int device = 0, sms = 148;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  std::vector<Mlp> mlps;  // n, e, (e_l, n_l) ..., d
  int64_t P = 0;
  float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  long long adam_t = 0;
  int *src = nullptr, *dst = nullptr, *in_off = nullptr, *in_idx = nullptr, *out_off = nullptr,
      *out_idx = nullptr;
  float *feat_n = nullptr, *feat_e = nullptr, *target = nullptr, *y = nullptr, *dy = nullptr;
  std::vector<float*> h, e, zn, ze;  // h[0..L], e[0..L]; pre-activations per MLP
  float *z_enc_n = nullptr, *z_enc_e = nullptr, *z_dec = nullptr;
  float *dh = nullptr, *dh2 = nullptr, *de = nullptr, *de2 = nullptr, *dsrc = nullptr,
        *ddst = nullptr, *dagg = nullptr, *part = nullptr;
  double* loss_part = nullptr;
  int loss_blocks = 0;
  int use_tc = 1;           // MLPs on tcgen05 (1) or mma.sync (0)
  int* tc_err = nullptr;    // set by the tcgen05 kernel if an MMA wait gave up
  std::string err;
};

namespace {

thread_local std::string g_gnn_err;  // errors without a network, per calling thread

int gerr(plfbs_gnn* g, int code, const std::string& m) {
  if (g)
    g->err = m;
  else
    g_gnn_err = m;
  return code;
}

#define GCK(call)                                                                         \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return gerr(g, PLFBS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define GTRY(x)             \
  do {                      \
    int r_ = (x);           \
    if (r_ != 0) return r_; \
  } while (0)

template <typename T>
int galloc(plfbs_gnn* g, T** p, size_t count) {
  void* q = nullptr;
  GCK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  g->allocs.push_back(q);
  GCK(cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), g->stream));
  *p = static_cast<T*>(q);
  return 0;
}

template <int MODE, int K1, int NOUT>
int set_smem(plfbs_gnn* g) {
  GCK(cudaFuncSetAttribute(k_mlp_fwd<MODE, K1, NOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)fwd_smem<K1, NOUT>()));
  GCK(cudaFuncSetAttribute(k_mlp_bwd<MODE, K1, NOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)bwd_smem<K1, NOUT>()));
  return 0;
}

template <int MODE, int K1, int NOUT>
int set_smem_tc(plfbs_gnn* g) {
  GCK(cudaFuncSetAttribute(k_mlp_fwd_tc<MODE, K1, NOUT>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem<K1, NOUT>()));
  GCK(cudaFuncSetAttribute(k_mlp_bwd_tc<MODE, K1, NOUT>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)bwd_tc_smem<K1, NOUT>()));
  return 0;
}

int grid_for(plfbs_gnn* g, int M, int per_sm) {
  const int tiles = (M + TM - 1) / TM;
  return std::max(1, std::min(tiles, g->sms * per_sm));
}

template <int MODE, int K1, int NOUT>
int launch_fwd(plfbs_gnn* g, const Mlp& p, const Rows& x, float* z1, float* y) {
  Fwd a{x, p.W1, p.b1, p.W2, p.b2, z1, y};
  if (g->use_tc) {
    // two blocks per SM: 2 x 98 KB of shared memory, 2 x 128 tensor-memory columns
    k_mlp_fwd_tc<MODE, K1, NOUT><<<grid_for(g, x.M, 2), kTcThreads, tc_smem<K1, NOUT>(),
                                   g->stream>>>(
        a, g->tc_err);
    GCK(cudaGetLastError());
    return 0;
  }
  k_mlp_fwd<MODE, K1, NOUT><<<grid_for(g, x.M, 2), kThreads, fwd_smem<K1, NOUT>(), g->stream>>>(a);
  GCK(cudaGetLastError());
  return 0;
}

template <int MODE, int K1, int NOUT>
int launch_bwd(plfbs_gnn* g, const Mlp& p, const Rows& x, const float* dy, const float* dadd,
               const float* z1, float* dx0, float* dseg1, float* dseg2) {
  const int grid = grid_for(g, x.M, 1);
  Bwd a{x, dy, dadd, z1, p.W1, p.W2, dx0, dseg1, dseg2, g->part};
  if (g->use_tc)
    k_mlp_bwd_tc<MODE, K1, NOUT><<<grid, kTcThreads, bwd_tc_smem<K1, NOUT>(), g->stream>>>(
        a, g->tc_err);
  else
    k_mlp_bwd<MODE, K1, NOUT><<<grid, kThreads, bwd_smem<K1, NOUT>(), g->stream>>>(a);
  GCK(cudaGetLastError());
  const int n = p.kin * H + H + H * p.out + p.out;
  k_reduce_parts<<<(n + 31) / 32, 32 * kReduceWarps, 0, g->stream>>>(g->part, grid, K1, NOUT,
                                                                    p.kin, p.out, g->grad + p.off);
  GCK(cudaGetLastError());
  return 0;
}

Rows rows_enc(int M, const float* f) { return Rows{M, f, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr}; }

int pack_all(plfbs_gnn* g) {
  for (const Mlp& p : g->mlps) {
    k_pack<<<64, 256, 0, g->stream>>>(g->params + p.off, p.K1, p.NOUT, p.kin, p.out, p.W1, p.b1,
                                      p.W2, p.b2);
    GCK(cudaGetLastError());
  }
  return 0;
}

// The tcgen05 kernels' error flag: set when an MMA wait gave up.
int check_tc(plfbs_gnn* g) {
  if (!g->use_tc) return 0;
  int flag = 0;
  GCK(cudaMemcpyAsync(&flag, g->tc_err, sizeof flag, cudaMemcpyDeviceToHost, g->stream));
  GCK(cudaStreamSynchronize(g->stream));
  if (flag) {
    GCK(cudaMemsetAsync(g->tc_err, 0, sizeof flag, g->stream));
    return gerr(g, PLFBS_ERR_CUDA, "a tensor-core MMA did not complete within its wait limit");
  }
  return 0;
}

// forward over the whole graph; z1 buffers are written when `train`
int forward(plfbs_gnn* g, bool train) {
  const int N = g->s.n_nodes, E = g->s.n_edges, L = g->s.layers;
  GTRY((launch_fwd<ENC, FP, H>(g, g->mlps[0], rows_enc(N, g->feat_n), train ? g->z_enc_n : nullptr,
                               g->h[0])));
  GTRY((launch_fwd<ENC, FP, H>(g, g->mlps[1], rows_enc(E, g->feat_e), train ? g->z_enc_e : nullptr,
                               g->e[0])));
  for (int l = 1; l <= L; l++) {
    Rows re{E, g->e[l - 1], g->h[l - 1], g->src, g->dst, nullptr, nullptr, nullptr};
    GTRY((launch_fwd<EDGE, 3 * H, H>(g, g->mlps[2 * l], re, train ? g->ze[l - 1] : nullptr,
                                     g->e[l])));
    Rows rn{N, g->h[l - 1], nullptr, nullptr, nullptr, g->in_off, g->in_idx, g->e[l]};
    GTRY((launch_fwd<NODE, 2 * H, H>(g, g->mlps[2 * l + 1], rn, train ? g->zn[l - 1] : nullptr,
                                     g->h[l])));
  }
  Rows rd{N, g->h[L], nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  GTRY((launch_fwd<DEC, H, FP>(g, g->mlps[2 * L + 2], rd, train ? g->z_dec : nullptr, g->y)));
  return check_tc(g);
}

int loss_and_grad(plfbs_gnn* g, double* loss) {
  const int N = g->s.n_nodes, L = g->s.layers, E = g->s.n_edges;
  k_loss<<<g->loss_blocks, kThreads, 0, g->stream>>>(g->y, g->target, N, g->s.outputs, g->dy,
                                                     g->loss_part);
  GCK(cudaGetLastError());
  std::vector<double> lp(g->loss_blocks);
  GCK(cudaMemcpyAsync(lp.data(), g->loss_part, lp.size() * sizeof(double),
                      cudaMemcpyDeviceToHost, g->stream));
  // backward
  Rows rd{N, g->h[L], nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  GTRY((launch_bwd<DEC, H, FP>(g, g->mlps[2 * L + 2], rd, g->dy, nullptr, g->z_dec, g->dh, nullptr,
                               nullptr)));
  bool have_de = false;  // e_L feeds only the aggregate of node layer L
  for (int l = L; l >= 1; l--) {
    Rows rn{N, g->h[l - 1], nullptr, nullptr, nullptr, g->in_off, g->in_idx, g->e[l]};
    GTRY((launch_bwd<NODE, 2 * H, H>(g, g->mlps[2 * l + 1], rn, g->dh, nullptr, g->zn[l - 1],
                                     g->dh2, g->dagg, nullptr)));
    Rows re{E, g->e[l - 1], g->h[l - 1], g->src, g->dst, nullptr, nullptr, nullptr};
    GTRY((launch_bwd<EDGE, 3 * H, H>(g, g->mlps[2 * l], re, have_de ? g->de : nullptr, g->dagg,
                                     g->ze[l - 1], g->de2, g->dsrc, g->ddst)));
    const int th = N * (H / 4);
    k_node_grad<<<(th + 255) / 256, 256, 0, g->stream>>>(N, g->out_off, g->out_idx, g->in_off,
                                                         g->in_idx, g->dsrc, g->ddst, g->dh2);
    GCK(cudaGetLastError());
    std::swap(g->dh, g->dh2);
    std::swap(g->de, g->de2);
    have_de = true;
  }
  GTRY((launch_bwd<ENC, FP, H>(g, g->mlps[0], rows_enc(N, g->feat_n), g->dh, nullptr, g->z_enc_n,
                               nullptr, nullptr, nullptr)));
  GTRY((launch_bwd<ENC, FP, H>(g, g->mlps[1], rows_enc(E, g->feat_e), g->de, nullptr, g->z_enc_e,
                               nullptr, nullptr, nullptr)));
  GCK(cudaStreamSynchronize(g->stream));
  GTRY(check_tc(g));
  double s = 0.0;
  for (double v : lp) s += v;
  *loss = s / ((double)N * g->s.outputs);
  return 0;
}

int upload_padded(plfbs_gnn* g, float* dst, const float* src, int rows, int cols) {
  std::vector<float> buf((size_t)rows * FP, 0.f);
  for (int r = 0; r < rows; r++)
    for (int c = 0; c < cols; c++) buf[(size_t)r * FP + c] = src[(size_t)r * cols + c];
  GCK(cudaMemcpyAsync(dst, buf.data(), buf.size() * sizeof(float), cudaMemcpyHostToDevice,
                      g->stream));
  GCK(cudaStreamSynchronize(g->stream));
  return 0;
}

int check_g(plfbs_gnn* g) {
  if (!g) return gerr(nullptr, PLFBS_ERR_ARG, "null network");
  GCK(cudaSetDevice(g->device));
  return 0;
}

void csr(int n, const std::vector<int>& key, std::vector<int>& off, std::vector<int>& idx) {
  off.assign(n + 1, 0);
  for (int k : key) off[k + 1]++;
  for (int i = 0; i < n; i++) off[i + 1] += off[i];
  idx.resize(key.size());
  std::vector<int> pos(off.begin(), off.end() - 1);
  for (size_t m = 0; m < key.size(); m++) idx[pos[key[m]]++] = (int)m;
}

}  // namespace

extern "C" {

int plfbs_gnn_create(const plfbs_gnn_shape* shape, const int32_t* src, const int32_t* dst,
                     const float* edge_features, int32_t device, plfbs_gnn** out) {
  if (!shape || !src || !dst || !edge_features || !out)
    return gerr(nullptr, PLFBS_ERR_ARG, "null argument");
  *out = nullptr;
  const plfbs_gnn_shape s = *shape;
  if (s.n_nodes <= 0 || s.n_edges <= 0 || s.node_features < 1 || s.node_features > FP ||
      s.edge_features < 1 || s.edge_features > FP || s.layers < 1 || s.layers > 16 ||
      s.outputs < 1 || s.outputs > FP)
    return gerr(nullptr, PLFBS_ERR_ARG,
                "shape: nodes, edges > 0; features and outputs 1..16; layers 1..16");
  for (int m = 0; m < s.n_edges; m++)
    if (src[m] < 0 || src[m] >= s.n_nodes || dst[m] < 0 || dst[m] >= s.n_nodes)
      return gerr(nullptr, PLFBS_ERR_MESH, "edge endpoint out of range");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return gerr(nullptr, PLFBS_ERR_NO_DEVICE, "no CUDA device with that index");
  // two attributes (cudaGetDeviceProperties fills every field and can be slow)
  int major = 0, sms = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
      major != 10 ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return gerr(nullptr, PLFBS_ERR_NO_DEVICE, "this library is built for sm_100a (B200)");
  plfbs_gnn* g = new (std::nothrow) plfbs_gnn();
  if (!g) return gerr(nullptr, PLFBS_ERR_ARG, "out of host memory");
  g->s = s;
  g->device = device;
  g->sms = sms;
  auto fail = [&](int rc) {
    g_gnn_err = g->err;
    plfbs_gnn_destroy(g);
    return rc;
  };
  int rc;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(gerr(g, PLFBS_ERR_CUDA, "stream creation failed"));
  if ((rc = set_smem<ENC, FP, H>(g)) || (rc = set_smem<EDGE, 3 * H, H>(g)) ||
      (rc = set_smem<NODE, 2 * H, H>(g)) || (rc = set_smem<DEC, H, FP>(g)) ||
      (rc = set_smem_tc<ENC, FP, H>(g)) || (rc = set_smem_tc<EDGE, 3 * H, H>(g)) ||
      (rc = set_smem_tc<NODE, 2 * H, H>(g)) || (rc = set_smem_tc<DEC, H, FP>(g)))
    return fail(rc);
  if ((rc = galloc(g, &g->tc_err, 1))) return fail(rc);
  // parameter layout
  auto add = [&](int mode, int K1, int NOUT, int kin, int o) {
    Mlp p;
    p.mode = mode;
    p.K1 = K1;
    p.NOUT = NOUT;
    p.kin = kin;
    p.out = o;
    p.off = g->P;
    p.count = (int64_t)kin * H + H + (int64_t)H * o + o;
    g->P += p.count;
    g->mlps.push_back(p);
  };
  add(ENC, FP, H, s.node_features, H);
  add(ENC, FP, H, s.edge_features, H);
  for (int l = 0; l < s.layers; l++) {
    add(EDGE, 3 * H, H, 3 * H, H);
    add(NODE, 2 * H, H, 2 * H, H);
  }
  add(DEC, H, FP, H, s.outputs);
  const int N = s.n_nodes, E = s.n_edges, L = s.layers;
  if ((rc = galloc(g, &g->params, g->P)) || (rc = galloc(g, &g->grad, g->P)) ||
      (rc = galloc(g, &g->adam_m, g->P)) || (rc = galloc(g, &g->adam_v, g->P)))
    return fail(rc);
  for (Mlp& p : g->mlps) {
    if ((rc = galloc(g, &p.W1, (size_t)p.K1 * H)) || (rc = galloc(g, &p.b1, H)) ||
        (rc = galloc(g, &p.W2, (size_t)H * p.NOUT)) || (rc = galloc(g, &p.b2, p.NOUT)))
      return fail(rc);
  }
  // graph
  std::vector<int> vs(src, src + E), vd(dst, dst + E), ioff, iidx, ooff, oidx;
  csr(N, vd, ioff, iidx);
  csr(N, vs, ooff, oidx);
  auto up = [&](int** d, const std::vector<int>& v) {
    int r = galloc(g, d, v.size());
    if (r) return r;
    GCK(cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, g->stream));
    GCK(cudaStreamSynchronize(g->stream));
    return 0;
  };
  if ((rc = up(&g->src, vs)) || (rc = up(&g->dst, vd)) || (rc = up(&g->in_off, ioff)) ||
      (rc = up(&g->in_idx, iidx)) || (rc = up(&g->out_off, ooff)) || (rc = up(&g->out_idx, oidx)))
    return fail(rc);
  if ((rc = galloc(g, &g->feat_n, (size_t)N * FP)) || (rc = galloc(g, &g->feat_e, (size_t)E * FP)) ||
      (rc = galloc(g, &g->target, (size_t)N * FP)) || (rc = galloc(g, &g->y, (size_t)N * FP)) ||
      (rc = galloc(g, &g->dy, (size_t)N * FP)))
    return fail(rc);
  if ((rc = upload_padded(g, g->feat_e, edge_features, E, s.edge_features))) return fail(rc);
  g->h.resize(L + 1);
  g->e.resize(L + 1);
  g->zn.resize(L);
  g->ze.resize(L);
  for (int l = 0; l <= L; l++)
    if ((rc = galloc(g, &g->h[l], (size_t)N * H)) || (rc = galloc(g, &g->e[l], (size_t)E * H)))
      return fail(rc);
  for (int l = 0; l < L; l++)
    if ((rc = galloc(g, &g->zn[l], (size_t)N * H)) || (rc = galloc(g, &g->ze[l], (size_t)E * H)))
      return fail(rc);
  if ((rc = galloc(g, &g->z_enc_n, (size_t)N * H)) || (rc = galloc(g, &g->z_enc_e, (size_t)E * H)) ||
      (rc = galloc(g, &g->z_dec, (size_t)N * H)) || (rc = galloc(g, &g->dh, (size_t)N * H)) ||
      (rc = galloc(g, &g->dh2, (size_t)N * H)) || (rc = galloc(g, &g->de, (size_t)E * H)) ||
      (rc = galloc(g, &g->de2, (size_t)E * H)) || (rc = galloc(g, &g->dsrc, (size_t)E * H)) ||
      (rc = galloc(g, &g->ddst, (size_t)E * H)) || (rc = galloc(g, &g->dagg, (size_t)N * H)))
    return fail(rc);
  const size_t part = (size_t)g->sms * (3 * H * H + H + H * H + H);
  if ((rc = galloc(g, &g->part, part))) return fail(rc);
  g->loss_blocks = std::max(1, std::min(4 * g->sms, (N * FP + kThreads - 1) / kThreads));
  if ((rc = galloc(g, &g->loss_part, g->loss_blocks))) return fail(rc);
  if ((rc = pack_all(g))) return fail(rc);
  if (cudaStreamSynchronize(g->stream) != cudaSuccess)
    return fail(gerr(g, PLFBS_ERR_CUDA, "setup failed"));
  *out = g;
  return PLFBS_OK;
}

int plfbs_gnn_param_count(plfbs_gnn* g, int64_t* n) {
  if (!g || !n) return gerr(g, PLFBS_ERR_ARG, "null argument");
  *n = g->P;
  return PLFBS_OK;
}

int plfbs_gnn_set_params(plfbs_gnn* g, const float* params, int64_t n) {
  GTRY(check_g(g));
  if (!params || n != g->P) return gerr(g, PLFBS_ERR_ARG, "parameter count mismatch");
  GCK(cudaMemcpyAsync(g->params, params, n * sizeof(float), cudaMemcpyHostToDevice, g->stream));
  GCK(cudaMemsetAsync(g->adam_m, 0, n * sizeof(float), g->stream));
  GCK(cudaMemsetAsync(g->adam_v, 0, n * sizeof(float), g->stream));
  g->adam_t = 0;
  GTRY(pack_all(g));
  GCK(cudaStreamSynchronize(g->stream));
  return PLFBS_OK;
}

int plfbs_gnn_get_params(plfbs_gnn* g, float* params, int64_t n) {
  GTRY(check_g(g));
  if (!params || n != g->P) return gerr(g, PLFBS_ERR_ARG, "parameter count mismatch");
  GCK(cudaMemcpyAsync(params, g->params, n * sizeof(float), cudaMemcpyDeviceToHost, g->stream));
  GCK(cudaStreamSynchronize(g->stream));
  return PLFBS_OK;
}

int plfbs_gnn_forward(plfbs_gnn* g, const float* node_features, float* y) {
  GTRY(check_g(g));
  if (!node_features || !y) return gerr(g, PLFBS_ERR_ARG, "null argument");
  GTRY(upload_padded(g, g->feat_n, node_features, g->s.n_nodes, g->s.node_features));
  GTRY(forward(g, false));
  std::vector<float> buf((size_t)g->s.n_nodes * FP);
  GCK(cudaMemcpyAsync(buf.data(), g->y, buf.size() * sizeof(float), cudaMemcpyDeviceToHost,
                      g->stream));
  GCK(cudaStreamSynchronize(g->stream));
  for (int i = 0; i < g->s.n_nodes; i++)
    for (int c = 0; c < g->s.outputs; c++) y[(size_t)i * g->s.outputs + c] = buf[(size_t)i * FP + c];
  return PLFBS_OK;
}

int plfbs_gnn_gradients(plfbs_gnn* g, const float* node_features, const float* target,
                        double* loss, float* grad) {
  GTRY(check_g(g));
  if (!node_features || !target || !loss) return gerr(g, PLFBS_ERR_ARG, "null argument");
  GTRY(upload_padded(g, g->feat_n, node_features, g->s.n_nodes, g->s.node_features));
  GTRY(upload_padded(g, g->target, target, g->s.n_nodes, g->s.outputs));
  GTRY(forward(g, true));
  GTRY(loss_and_grad(g, loss));
  if (grad) {
    GCK(cudaMemcpyAsync(grad, g->grad, g->P * sizeof(float), cudaMemcpyDeviceToHost, g->stream));
    GCK(cudaStreamSynchronize(g->stream));
  }
  return PLFBS_OK;
}

int plfbs_gnn_train_step(plfbs_gnn* g, const float* node_features, const float* target,
                         float learning_rate, double* loss) {
  GTRY(plfbs_gnn_gradients(g, node_features, target, loss, nullptr));
  g->adam_t++;
  const float c1 = 1.f / (1.f - powf(0.9f, (float)g->adam_t));
  const float c2 = 1.f / (1.f - powf(0.999f, (float)g->adam_t));
  k_adam<<<256, 256, 0, g->stream>>>(g->params, g->grad, g->adam_m, g->adam_v, g->P,
                                     learning_rate, c1, c2);
  GCK(cudaGetLastError());
  GTRY(pack_all(g));
  GCK(cudaStreamSynchronize(g->stream));
  return PLFBS_OK;
}

int plfbs_gnn_set_tensor_cores(plfbs_gnn* g, int32_t kind) {
  if (!g) return gerr(nullptr, PLFBS_ERR_ARG, "null network");
  if (kind != 0 && kind != 1) return gerr(g, PLFBS_ERR_ARG, "kind is 0 (mma.sync) or 1 (tcgen05)");
  g->use_tc = kind;
  return PLFBS_OK;
}

const char* plfbs_gnn_last_error(const plfbs_gnn* g) { return g ? g->err.c_str() : g_gnn_err.c_str(); }

void plfbs_gnn_destroy(plfbs_gnn* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  for (void* p : g->allocs) cudaFree(p);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

}  // extern "C"
