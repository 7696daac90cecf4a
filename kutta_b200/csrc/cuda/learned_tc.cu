// Tensor-core forward of the learned stage (no reference counterpart): the
// network of learned.cu evaluated in three launches, the two 32-wide layers
// as tcgen05 GEMMs with BF16 operands in shared memory and FP32 accumulators
// in tensor memory.
//
//   lift:    u_i = s_i t_i and v_i = sum_j w_ij s_j t_j (= (W u)_i), plus the
//            sum of u^2 (reduced in a fixed order; rho = sqrt(sum / n));
//   layer A: H1 = relu(ws1 u/rho + wn1 v/rho + b1), evaluated on the fly for
//            a row and its neighbours; A-tile rows [H1_i | sum_j w_ij H1_j]
//            in BF16; D = A [Ws2 | Wn2]^T on the tensor cores; H2 =
//            relu(D + b2) stored as BF16 rows of 64 bytes;
//   layer B: A-tile rows [H2_i | sum_j w_ij H2_j]; D = A [Ws3 | Wn3]^T;
//            z_i = beta z_i + rho s_i sum_c wo_c relu(D_ic + b3_c).
//
// A CTA of 256 threads owns one 128-row tile at a time (persistent loop). All
// threads gather the tile into a 128-byte-swizzled K-major BF16 tile (128 rows
// x 64 values, 16 KB): thread (row r, half h) gathers channels 16h..16h+15 of
// the row and of its neighbours. One thread issues the four K = 16 MMAs
// (M = 128, N = 32) and commits them to an mbarrier; warps 0-3 read the
// 128 x 32 FP32 accumulator back from tensor memory (lanes 32w..32w+31) for
// the epilogue while warps 4-7 start gathering the next tile. Several CTAs
// per SM overlap one tile's gather with another's MMA and epilogue.
//
// Every wait is bounded: a CTA whose MMA does not complete sets fault[0],
// waits once more (bounded) for it, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "common.cuh"
#include "kernels.hpp"

namespace kb2 {
namespace {
using namespace dev;

constexpr int kC = 32;                        // hidden width (MMA N)
constexpr int kTile = 128;                    // rows per tile (MMA M)
constexpr int kWidth = 2 * kC;                // A-tile row: [H | W H]
constexpr int kTcThreads = 256;
constexpr int kTileBytes = kTile * kWidth * 2;  // 16 KB
constexpr int kWeightBytes = kC * kWidth * 2;   // 4 KB
constexpr int kMiscFloats = 160;                // bias, wo, first-layer ws/wn/b
constexpr int kTcSmem = 1024 + kTileBytes + kWeightBytes + kMiscFloats * 4 + 16;
constexpr int kTcPerSm = 4;
constexpr long long kSpinLimit = 1LL << 22;     // mbarrier polls before giving up
constexpr uint32_t kTmemColumns = 32;
// Neighbours whose loads are issued together: all of a tet or hex row for the
// lifted pairs (8 bytes each), half of it for the 64-byte BF16 rows, whose
// registers would otherwise spill.
template <bool kLift>
constexpr int kBatch = kLift ? 8 : 4;

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits
// 4-5 = 1), BF16 A and B (bits 7-9 and 10-12 = 1), both K-major (bits 15 and
// 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                            ((static_cast<uint32_t>(kC) >> 3) << 17) |
                            ((static_cast<uint32_t>(kTile) >> 4) << 24);

// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzle
// layout (rows of 128 bytes, 8-row groups 1024 bytes apart): start address,
// leading byte offset 1 (unused by this layout), stride byte offset 1024, all
// in 16-byte units; version 1 at bit 46; layout type 2 (128-byte swizzle) at
// bits 61-63. The operand must start on a 1024-byte boundary; the K = 16 step
// i of a 64-wide row starts 32 i bytes in (descriptor + 2 i).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>(1) << 16) |
         (static_cast<uint64_t>(1024 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
         (static_cast<uint64_t>(2) << 61);
}

// Byte offset of 16-byte chunk q (0-7) of row r in that layout: chunk q of
// row r sits at chunk position q ^ (r mod 8).
__device__ __forceinline__ uint32_t sw128_offset(int r, int q) {
  return static_cast<uint32_t>((r >> 3) * 1024 + (r & 7) * 128 + ((q ^ (r & 7)) << 4));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// m[0..7] += w * (8 BF16 values of q).
__device__ __forceinline__ void accumulate8(float w, uint4 q, float* m) {
  m[0] = fmaf(w, bf16_lo(q.x), m[0]);
  m[1] = fmaf(w, bf16_hi(q.x), m[1]);
  m[2] = fmaf(w, bf16_lo(q.y), m[2]);
  m[3] = fmaf(w, bf16_hi(q.y), m[3]);
  m[4] = fmaf(w, bf16_lo(q.z), m[4]);
  m[5] = fmaf(w, bf16_hi(q.z), m[5]);
  m[6] = fmaf(w, bf16_lo(q.w), m[6]);
  m[7] = fmaf(w, bf16_hi(q.w), m[7]);
}

__device__ __forceinline__ uint4 pack8(const float* v) {
  return make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]),
                    pack_bf16(v[6], v[7]));
}

// ---- tcgen05 / mbarrier primitives (inline PTX) ---------------------------
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy writes to shared memory made visible to the tensor core.
__device__ __forceinline__ void proxy_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long polls) {
  for (long long k = 0; k < polls; ++k)
    if (mbar_try(bar, parity)) return true;
  return false;
}
// Whole warp: allocate `cols` tensor-memory columns, address written to `slot`.
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
               : "memory");
}
// D (tensor memory) = A B^T (+ D when accumulate != 0), one thread; `idesc`
// the instruction descriptor (shape and types).
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate,
                                         uint32_t idesc = kIdesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// Arrives once on the mbarrier when this thread's issued MMAs complete.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}
// Whole warp: 32 FP32 columns of this thread's tensor-memory lane, the load
// and its wait in one statement so no use of v can precede the wait.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ double input_rms(int n, const double* sum2) {
  const double m = sum2[0] / static_cast<double>(n);
  return m > 0.0 ? sqrt(m) : 0.0;
}

// ---- lift ----------------------------------------------------------------
// uv_i = (s_i t_i, sum_j lift_ij t_j) with lift_ij = w_ij s_j; sum2[0] =
// sum_i (s_i t_i)^2 (block partials summed in block order by the last block).
__global__ void k_gnn_lift(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                           const float* __restrict__ lift, const float* __restrict__ t,
                           const float* __restrict__ node_scale, float2* __restrict__ uv,
                           DeviceReducer red, double* __restrict__ sum2) {
  __shared__ double shared[32];
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float u = node_scale[i] * t[i];
    float v = 0.0f;
    const int end = rows[i + 1];
    for (int j = rows[i]; j < end; ++j) v = fmaf(lift[j], t[cols[j]], v);
    uv[i] = make_float2(u, v);
    acc += static_cast<double>(u) * u;
  }
  const Reducer r{red.partials, red.ticket};
  acc = block_sum(acc, shared);
  if (!publish(r, acc, 0.0, false)) return;
  const double total = gather(r, 0, shared);
  if (threadIdx.x == 0) {
    sum2[0] = total;
    *r.ticket = 0;
  }
}

// ---- one tensor-core layer -----------------------------------------------
// kLift: the input is the lifted pair uv (layer A, output BF16 rows hout);
// otherwise the BF16 rows hin (layer B, output z).
template <bool kLift>
__global__ void __launch_bounds__(kTcThreads, kLift ? 2 : 4)
    k_gnn_layer_tc(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                   const float* __restrict__ edge, const float2* __restrict__ uv,
                   const uint4* __restrict__ hin, const float* __restrict__ first,
                   const float* __restrict__ ws, const float* __restrict__ wn,
                   const float* __restrict__ bias, const float* __restrict__ wo,
                   const float* __restrict__ node_scale, const double* __restrict__ sum2,
                   uint4* __restrict__ hout, float* __restrict__ z, float beta,
                   int* __restrict__ fault, long long first_polls) {
  extern __shared__ uint8_t raw[];
  const uint32_t pad = (1024u - (smem_u32(raw) & 1023u)) & 1023u;
  uint8_t* tile_a = raw + pad;
  uint8_t* tile_b = tile_a + kTileBytes;
  float* misc = reinterpret_cast<float*>(tile_b + kWeightBytes);  // bias | wo | ws1 wn1 b1
  uint64_t* bar = reinterpret_cast<uint64_t*>(misc + kMiscFloats);
  uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  {  // B operand: row c = output channel, chunk q < 4 from Ws[c], q >= 4 from Wn[c].
    const int c = tid >> 3, q = tid & 7;
    const float* src = (q < 4 ? ws : wn) + c * kC + (q & 3) * 8;
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = src[k];
    *reinterpret_cast<uint4*>(tile_b + sw128_offset(c, q)) = pack8(v);
  }
  if (tid < kC) {
    misc[tid] = bias[tid];
    misc[kC + tid] = kLift ? 0.0f : wo[tid];
  }
  if (kLift && tid < 3 * kC) misc[2 * kC + tid] = first[tid];
  if (tid == 0) mbar_init(smem_u32(bar), 1);
  __syncwarp();
  if (warp == 0) tmem_alloc(smem_u32(slot), kTmemColumns);
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;
  const float* ws1 = misc + 2 * kC;
  const float* wn1 = misc + 3 * kC;
  const float* b1 = misc + 4 * kC;

  const double rho_d = input_rms(n, sum2);
  const float rho = static_cast<float>(rho_d);
  const float inv_rho = rho_d > 0.0 ? static_cast<float>(1.0 / rho_d) : 0.0f;
  const uint64_t adesc = sw128_desc(smem_u32(tile_a));
  const uint64_t bdesc = sw128_desc(smem_u32(tile_b));
  const uint32_t bar_addr = smem_u32(bar);
  const int tiles = (n + kTile - 1) / kTile;
  const int r = tid >> 1, half = tid & 1;  // the tile row and channel half this thread gathers
  const int c0 = 16 * half;
  uint32_t phase = 0;
  bool failed = false;

  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int i = tile * kTile + r;
    float m[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) m[k] = 0.0f;
    uint4 own[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
    if (i < n) {
      const int start = rows[i], end = rows[i + 1];
      if constexpr (kLift) {
        const float2 p = uv[i];
        const float u = p.x * inv_rho, v = p.y * inv_rho;
        float h[16];
#pragma unroll
        for (int k = 0; k < 16; ++k)
          h[k] = fmaxf(fmaf(ws1[c0 + k], u, fmaf(wn1[c0 + k], v, b1[c0 + k])), 0.0f);
        own[0] = pack8(h);
        own[1] = pack8(h + 8);
        for (int j0 = start; j0 < end; j0 += kBatch<kLift>) {
          int cc[kBatch<kLift>];
          float ww[kBatch<kLift>];
          float2 q[kBatch<kLift>];
#pragma unroll
          for (int k = 0; k < kBatch<kLift>; ++k) {
            const int j = j0 + k;
            cc[k] = j < end ? cols[j] : i;
            ww[k] = j < end ? edge[j] : 0.0f;
          }
#pragma unroll
          for (int k = 0; k < kBatch<kLift>; ++k)
            q[k] = (cc[k] != i && ww[k] != 0.0f) ? uv[cc[k]] : make_float2(0.0f, 0.0f);
#pragma unroll
          for (int k = 0; k < kBatch<kLift>; ++k) {
            if (cc[k] == i || ww[k] == 0.0f) continue;
            const float uj = q[k].x * inv_rho, vj = q[k].y * inv_rho;
#pragma unroll
            for (int c = 0; c < 16; ++c)
              m[c] = fmaf(ww[k], fmaxf(fmaf(ws1[c0 + c], uj, fmaf(wn1[c0 + c], vj, b1[c0 + c])), 0.0f),
                          m[c]);
          }
        }
      } else {
        const uint4* self = hin + static_cast<std::size_t>(i) * 4 + half * 2;
        own[0] = __ldg(self);
        own[1] = __ldg(self + 1);
        for (int j0 = start; j0 < end; j0 += kBatch<kLift>) {
          int cc[kBatch<kLift>];
          float ww[kBatch<kLift>];
          uint4 qa[kBatch<kLift>], qb[kBatch<kLift>];
#pragma unroll
          for (int k = 0; k < kBatch<kLift>; ++k) {
            const int j = j0 + k;
            cc[k] = j < end ? cols[j] : i;
            ww[k] = j < end ? edge[j] : 0.0f;
          }
#pragma unroll
          for (int k = 0; k < kBatch<kLift>; ++k) {
            if (cc[k] != i && ww[k] != 0.0f) {
              const uint4* nb = hin + static_cast<std::size_t>(cc[k]) * 4 + half * 2;
              qa[k] = __ldg(nb);
              qb[k] = __ldg(nb + 1);
            } else {
              qa[k] = make_uint4(0, 0, 0, 0);
              qb[k] = qa[k];
            }
          }
#pragma unroll
          for (int k = 0; k < kBatch<kLift>; ++k) {
            const float w = (cc[k] != i) ? ww[k] : 0.0f;
            accumulate8(w, qa[k], m);
            accumulate8(w, qb[k], m + 8);
          }
        }
      }
    }
    // Row r: H chunks 2h, 2h+1 (channels 16h..16h+15), W H chunks 4+2h, 5+2h.
    *reinterpret_cast<uint4*>(tile_a + sw128_offset(r, 2 * half)) = own[0];
    *reinterpret_cast<uint4*>(tile_a + sw128_offset(r, 2 * half + 1)) = own[1];
    *reinterpret_cast<uint4*>(tile_a + sw128_offset(r, 4 + 2 * half)) = pack8(m);
    *reinterpret_cast<uint4*>(tile_a + sw128_offset(r, 5 + 2 * half)) = pack8(m + 8);
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int k = 0; k < kWidth / 16; ++k)
        mma_bf16(tmem, adesc + 2 * k, bdesc + 2 * k, k > 0 ? 1u : 0u);
      mma_commit(bar_addr);
    }
    const bool done = mbar_wait(bar_addr, phase, first_polls);
    if (__syncthreads_or(!done)) {
      failed = true;
      break;
    }
    phase ^= 1u;
    tc_fence_after();
    if (warp < 4) {
      float acc[32];
      tmem_load32(tmem + (static_cast<uint32_t>(warp * 32) << 16), acc);
      const int row = tile * kTile + warp * 32 + lane;
      if constexpr (kLift) {
        float o[32];
#pragma unroll
        for (int c = 0; c < kC; ++c) o[c] = fmaxf(acc[c] + misc[c], 0.0f);
        if (row < n) {
          uint4* dst = hout + static_cast<std::size_t>(row) * 4;
#pragma unroll
          for (int k = 0; k < 4; ++k) dst[k] = pack8(o + 8 * k);
        }
      } else {
        float v = 0.0f;
#pragma unroll
        for (int c = 0; c < kC; ++c) v = fmaf(misc[kC + c], fmaxf(acc[c] + misc[c], 0.0f), v);
        if (row < n) z[row] = (beta != 0.0f ? beta * z[row] : 0.0f) + rho * node_scale[row] * v;
      }
    }
    tc_fence_before();
  }
  if (failed) {
    if (tid == 0) atomicOr(fault, 1);
    mbar_wait(bar_addr, phase, kSpinLimit);  // the late MMA, once more (full bound)
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemColumns);
  }
}

// ---- backward of a 32-wide layer on the tensor cores ------------------------
// Layer: out = relu(Ws H + Wn M + b), H and M n x 32 (M = W H), FP32 saved
// activations. With G = dOut * (out > 0) (n x 32):
//   dH = G Ws and dM = G Wn (rows i: dH_i[k] = sum_c Ws[c][k] G_i[c]),
//   dWs = G^T H, dWn = G^T M, db = sum_i G_i.
// A CTA of 256 threads owns one 128-row tile at a time and issues two GEMMs:
//   1. D1 (128 x 64) = [G | 0] B1^T with B1[n][c] = Ws[c][n] (n < 32) or
//      Wn[c][n - 32]: the tile's [dH | dM], read back by warps 0-3 and
//      stored in FP32 (K = 32: two K = 16 steps of the 64-wide layout);
//   2. D2 (128 x 32) += A2 B2^T with A2 = [H | M | 1]^T (M-rows: 32 channels
//      of H, 32 of M, a row of ones; K = the tile's 128 rows in two 64-wide
//      blocks) and B2 = G^T: accumulated in tensor memory over all the CTA's
//      tiles, so D2 rows hold dWs^T, dWn^T and db. At the end warps 0-2 write
//      the CTA's 65 x 32 partial sums; gnn_dense_back_reduce adds the CTAs'
//      partials in block order.
// Both GEMMs use the forward's operand layout: K-major, 128-byte rows,
// 128-byte swizzle, BF16 operands, FP32 accumulators, M = 128. Waits are
// bounded as in the forward.
constexpr int kBackThreads = 256;
constexpr int kBackA1 = 0;                     // [G | 0]: 128 rows x 128 B
constexpr int kBackB1 = kBackA1 + 16384;       // [Ws | Wn]^T: 64 rows x 128 B
constexpr int kBackA2 = kBackB1 + 8192;        // two K-blocks of 128 rows x 128 B
constexpr int kBackB2 = kBackA2 + 2 * 16384;   // two K-blocks of 32 rows x 128 B
constexpr int kBackTiles = kBackB2 + 2 * 4096;  // 64 KB of operand tiles
constexpr int kBackSmem = 1024 + kBackTiles + 16;
constexpr uint32_t kBackColumns = 128;         // D1: columns 0-63, D2: 64-95
constexpr int kBackPartialRows = 65;           // dWs^T (32), dWn^T (32), db (1)
// M = 128, N = 64 (D1).
constexpr uint32_t kIdescN64 = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) |
                               ((static_cast<uint32_t>(kTile) >> 4) << 24);

__device__ __forceinline__ void store_bf16(uint8_t* p, float v) {
  *reinterpret_cast<__nv_bfloat16*>(p) = __float2bfloat16_rn(v);
}

__global__ void __launch_bounds__(kBackThreads, 2)
    k_gnn_dense_back_tc(int n, const float* __restrict__ H, const float* __restrict__ M,
                        const float* __restrict__ out, const float* __restrict__ dOut,
                        const float* __restrict__ Ws, const float* __restrict__ Wn,
                        float* __restrict__ dH, float* __restrict__ dM,
                        float* __restrict__ partials, int* __restrict__ fault) {
  extern __shared__ uint8_t raw[];
  const uint32_t pad = (1024u - (smem_u32(raw) & 1023u)) & 1023u;
  uint8_t* base = raw + pad;
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + kBackTiles);
  uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  {  // B1 row n (output channel of [dH | dM]), chunk q < 4 (8 input channels).
    const int nrow = tid >> 2, q = tid & 3;
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int c = 8 * q + k;
      v[k] = nrow < kC ? Ws[c * kC + nrow] : Wn[c * kC + nrow - kC];
    }
    *reinterpret_cast<uint4*>(base + kBackB1 + sw128_offset(nrow, q)) = pack8(v);
  }
  // Rows 65-127 of both A2 blocks stay zero (they only feed D2 rows that are
  // never read).
  for (int k = tid; k < 2 * 63 * 8; k += kBackThreads) {
    const int blk = k / (63 * 8), rest = k % (63 * 8);
    *reinterpret_cast<uint4*>(base + kBackA2 + blk * 16384 + sw128_offset(65 + rest / 8, rest % 8)) =
        make_uint4(0, 0, 0, 0);
  }
  if (tid == 0) mbar_init(smem_u32(bar), 1);
  __syncwarp();
  if (warp == 0) tmem_alloc(smem_u32(slot), kBackColumns);
  proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;
  const uint32_t d1 = tmem, d2 = tmem + 64;
  const uint64_t a1 = sw128_desc(smem_u32(base + kBackA1));
  const uint64_t b1 = sw128_desc(smem_u32(base + kBackB1));
  const uint32_t bar_addr = smem_u32(bar);
  const int tiles = (n + kTile - 1) / kTile;
  const int r = tid >> 1, half = tid & 1, c0 = 16 * half;
  const int kb = r >> 6, kk = r & 63, kq = kk >> 3, ke = kk & 7;  // r as a K index of GEMM 2
  uint8_t* a2 = base + kBackA2 + kb * 16384;
  uint8_t* b2 = base + kBackB2 + kb * 4096;
  uint32_t phase = 0;
  bool failed = false, any = false;

  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int i = tile * kTile + r;
    const bool valid = i < n;
    float g[16], h[16], m[16];
    if (valid) {
      const std::size_t row = static_cast<std::size_t>(i) * kC + c0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float4 o = *reinterpret_cast<const float4*>(out + row + 4 * q);
        const float4 d = *reinterpret_cast<const float4*>(dOut + row + 4 * q);
        const float4 hv = *reinterpret_cast<const float4*>(H + row + 4 * q);
        const float4 mv = *reinterpret_cast<const float4*>(M + row + 4 * q);
        g[4 * q] = o.x > 0.0f ? d.x : 0.0f;
        g[4 * q + 1] = o.y > 0.0f ? d.y : 0.0f;
        g[4 * q + 2] = o.z > 0.0f ? d.z : 0.0f;
        g[4 * q + 3] = o.w > 0.0f ? d.w : 0.0f;
        h[4 * q] = hv.x;
        h[4 * q + 1] = hv.y;
        h[4 * q + 2] = hv.z;
        h[4 * q + 3] = hv.w;
        m[4 * q] = mv.x;
        m[4 * q + 1] = mv.y;
        m[4 * q + 2] = mv.z;
        m[4 * q + 3] = mv.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) g[k] = h[k] = m[k] = 0.0f;
    }
    // GEMM 1 operand: row r, K chunks 2 half and 2 half + 1 (channels c0..c0+15).
    *reinterpret_cast<uint4*>(base + kBackA1 + sw128_offset(r, 2 * half)) = pack8(g);
    *reinterpret_cast<uint4*>(base + kBackA1 + sw128_offset(r, 2 * half + 1)) = pack8(g + 8);
    // GEMM 2 operands, transposed: element (channel, r) of A2 and B2.
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int c = c0 + k;
      store_bf16(a2 + sw128_offset(c, kq) + 2 * ke, h[k]);
      store_bf16(a2 + sw128_offset(kC + c, kq) + 2 * ke, m[k]);
      store_bf16(b2 + sw128_offset(c, kq) + 2 * ke, g[k]);
    }
    if (half == 0) store_bf16(a2 + sw128_offset(2 * kC, kq) + 2 * ke, valid ? 1.0f : 0.0f);
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int k = 0; k < 2; ++k) mma_bf16(d1, a1 + 2 * k, b1 + 2 * k, k > 0 ? 1u : 0u, kIdescN64);
#pragma unroll
      for (int blk = 0; blk < 2; ++blk) {
        const uint64_t a2d = sw128_desc(smem_u32(base + kBackA2 + blk * 16384));
        const uint64_t b2d = sw128_desc(smem_u32(base + kBackB2 + blk * 4096));
#pragma unroll
        for (int k = 0; k < 4; ++k)
          mma_bf16(d2, a2d + 2 * k, b2d + 2 * k, (any || blk > 0 || k > 0) ? 1u : 0u);
      }
      mma_commit(bar_addr);
    }
    any = true;
    const bool done = mbar_wait(bar_addr, phase, kSpinLimit);
    if (__syncthreads_or(!done)) {
      failed = true;
      break;
    }
    phase ^= 1u;
    tc_fence_after();
    if (warp < 4) {
      float acc[32];
      const uint32_t lanes = static_cast<uint32_t>(warp * 32) << 16;
      const int row = tile * kTile + warp * 32 + lane;
      tmem_load32(d1 + lanes, acc);
      if (row < n) {
        float4* dst = reinterpret_cast<float4*>(dH + static_cast<std::size_t>(row) * kC);
#pragma unroll
        for (int q = 0; q < 8; ++q)
          dst[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
      }
      tmem_load32(d1 + lanes + 32, acc);
      if (row < n) {
        float4* dst = reinterpret_cast<float4*>(dM + static_cast<std::size_t>(row) * kC);
#pragma unroll
        for (int q = 0; q < 8; ++q)
          dst[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
      }
    }
    tc_fence_before();
  }
  if (failed) {
    if (tid == 0) atomicOr(fault, 1);
    mbar_wait(bar_addr, phase, kSpinLimit);  // the late MMAs, once more (full bound)
  } else if (warp < 3) {
    // This CTA's partial sums: D2 rows 0-64, 32 columns (zeros if it had no tile).
    tc_fence_after();
    float acc[32];
    const int mrow = warp * 32 + lane;
    if (any) {
      tmem_load32(d2 + (static_cast<uint32_t>(warp * 32) << 16), acc);
    } else {
#pragma unroll
      for (int k = 0; k < 32; ++k) acc[k] = 0.0f;
    }
    if (mrow < kBackPartialRows) {
      float* dst = partials + (static_cast<std::size_t>(blockIdx.x) * kBackPartialRows + mrow) * kC;
#pragma unroll
      for (int k = 0; k < 32; ++k) dst[k] = acc[k];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kBackColumns);
  }
}

// dWs[c][k] += sum_b P_b[k][c], dWn[c][k] += sum_b P_b[32 + k][c], db[c] +=
// sum_b P_b[64][c], blocks in order.
__global__ void k_gnn_dense_back_reduce(int blocks, const float* __restrict__ partials,
                                        float* __restrict__ dWs, float* __restrict__ dWn,
                                        float* __restrict__ db) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kBackPartialRows * kC) return;
  const int mrow = e / kC, c = e % kC;
  float sum = 0.0f;
  for (int b = 0; b < blocks; ++b)
    sum += partials[(static_cast<std::size_t>(b) * kBackPartialRows + mrow) * kC + c];
  if (mrow < kC) dWs[c * kC + mrow] += sum;
  else if (mrow < 2 * kC) dWn[c * kC + mrow - kC] += sum;
  else db[c] += sum;
}

int back_grid(int n) {
  const int tiles = (n + kTile - 1) / kTile;
  return std::max(1, std::min(tiles, kSms * 2));
}

// The poll count of each tile's first wait for its MMA: kSpinLimit unless a
// test asked for fewer (0..kSpinLimit).
long long wait_polls(long long requested) {
  return requested < 0 || requested > kSpinLimit ? kSpinLimit : requested;
}

int tc_grid(int n) {
  const int tiles = (n + kTile - 1) / kTile;
  return std::max(1, std::min(tiles, kSms * kTcPerSm));
}

}  // namespace

namespace launch {

int gnn_back_partials_floats() { return kSms * 2 * kBackPartialRows * kC; }

void gnn_dense_back_tc(int n, const float* H, const float* M, const float* out,
                       const float* dOut, const float* Ws, const float* Wn, float* dH, float* dM,
                       float* dWs, float* dWn, float* db, float* partials, int* fault,
                       cudaStream_t s) {
  if (n <= 0) return;
  static std::atomic<unsigned long long> raised{0};
  raise_shared_limit(reinterpret_cast<const void*>(k_gnn_dense_back_tc), kBackSmem, raised);
  counter += 2;
  const int blocks = back_grid(n);
  k_gnn_dense_back_tc<<<blocks, kBackThreads, kBackSmem, s>>>(n, H, M, out, dOut, Ws, Wn, dH, dM,
                                                               partials, fault);
  k_gnn_dense_back_reduce<<<(kBackPartialRows * kC + kBlock - 1) / kBlock, kBlock, 0, s>>>(
      blocks, partials, dWs, dWn, db);
}

void gnn_lift(int n, const int* rows, const int* cols, const float* lift, const float* t,
              const float* node_scale, float2* uv, DeviceReducer red, double* sum2,
              cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_lift<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, lift, t, node_scale, uv, red, sum2);
}

void gnn_layer_a(int n, const int* rows, const int* cols, const float* edge, const float2* uv,
                 const float* first, const float* ws, const float* wn, const float* bias,
                 const double* sum2, unsigned short* hout, int* fault, long long first_polls,
                 cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_layer_tc<true><<<tc_grid(n), kTcThreads, kTcSmem, s>>>(
      n, rows, cols, edge, uv, nullptr, first, ws, wn, bias, nullptr, nullptr, sum2,
      reinterpret_cast<uint4*>(hout), nullptr, 0.0f, fault, wait_polls(first_polls));
}

void gnn_layer_b(int n, const int* rows, const int* cols, const float* edge,
                 const unsigned short* hin, const float* ws, const float* wn, const float* bias,
                 const float* wo, const float* node_scale, const double* sum2, float* z,
                 float beta, int* fault, long long first_polls, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_layer_tc<false><<<tc_grid(n), kTcThreads, kTcSmem, s>>>(
      n, rows, cols, edge, nullptr, reinterpret_cast<const uint4*>(hin), nullptr, ws, wn, bias,
      wo, node_scale, sum2, nullptr, z, beta, fault, wait_polls(first_polls));
}

}  // namespace launch
}  // namespace kb2
