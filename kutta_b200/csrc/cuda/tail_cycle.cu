// The small coarse levels of the mixed-precision V-cycle in one launch (no
// reference counterpart).
//
// Below about sixteen thousand rows a level's kernels are latency-bound: each
// sweep, residual, restriction or prolongation costs a launch and a few
// microseconds whatever its size. Here one thread-block cluster (16 CTAs of
// 1024 threads where the device allows, else 8) runs the whole V-cycle of
// those levels, with a cluster barrier between dependent steps.
//
// Each CTA owns a power-of-two chunk of rows per level and keeps, in its own
// shared memory, a full copy of every level vector that rows gather from (the
// iterate, and the residual the restriction sums). A step computes the owned
// rows from the local copies and pushes each new value into every CTA's copy
// with distributed-shared-memory stores; the cluster barrier that follows
// makes them visible. So every gather is a local shared-memory read, and the
// only traffic between SMs is one posted store per row and CTA per step. The
// operators, constant during the launch, are read through the read-only
// cache; each CTA reads only its own rows of them.
//
// The first tail level's right-hand side comes from global memory and its
// result goes back there; nothing else in between leaves the cluster. The
// zero-start sweep of a level is done by whoever writes its right-hand side
// (the first step, or the restriction), and every CTA solves the dense
// coarsest level itself, so its solution needs no exchange.
#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.hpp"

namespace kb2 {
namespace {
namespace cg = cooperative_groups;
using launch::kMaxTailLevels;
using launch::TailLevel;
using launch::TailPlan;

constexpr int kTailThreads = 1024;
constexpr int kBatch = 8;
constexpr float kOmega = 2.0f / 3.0f;

__device__ __forceinline__ float bf(unsigned short v) {
  return __bfloat162float(__ushort_as_bfloat16(v));
}

struct Rows {
  int base, count;
};
__device__ __forceinline__ Rows owned(const TailLevel& l, int rank) {
  const int base = rank << l.shift;
  return Rows{base, max(0, min(1 << l.shift, l.n - base))};
}

// sum_j a_ij v_j of row i with the BF16 operator (without the row scale), v
// a full copy in this CTA's shared memory. The entries are taken eight at a
// time, their columns and values all requested before any is used.
__device__ __forceinline__ float row_product(const TailLevel& l, const float* v, int i) {
  float acc = 0.0f;
  const int end = __ldg(l.rows + i + 1);
  for (int j0 = __ldg(l.rows + i); j0 < end; j0 += kBatch) {
    int c[kBatch];
    float a[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      c[u] = j0 + u < end ? __ldg(l.cols + j0 + u) : -1;
      a[u] = j0 + u < end ? bf(__ldg(l.v16 + j0 + u)) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) acc = fmaf(a[u], c[u] >= 0 ? v[c[u]] : 0.0f, acc);
  }
  return acc;
}

// Row i's value into every CTA's copy of the vector at shared offset `at`
// (this CTA's own included). Visible to all after the next cluster barrier.
__device__ __forceinline__ void push(cg::cluster_group& cluster, float* shared, int at, int i,
                                     float v, int size) {
  for (int d = 0; d < size; ++d) *cluster.map_shared_rank(shared + at + i, d) = v;
}

// One damped L1-Jacobi sweep of the owned rows, x read from the local copy at
// `from`: the new values pushed to every copy at `to`, or, on the final sweep
// of the first tail level, written to global memory.
__device__ void sweep(cg::cluster_group& cluster, float* shared, const TailLevel& l, int rank,
                      int size, int from, int to, bool final) {
  const Rows own = owned(l, rank);
  const float* x = shared + from;
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int i = own.base + k;
    const float r = shared[l.bs + k] - __ldg(l.scale + i) * row_product(l, x, i);
    const float next = x[i] + kOmega * __ldg(l.inv + i) * r;
    if (final) __stcg(l.xg + i, next);
    else push(cluster, shared, to, i, next, size);
  }
}

__global__ void __launch_bounds__(kTailThreads)
    k_tail_cycle(const __grid_constant__ TailPlan p, const int* __restrict__ status) {
  dev::pdl_entry();
  // Uniform across the cluster: nothing else writes status while this runs.
  if (status[0] != 0) return;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ float shared[];
  const int rank = static_cast<int>(cluster.block_rank());
  const int size = static_cast<int>(cluster.num_blocks());
  const int last = p.levels - 1;
  const bool dense = p.dense != nullptr;
  // Shared offsets of each level's current iterate copy and of its spare copy
  // (the residual, or the next sweep's iterate). Uniform across the cluster.
  int x[kMaxTailLevels], spare[kMaxTailLevels];
  for (int l = 0; l < p.levels; ++l) {
    x[l] = p.level[l].xs;
    spare[l] = p.level[l].rs;
  }
  {
    // The first tail level's right-hand side (owned rows) and its zero-start
    // sweep.
    const TailLevel& L = p.level[0];
    const Rows own = owned(L, rank);
    for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
      const int i = own.base + k;
      const float b = __ldcg(L.bg + i);
      shared[L.bs + k] = b;
      push(cluster, shared, x[0], i, kOmega * __ldg(L.inv + i) * b, size);
    }
  }
  cluster.sync();
  for (int l = 0; l < last; ++l) {
    const TailLevel& L = p.level[l];
    for (int s = 1; s < p.pre; ++s) {
      sweep(cluster, shared, L, rank, size, x[l], spare[l], false);
      cluster.sync();
      const int t = x[l];
      x[l] = spare[l];
      spare[l] = t;
    }
    {
      // Residual of the owned rows into every copy of the spare vector.
      const Rows own = owned(L, rank);
      for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
        const int i = own.base + k;
        push(cluster, shared, spare[l], i,
             shared[L.bs + k] - __ldg(L.scale + i) * row_product(L, shared + x[l], i), size);
      }
    }
    cluster.sync();
    {
      // Coarse b = Kahan sum of the residual over each owned aggregate's
      // members, in member order; then the coarse zero-start sweep, or, for
      // the dense coarsest, b itself into every CTA's copy.
      const TailLevel& C = p.level[l + 1];
      const bool to_dense = l + 1 == last && dense;
      const Rows own = owned(C, rank);
      const float* r = shared + spare[l];
      for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
        const int g = own.base + k;
        float sum = 0.0f, error = 0.0f;
        const int end = __ldg(L.offsets + g + 1);
        for (int j0 = __ldg(L.offsets + g); j0 < end; j0 += kBatch) {
          int m[kBatch];
#pragma unroll
          for (int u = 0; u < kBatch; ++u) m[u] = j0 + u < end ? __ldg(L.members + j0 + u) : -1;
#pragma unroll
          for (int u = 0; u < kBatch; ++u) {
            if (m[u] < 0) break;
            const float term = r[m[u]] - error;
            const float next = sum + term;
            error = (next - sum) - term;
            sum = next;
          }
        }
        shared[C.bs + k] = sum;
        if (to_dense) push(cluster, shared, C.rs, g, sum, size);
        else push(cluster, shared, x[l + 1], g, kOmega * __ldg(C.inv + g) * sum, size);
      }
    }
    cluster.sync();
  }
  if (dense) {
    // Every CTA: the whole coarsest solution x = W b with the dense FP64
    // inverse, a warp per row, into its own copy.
    const TailLevel& C = p.level[last];
    const float* b = shared + C.rs;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (int i = warp; i < C.n; i += warps) {
      const double* row = p.dense + static_cast<std::size_t>(i) * C.n;
      double acc = 0.0;
      for (int c = lane; c < C.n; c += 32) acc += __ldg(row + c) * static_cast<double>(b[c]);
      for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
      if (lane == 0) shared[x[last] + i] = static_cast<float>(acc);
    }
    __syncthreads();
  } else {
    // x[last] holds the zero-start sweep (pushed with the restriction).
    for (int s = 1; s < p.coarse_sweeps; ++s) {
      sweep(cluster, shared, p.level[last], rank, size, x[last], spare[last], false);
      cluster.sync();
      const int t = x[last];
      x[last] = spare[last];
      spare[last] = t;
    }
  }
  for (int l = last - 1; l >= 0; --l) {
    const TailLevel& L = p.level[l];
    {
      // x += e[aggregate] on the owned rows, e the coarser level's result
      // (every CTA holds all of it), into every copy.
      const Rows own = owned(L, rank);
      const float* e = shared + x[l + 1];
      for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
        const int i = own.base + k;
        const int g = __ldg(L.aggregate + i);
        const float xi = shared[x[l] + i];
        push(cluster, shared, x[l], i, g >= 0 ? xi + e[g] : xi, size);
      }
    }
    cluster.sync();
    for (int s = 0; s < p.post; ++s) {
      const bool final = l == 0 && s + 1 == p.post;
      sweep(cluster, shared, L, rank, size, x[l], spare[l], final);
      if (final) break;
      cluster.sync();
      const int t = x[l];
      x[l] = spare[l];
      spare[l] = t;
    }
  }
  // The last cluster barrier above followed the last store into another CTA's
  // shared memory, so every CTA may exit now.
}

// The attribute is per function, shared by every solver on the device, so it
// is always the ceiling; each launch asks for its own plan's size.
cudaError_t configure(int cluster) {
  cudaError_t e = cudaFuncSetAttribute(k_tail_cycle, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       launch::kTailSharedBytes);
  if (e != cudaSuccess) return e;
  if (cluster > 8)
    e = cudaFuncSetAttribute(k_tail_cycle, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

cudaLaunchConfig_t config_for(const TailPlan& p, cudaLaunchAttribute* attr, cudaStream_t s) {
  cudaLaunchConfig_t c = {};
  c.gridDim = dim3(static_cast<unsigned>(p.cluster), 1, 1);
  c.blockDim = dim3(kTailThreads, 1, 1);
  c.dynamicSmemBytes = static_cast<std::size_t>(p.smem_bytes);
  c.stream = s;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = static_cast<unsigned>(p.cluster);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  // Programmatic dependent launch, as for every solve-path kernel (common.cuh).
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  c.attrs = attr;
  c.numAttrs = dev::pdl_enabled() ? 2 : 1;
  return c;
}

}  // namespace

namespace launch {

bool tail_cluster_fits(int cluster, int smem_bytes) {
  if (smem_bytes > kTailSharedBytes || configure(cluster) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  TailPlan probe{};
  probe.cluster = cluster;
  probe.smem_bytes = smem_bytes;
  cudaLaunchAttribute attr[2];
  cudaLaunchConfig_t c = config_for(probe, attr, nullptr);
  int count = 0;
  if (cudaOccupancyMaxActiveClusters(&count, k_tail_cycle, &c) == cudaSuccess && count > 0)
    return true;
  cudaGetLastError();
  return false;
}

void tail_cycle(const TailPlan& plan, const int* status, cudaStream_t s) {
  ++counter;
  cudaLaunchAttribute attr[2];
  cudaLaunchConfig_t c = config_for(plan, attr, s);
  cudaLaunchKernelEx(&c, k_tail_cycle, plan, status);
}

}  // namespace launch
}  // namespace kb2
