// The small coarse levels of the mixed-precision V-cycle in one launch (no
// reference counterpart).
//
// Below about sixteen thousand rows a level's kernels are latency-bound: each
// sweep, residual, restriction or prolongation costs a launch and a few
// microseconds whatever its size. Here one thread-block cluster (16 CTAs of
// 1024 threads where the device allows, else 8) runs the whole V-cycle of
// those levels. Each CTA owns a power-of-two chunk of rows per level and keeps
// that chunk's x, r and b in its shared memory; a row's neighbours are read
// from whichever CTA owns them through distributed shared memory, and each
// step ends with a cluster barrier. The operators are the BF16 copies with
// row scales, read from global memory (they stay in L2).
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

__device__ __forceinline__ float bf(unsigned short v) {
  return __bfloat162float(__ushort_as_bfloat16(v));
}

// Value j of a level vector whose chunks start at `offset` in every CTA's
// shared memory.
__device__ __forceinline__ float remote(cg::cluster_group& cluster, float* shared, int offset,
                                        int shift, int j) {
  const int owner = j >> shift;
  const int local = j & ((1 << shift) - 1);
  return *cluster.map_shared_rank(shared + offset + local, owner);
}

struct Rows {
  int base, count;
};
__device__ __forceinline__ Rows owned(const TailLevel& l, int rank) {
  const int base = rank << l.shift;
  return Rows{base, max(0, min(1 << l.shift, l.n - base))};
}

// sum_j a_ij x_j with the BF16 operator (without the row scale). Columns and
// values are loaded eight at a time before the neighbour reads, so a thread
// keeps several loads in flight instead of one dependent chain per entry.
__device__ __forceinline__ float row_product(cg::cluster_group& cluster, float* shared,
                                             const TailLevel& l, int x, int i) {
  constexpr int kBatch = 8;
  float acc = 0.0f;
  const int end = l.rows[i + 1];
  for (int j0 = l.rows[i]; j0 < end; j0 += kBatch) {
    int col[kBatch];
    float val[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const bool in = j0 + u < end;
      col[u] = in ? l.cols[j0 + u] : -1;
      val[u] = in ? bf(l.v16[j0 + u]) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u)
      if (col[u] >= 0) acc = fmaf(val[u], remote(cluster, shared, x, l.shift, col[u]), acc);
  }
  return acc;
}

// next = x + (2/3) inv (b - A x); zero: x taken as zero without reading it.
__device__ void sweep(cg::cluster_group& cluster, float* shared, const TailLevel& l, int rank,
                      int x, int next, bool zero) {
  const Rows own = owned(l, rank);
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int i = own.base + k;
    const float b = shared[l.b + k];
    if (zero) {
      shared[next + k] = (2.0f / 3.0f) * l.inv[i] * b;
    } else {
      const float r = b - l.scale[i] * row_product(cluster, shared, l, x, i);
      shared[next + k] = shared[x + k] + (2.0f / 3.0f) * l.inv[i] * r;
    }
  }
}

__device__ void residual(cg::cluster_group& cluster, float* shared, const TailLevel& l, int rank,
                         int x, int r) {
  const Rows own = owned(l, rank);
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int i = own.base + k;
    shared[r + k] = shared[l.b + k] - l.scale[i] * row_product(cluster, shared, l, x, i);
  }
}

// Coarse b = Kahan sum of the fine residual over each aggregate's members.
__device__ void restrict_to(cg::cluster_group& cluster, float* shared, const TailLevel& fine,
                            int r, const TailLevel& coarse, int rank) {
  const Rows own = owned(coarse, rank);
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int g = own.base + k;
    float sum = 0.0f, error = 0.0f;
    for (int j = fine.offsets[g]; j < fine.offsets[g + 1]; ++j) {
      const float term = remote(cluster, shared, r, fine.shift, fine.members[j]) - error;
      const float next = sum + term;
      error = (next - sum) - term;
      sum = next;
    }
    shared[coarse.b + k] = sum;
  }
}

__device__ void prolong_from(cg::cluster_group& cluster, float* shared, const TailLevel& fine,
                             int x, const TailLevel& coarse, int coarse_x, int rank) {
  const Rows own = owned(fine, rank);
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int g = fine.aggregate[own.base + k];
    if (g >= 0) shared[x + k] += remote(cluster, shared, coarse_x, coarse.shift, g);
  }
}

// x = W b with the dense FP64 inverse: b gathered into this CTA first, then a
// warp per owned row.
__device__ void dense_solve(cg::cluster_group& cluster, float* shared, const TailLevel& l,
                            int rank, const double* W, int x, int gathered) {
  for (int k = threadIdx.x; k < l.n; k += blockDim.x)
    shared[gathered + k] = remote(cluster, shared, l.b, l.shift, k);
  __syncthreads();
  const Rows own = owned(l, rank);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  for (int k = warp; k < own.count; k += warps) {
    const double* row = W + static_cast<std::size_t>(own.base + k) * l.n;
    double acc = 0.0;
    for (int c = lane; c < l.n; c += 32) acc += row[c] * static_cast<double>(shared[gathered + c]);
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if (lane == 0) shared[x + k] = static_cast<float>(acc);
  }
}

__global__ void __launch_bounds__(kTailThreads)
    k_tail_cycle(const __grid_constant__ TailPlan p, const float* __restrict__ b_in,
                 float* __restrict__ x_out, const int* __restrict__ status) {
  // Uniform across the cluster: nothing else writes status while this runs.
  if (status[0] != 0) return;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ float shared[];
  const int rank = static_cast<int>(cluster.block_rank());
  const int last = p.levels - 1;
  int x[kMaxTailLevels], spare[kMaxTailLevels];
  for (int l = 0; l < p.levels; ++l) {
    x[l] = p.level[l].x;
    spare[l] = p.level[l].r;
  }
  {
    const Rows own = owned(p.level[0], rank);
    for (int k = threadIdx.x; k < own.count; k += blockDim.x)
      shared[p.level[0].b + k] = b_in[own.base + k];
  }
  cluster.sync();
  for (int l = 0; l < last; ++l) {
    const TailLevel& L = p.level[l];
    sweep(cluster, shared, L, rank, x[l], x[l], true);
    cluster.sync();
    for (int s = 1; s < p.pre; ++s) {
      sweep(cluster, shared, L, rank, x[l], spare[l], false);
      cluster.sync();
      const int t = x[l];
      x[l] = spare[l];
      spare[l] = t;
    }
    residual(cluster, shared, L, rank, x[l], spare[l]);
    cluster.sync();
    restrict_to(cluster, shared, L, spare[l], p.level[l + 1], rank);
    cluster.sync();
  }
  {
    const TailLevel& C = p.level[last];
    if (p.dense) {
      dense_solve(cluster, shared, C, rank, p.dense, x[last], p.gathered);
      cluster.sync();
    } else {
      sweep(cluster, shared, C, rank, x[last], x[last], true);
      cluster.sync();
      for (int s = 1; s < p.coarse_sweeps; ++s) {
        sweep(cluster, shared, C, rank, x[last], spare[last], false);
        cluster.sync();
        const int t = x[last];
        x[last] = spare[last];
        spare[last] = t;
      }
    }
  }
  for (int l = last - 1; l >= 0; --l) {
    const TailLevel& L = p.level[l];
    prolong_from(cluster, shared, L, x[l], p.level[l + 1], x[l + 1], rank);
    cluster.sync();
    for (int s = 0; s < p.post; ++s) {
      sweep(cluster, shared, L, rank, x[l], spare[l], false);
      cluster.sync();
      const int t = x[l];
      x[l] = spare[l];
      spare[l] = t;
    }
  }
  {
    const Rows own = owned(p.level[0], rank);
    for (int k = threadIdx.x; k < own.count; k += blockDim.x)
      x_out[own.base + k] = shared[x[0] + k];
  }
  // No CTA leaves while another may still read its shared memory.
  cluster.sync();
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
  c.attrs = attr;
  c.numAttrs = 1;
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
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t c = config_for(probe, attr, nullptr);
  int count = 0;
  if (cudaOccupancyMaxActiveClusters(&count, k_tail_cycle, &c) == cudaSuccess && count > 0)
    return true;
  cudaGetLastError();
  return false;
}

void tail_cycle(const TailPlan& plan, const float* b, float* x, const int* status,
                cudaStream_t s) {
  ++counter;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t c = config_for(plan, attr, s);
  cudaLaunchKernelEx(&c, k_tail_cycle, plan, b, x, status);
}

}  // namespace launch
}  // namespace kb2
