// The small coarse levels of the mixed-precision V-cycle in one launch (no
// reference counterpart).
//
// Below about sixteen thousand rows a level's kernels are latency-bound: each
// sweep, residual, restriction or prolongation costs a launch and a few
// microseconds whatever its size. Here one thread-block cluster (16 CTAs of
// 1024 threads where the device allows, else 8) runs the whole V-cycle of
// those levels, with a cluster barrier between dependent steps.
//
// Each CTA owns a power-of-two chunk of rows per level. The level vectors stay
// in global memory, where they are L2-resident: values written during the
// launch are read with L2-only loads, which keeps them coherent across the
// cluster's SMs (for these scattered gathers L2 measured faster than reading
// other CTAs' shared memory), while the operators, constant during the launch,
// are read through the read-only cache, where a CTA's rows stay between steps.
//
// Steps are merged where no neighbour value is needed: the zero-start sweep of
// a level is done by whoever writes its right-hand side (the first step, or
// the restriction), and every CTA solves the dense coarsest level itself, so
// the prolongation from it reads the correction from the CTA's own shared
// memory.
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

// sum_j a_ij x_j of row i with the BF16 operator (without the row scale). The
// entries are taken eight at a time, their neighbour values all requested
// before any is used, so a thread keeps several loads in flight.
__device__ __forceinline__ float row_product(const TailLevel& l, const float* x, int i) {
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
    float v[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) v[u] = c[u] >= 0 ? __ldcg(x + c[u]) : 0.0f;
#pragma unroll
    for (int u = 0; u < kBatch; ++u) acc = fmaf(a[u], v[u], acc);
  }
  return acc;
}

// next = x + omega inv (b - A x) on the owned rows.
__device__ void sweep(const TailLevel& l, int rank, const float* x, float* next) {
  const Rows own = owned(l, rank);
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int i = own.base + k;
    const float r = __ldcg(l.bg + i) - __ldg(l.scale + i) * row_product(l, x, i);
    __stcg(next + i, __ldcg(x + i) + kOmega * __ldg(l.inv + i) * r);
  }
}

__device__ void residual(const TailLevel& l, int rank, const float* x, float* r) {
  const Rows own = owned(l, rank);
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int i = own.base + k;
    __stcg(r + i, __ldcg(l.bg + i) - __ldg(l.scale + i) * row_product(l, x, i));
  }
}

// Coarse b = Kahan sum of the fine residual over each aggregate's members, in
// member order; with `zero`, also the coarse zero-start sweep x = omega inv b.
__device__ void restrict_to(const TailLevel& fine, const float* r, const TailLevel& coarse,
                            float* coarse_x, bool zero, int rank) {
  const Rows own = owned(coarse, rank);
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int g = own.base + k;
    float sum = 0.0f, error = 0.0f;
    const int end = __ldg(fine.offsets + g + 1);
    for (int j0 = __ldg(fine.offsets + g); j0 < end; j0 += kBatch) {
      int m[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) m[u] = j0 + u < end ? __ldg(fine.members + j0 + u) : -1;
      float v[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) v[u] = m[u] >= 0 ? __ldcg(r + m[u]) : 0.0f;
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        if (m[u] < 0) break;
        const float term = v[u] - error;
        const float next = sum + term;
        error = (next - sum) - term;
        sum = next;
      }
    }
    __stcg(coarse.bg + g, sum);
    if (zero) __stcg(coarse_x + g, kOmega * __ldg(coarse.inv + g) * sum);
  }
}

// x += e[aggregate] on the owned rows; e in global memory or, for the dense
// coarsest, in this CTA's shared memory.
__device__ void prolong(const TailLevel& fine, float* x, const float* e, bool e_shared, int rank) {
  const Rows own = owned(fine, rank);
  for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
    const int i = own.base + k;
    const int g = __ldg(fine.aggregate + i);
    if (g >= 0) __stcg(x + i, __ldcg(x + i) + (e_shared ? e[g] : __ldcg(e + g)));
  }
}

// The whole coarsest solution x = W b with the dense FP64 inverse, into this
// CTA's shared memory (every CTA computes it): b gathered first, then a warp
// per row.
__device__ void dense_solve(float* shared, const TailLevel& l, const double* W, int gathered,
                            int solution) {
  for (int k = threadIdx.x; k < l.n; k += blockDim.x) shared[gathered + k] = __ldcg(l.bg + k);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  for (int i = warp; i < l.n; i += warps) {
    const double* row = W + static_cast<std::size_t>(i) * l.n;
    double acc = 0.0;
    for (int c = lane; c < l.n; c += 32) acc += row[c] * static_cast<double>(shared[gathered + c]);
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if (lane == 0) shared[solution + i] = static_cast<float>(acc);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kTailThreads)
    k_tail_cycle(const __grid_constant__ TailPlan p, const int* __restrict__ status) {
  dev::pdl_entry();
  // Uniform across the cluster: nothing else writes status while this runs.
  if (status[0] != 0) return;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ float shared[];
  const int rank = static_cast<int>(cluster.block_rank());
  const int last = p.levels - 1;
  const bool dense = p.dense != nullptr;
  // Current iterate and spare buffer of each level (uniform across threads).
  float* x[kMaxTailLevels];
  float* spare[kMaxTailLevels];
  for (int l = 0; l < p.levels; ++l) {
    x[l] = p.level[l].xg;
    spare[l] = p.level[l].rg;
  }
  // The first tail level swaps roles (pre - 1) + post times; start so that its
  // result ends in xg, the buffer the caller reads.
  if (((p.pre - 1 + p.post) & 1) != 0) {
    x[0] = p.level[0].rg;
    spare[0] = p.level[0].xg;
  }
  {
    // Zero-start sweep of the first tail level from its right-hand side.
    const TailLevel& L = p.level[0];
    const Rows own = owned(L, rank);
    for (int k = threadIdx.x; k < own.count; k += blockDim.x) {
      const int i = own.base + k;
      __stcg(x[0] + i, kOmega * __ldg(L.inv + i) * __ldcg(L.bg + i));
    }
  }
  cluster.sync();
  for (int l = 0; l < last; ++l) {
    const TailLevel& L = p.level[l];
    for (int s = 1; s < p.pre; ++s) {
      sweep(L, rank, x[l], spare[l]);
      cluster.sync();
      float* t = x[l];
      x[l] = spare[l];
      spare[l] = t;
    }
    residual(L, rank, x[l], spare[l]);
    cluster.sync();
    const bool coarse_sweeps = l + 1 < last || !dense;
    restrict_to(L, spare[l], p.level[l + 1], x[l + 1], coarse_sweeps, rank);
    cluster.sync();
  }
  const float* correction = nullptr;  // coarsest solution, when in shared memory
  if (dense) {
    dense_solve(shared, p.level[last], p.dense, p.gathered, p.solution);
    correction = shared + p.solution;
  } else {
    // x[last] holds the zero-start sweep (written with the restriction).
    for (int s = 1; s < p.coarse_sweeps; ++s) {
      sweep(p.level[last], rank, x[last], spare[last]);
      cluster.sync();
      float* t = x[last];
      x[last] = spare[last];
      spare[last] = t;
    }
  }
  for (int l = last - 1; l >= 0; --l) {
    const TailLevel& L = p.level[l];
    const bool from_shared = l + 1 == last && correction != nullptr;
    prolong(L, x[l], from_shared ? correction : x[l + 1], from_shared, rank);
    cluster.sync();
    for (int s = 0; s < p.post; ++s) {
      sweep(L, rank, x[l], spare[l]);
      // After the last sweep nothing in this launch reads another CTA's rows.
      if (l > 0 || s + 1 < p.post) cluster.sync();
      float* t = x[l];
      x[l] = spare[l];
      spare[l] = t;
    }
  }
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
