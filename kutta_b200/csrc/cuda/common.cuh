// Device helpers shared by the solver kernels.
//
// Everything here that feeds the plain (reference-parity) solve is compiled with
// --fmad=false so a*b+c is never contracted: the float arithmetic then rounds
// exactly as the reference's CPU path does (it is built without FMA contraction;
// its explicit fma in the pair product is kept explicit here too).
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <utility>

namespace kb2::dev {

// A kernel's dynamic shared-memory ceiling is an attribute of the function in
// one device's context, so it is raised once per device this process uses
// (bit d of `done` for device d < 64; higher devices raise it on every call).
inline void raise_shared_limit(const void* kernel, int bytes,
                               std::atomic<unsigned long long>& done) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return;
  const unsigned long long bit = device < 64 ? 1ull << device : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) ==
      cudaSuccess)
    done.fetch_or(bit, std::memory_order_release);
}

// ------------------------------------------------------------------------
// Programmatic dependent launch. The solve is a chain of short dependent
// kernels, each a few microseconds on these sizes, so the gap between one
// kernel's end and the next one's start is a large share of the time. Every
// solve-path kernel is launched with programmatic stream serialization: the
// next kernel may be scheduled while the current one drains, and it waits
// (griddepcontrol.wait, its very first instruction) until the previous grid
// has completed and its memory is visible before touching any memory. So the
// ordering of every read and write is exactly that of ordinary stream order;
// only the launch latency overlaps. After its own wait a kernel lets its
// dependents be scheduled.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// Whether launches carry the attribute (default yes; KUTTA_B200_PDL=0 turns it
// off, for comparisons). Read once per process.
bool pdl_enabled();
// kernel<<<grid, block, smem, s>>>(args...) with the attribute.
template <typename... Params, typename... Args>
inline void pdl(void (*kernel)(Params...), dim3 grid, dim3 block, std::size_t smem,
                cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t config = {};
  config.gridDim = grid;
  config.blockDim = block;
  config.dynamicSmemBytes = smem;
  config.stream = s;
  cudaLaunchAttribute attribute[1];
  attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attribute[0].val.programmaticStreamSerializationAllowed = 1;
  config.attrs = attribute;
  config.numAttrs = pdl_enabled() ? 1 : 0;
  cudaLaunchKernelEx(&config, kernel, std::forward<Args>(args)...);
}

constexpr int kBlock = 256;          // threads per block for row kernels
constexpr int kSms = 148;            // B200 streaming multiprocessors
constexpr int kMaxBlocks = kSms * 8; // grid cap: 8 resident 256-thread blocks per SM
constexpr int kPartials = 2 * kMaxBlocks;

// Grid for a grid-stride row loop: fixed for a given n, so every reduction's
// partition of rows into blocks (and hence its rounding) is deterministic.
inline int grid_for(long long n) {
  long long blocks = (n + kBlock - 1) / kBlock;
  if (blocks < 1) blocks = 1;
  if (blocks > kMaxBlocks) blocks = kMaxBlocks;
  return static_cast<int>(blocks);
}

// ------------------------------------------------------------------------
// Float-pair scalars: the reference's device-scalar wire format (normalised
// (hi, lo) floats, ~48 significant bits), src/kutta/kernels/scalars.kern.h:3-42.
struct Pair {
  float hi, lo;
};
__device__ __forceinline__ Pair kp(float hi, float lo) { return Pair{hi, lo}; }
__device__ __forceinline__ Pair kp_load(const float* p, int offset) {
  return kp(p[offset], p[offset + 1]);
}
__device__ __forceinline__ bool nonfinite(float v) { return v - v != 0.0f; }
__device__ __forceinline__ Pair kp_add(Pair a, Pair b) {
  const float s = a.hi + b.hi;
  if (s - s != 0.0f) return kp(s, 0.0f);
  const float v = s - a.hi;
  float e = (a.hi - (s - v)) + (b.hi - v);
  e = e + a.lo + b.lo;
  const float h = s + e;
  return kp(h, e - (h - s));
}
__device__ __forceinline__ Pair kp_neg(Pair a) { return kp(-a.hi, -a.lo); }
__device__ __forceinline__ Pair kp_mul(Pair a, Pair b) {
  const float h = a.hi * b.hi;
  const float l = fmaf(a.hi, b.hi, -h) + a.hi * b.lo + a.lo * b.hi;
  return kp_add(kp(h, 0.0f), kp(l, 0.0f));
}
__device__ __forceinline__ Pair kp_div(Pair a, Pair b) {
  const float q = a.hi / b.hi;
  const Pair r = kp_add(a, kp_neg(kp_mul(kp(q, 0.0f), b)));
  return kp_add(kp(q, 0.0f), kp((r.hi + r.lo) / b.hi, 0.0f));
}
__device__ __forceinline__ void kp_store(float* out, int offset, Pair p) {
  out[offset] = p.hi;
  out[offset + 1] = p.lo;
}
__device__ __forceinline__ float kp_float(Pair a) { return a.hi + a.lo; }
__device__ __forceinline__ bool kp_positive(Pair a) {
  return a.hi > 0.0f || (a.hi == 0.0f && a.lo > 0.0f);
}
__device__ __forceinline__ bool kp_finite(Pair a) {
  return a.hi - a.hi == 0.0f && a.lo - a.lo == 0.0f;
}
__device__ __forceinline__ bool kp_zero(Pair a) { return a.hi == 0.0f && a.lo == 0.0f; }
__device__ __forceinline__ bool kp_le(Pair a, Pair b) {
  return a.hi < b.hi || (a.hi == b.hi && a.lo <= b.lo);
}
__device__ __forceinline__ bool kp_coefficient(Pair a) {
  const float value = kp_float(a);
  return kp_finite(a) && value - value == 0.0f && (value != 0.0f || kp_zero(a));
}

// Stores an FP64 reduction as a normalised (hi, lo) pair, as the reference's
// reductions do (runtime/cuda/cuda_device.cu:82-110, cpu/cpu_device.cpp:72-89).
__device__ __forceinline__ void store_pair(float* out, int offset, double value) {
  const float hi = static_cast<float>(value);
  out[offset] = hi;
  out[offset + 1] = isfinite(hi) ? static_cast<float>(value - static_cast<double>(hi)) : 0.0f;
}

// ------------------------------------------------------------------------
// Compensated CSR row arithmetic, src/kutta/kernels/linalg.kern.h:5-45.

// Dekker's exact product error with the 4097 split, float only.
__device__ __forceinline__ float product_error(float a, float b, float product) {
  if (fabsf(a) > 1.0e30f || fabsf(b) > 1.0e30f) return 0.0f;
  const float ca = 4097.0f * a;
  const float cb = 4097.0f * b;
  const float ah = ca - (ca - a);
  const float bh = cb - (cb - b);
  const float al = a - ah;
  const float bl = b - bh;
  return ((ah * bh - product) + ah * bl + al * bh) + al * bl;
}

// One term of the Neumaier + Dekker residual sum: sum -= v*x, with both the
// addition error and the product error carried in `error`.
__device__ __forceinline__ void residual_term(float& sum, float& error, float v, float x) {
  const float product = v * x;
  const float term = -product;
  const float next = sum + term;
  error += fabsf(sum) >= fabsf(term) ? (sum - next) + term : (term - next) + sum;
  error -= product_error(v, x, product);
  sum = next;
}

// One term of the Kahan SpMV sum (csr_spmv).
__device__ __forceinline__ void kahan_term(float& sum, float& error, float v, float x) {
  const float term = v * x - error;
  const float next = sum + term;
  error = (next - sum) - term;
  sum = next;
}

// Neumaier sum of one float term (amg_galerkin).
__device__ __forceinline__ void neumaier_term(float& sum, float& error, float term) {
  const float next = sum + term;
  error += fabsf(sum) >= fabsf(term) ? (sum - next) + term : (term - next) + sum;
  sum = next;
}

// Upward-rounded sums, src/kutta/kernels/prelude.h:82-100.
__device__ __forceinline__ float add_up(float a, float b) {
  const float sum = a + b;
  const float part = sum - a;
  const float error = (a - (sum - part)) + (b - part);
  return error > 0.0f ? nextafterf(sum, __int_as_float(0x7f800000)) : sum;
}
struct UpperSum {
  float sum, error;
};
__device__ __forceinline__ UpperSum upper_add(UpperSum a, float b) {
  const float sum = a.sum + b;
  const float part = sum - a.sum;
  const float error = (a.sum - (sum - part)) + (b - part);
  return UpperSum{sum, add_up(a.error, error)};
}
__device__ __forceinline__ float upper_value(UpperSum a) { return add_up(a.sum, a.error); }

// ------------------------------------------------------------------------
// Deterministic FP64 block reduction: warp shuffles in a fixed order, then the
// per-warp values summed in warp order by warp 0.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
  return v;
}
// Returns the block total in thread 0 (other threads: unspecified).
__device__ __forceinline__ double block_sum(double v, double* shared /* >= 32 */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) shared[warp] = v;
  __syncthreads();
  double total = 0;
  if (warp == 0) {
    const int warps = (blockDim.x + 31) >> 5;
    total = lane < warps ? shared[lane] : 0.0;
    total = warp_sum(total);
  }
  __syncthreads();
  return total;
}
__device__ __forceinline__ double nan_max(double a, double b) { return (b > a || isnan(b)) ? b : a; }

// krylov_diagonal's row (src/kutta/kernels/linalg.kern.h:52-70): the inverse
// (L1) diagonal of row i into inverse[i]; returns its invalid flag (0 valid,
// 1 zero diagonal, 2 nonfinite, 3 negative diagonal under L1).
__device__ __forceinline__ float diagonal_row(int i, const int* __restrict__ rows,
                                              const int* __restrict__ diag,
                                              const float* __restrict__ vals,
                                              float* __restrict__ inverse, int use_l1) {
  const float d = vals[diag[i]];
  float off = 0.0f, bad = 0.0f;
  for (int j = rows[i]; j < rows[i + 1]; ++j) {
    const float v = vals[j];
    if (v - v != 0.0f) bad = 1.0f;
    if (j != diag[i]) off += fabsf(v);
  }
  const float inv = d != 0.0f ? 1.0f / d : 0.0f;
  const float l1 = fmaxf(fabsf(d), 0.5f * (fabsf(d) + off));
  inverse[i] = use_l1 != 0 ? (l1 != 0.0f ? 1.0f / l1 : 0.0f) : inv;
  return (bad != 0.0f || inv - inv != 0.0f || l1 - l1 != 0.0f)
             ? 2.0f
             : (use_l1 != 0 && d < 0.0f ? 3.0f : (d == 0.0f ? 1.0f : 0.0f));
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = nan_max(v, __shfl_down_sync(0xffffffffu, v, d));
  return v;
}
__device__ __forceinline__ double block_max(double v, double* shared) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_max(v);
  if (lane == 0) shared[warp] = v;
  __syncthreads();
  double total = 0;
  if (warp == 0) {
    const int warps = (blockDim.x + 31) >> 5;
    total = lane < warps ? shared[lane] : 0.0;
    total = warp_max(total);
  }
  __syncthreads();
  return total;
}

// Grid-wide reduction state: per-block partials and a ticket counter. The last
// block to finish (ticket == gridDim.x - 1) sums the partials in block order and
// resets the ticket, so the result is independent of scheduling.
struct Reducer {
  double* partials;   // kPartials doubles
  unsigned* ticket;   // one counter, zero between launches
};

// Publishes this block's partial(s); returns true in every thread of the last block.
__device__ __forceinline__ bool publish(const Reducer& red, double a, double b, bool dual) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    red.partials[blockIdx.x] = a;
    if (dual) red.partials[kMaxBlocks + blockIdx.x] = b;
    __threadfence();
    const unsigned t = atomicAdd(red.ticket, 1u);
    last = t == gridDim.x - 1;
  }
  __syncthreads();
  return last;
}
// In the last block: the fixed-order total of the partials (thread 0 gets it).
__device__ __forceinline__ double gather(const Reducer& red, int which, double* shared) {
  double v = 0;
  const volatile double* p = red.partials + which * kMaxBlocks;
  for (int k = threadIdx.x; k < static_cast<int>(gridDim.x); k += blockDim.x) v += p[k];
  return block_sum(v, shared);
}
__device__ __forceinline__ double gather_max(const Reducer& red, double* shared) {
  double v = 0;
  const volatile double* p = red.partials;
  for (int k = threadIdx.x; k < static_cast<int>(gridDim.x); k += blockDim.x) v = nan_max(v, p[k]);
  return block_max(v, shared);
}

}  // namespace kb2::dev
