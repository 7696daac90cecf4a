// Mixed-precision kernels (no reference counterpart): BF16 coarse operators,
// the dense FP64 coarsest-level inverse, and the FP64 refinement residual.
// Compiled with ordinary FMA contraction: these results are judged by the
// FP64 true residual, not by bitwise agreement with the reference.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "kernels.hpp"

namespace kb2 {
namespace {
using namespace dev;

#define ROWS(i, n) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

inline int rows_grid(int n) {
  if (n >= (1 << 21)) return grid_for(n);
  return n > 0 ? (n + kBlock - 1) / kBlock : 1;
}

__device__ __forceinline__ float bf(unsigned short v) {
  return __bfloat162float(__ushort_as_bfloat16(v));
}

// Row scale = max |a_ij| (FP32); stored value = bf16(a_ij / scale).
__global__ void k_bf16_pack(int n, const int* __restrict__ rows, const float* __restrict__ vals,
                            unsigned short* __restrict__ v16, float* __restrict__ scale) {
  ROWS(i, n) {
    float m = 0.0f;
    for (int j = rows[i]; j < rows[i + 1]; ++j) m = fmaxf(m, fabsf(vals[j]));
    const float s = m > 0.0f ? m : 1.0f;
    scale[i] = s;
    const float inv = 1.0f / s;
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      v16[j] = __bfloat16_as_ushort(__float2bfloat16_rn(vals[j] * inv));
  }
}

__device__ __forceinline__ float bf16_row(int i, const int* __restrict__ rows,
                                          const int* __restrict__ cols,
                                          const unsigned short* __restrict__ v16,
                                          const float* __restrict__ x) {
  float acc = 0.0f;
  const int end = rows[i + 1];
  for (int j = rows[i]; j < end; ++j) acc = fmaf(bf(v16[j]), x[cols[j]], acc);
  return acc;
}

// Damped L1-Jacobi sweep with the BF16 operator (FP32 accumulation).
template <bool kZero>
__global__ void k_bf16_smooth(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                              const unsigned short* __restrict__ v16,
                              const float* __restrict__ scale, const float* __restrict__ x,
                              const float* __restrict__ b, const float* __restrict__ inv,
                              float* __restrict__ next, const int* __restrict__ status) {
  if (status[0] != 0) return;
  ROWS(i, n) {
    if (kZero) {
      next[i] = (2.0f / 3.0f) * inv[i] * b[i];
    } else {
      const float r = b[i] - scale[i] * bf16_row(i, rows, cols, v16, x);
      next[i] = x[i] + (2.0f / 3.0f) * inv[i] * r;
    }
  }
}

__global__ void k_bf16_residual(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                                const unsigned short* __restrict__ v16,
                                const float* __restrict__ scale, const float* __restrict__ x,
                                const float* __restrict__ b, float* __restrict__ r,
                                const int* __restrict__ status) {
  if (status[0] != 0) return;
  ROWS(i, n) r[i] = b[i] - scale[i] * bf16_row(i, rows, cols, v16, x);
}

// Dense FP64 Cholesky of the coarsest operator and its explicit inverse, in one
// block (n <= 1024). L is n x n row-major scratch and W the n x n inverse, both
// in global memory (the level is small, so both stay in cache). *error is
// written at the end: 1 if a pivot was not positive (the operator is not SPD;
// such a pivot is replaced by 1 so the kernel ends), else 0.
__global__ void __launch_bounds__(1024)
    k_dense_inverse(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                    const float* __restrict__ vals, double* __restrict__ L,
                    double* __restrict__ W, double* error) {
  const int t = threadIdx.x, T = blockDim.x;
  __shared__ int failed;
  if (t == 0) failed = 0;
  for (int k = t; k < n * n; k += T) L[k] = 0.0;
  __syncthreads();
  for (int i = t; i < n; i += T)
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      if (cols[j] <= i) L[static_cast<std::size_t>(i) * n + cols[j]] = vals[j];
  __syncthreads();
  __shared__ double pivot;
  for (int k = 0; k < n; ++k) {
    if (t == 0) {
      double d = L[static_cast<std::size_t>(k) * n + k];
      if (!(d > 0.0)) {
        failed = 1;
        d = 1.0;
      }
      pivot = sqrt(d);
      L[static_cast<std::size_t>(k) * n + k] = pivot;
    }
    __syncthreads();
    for (int i = k + 1 + t; i < n; i += T) L[static_cast<std::size_t>(i) * n + k] /= pivot;
    __syncthreads();
    for (int i = k + 1 + t; i < n; i += T) {
      const double lik = L[static_cast<std::size_t>(i) * n + k];
      double* row = L + static_cast<std::size_t>(i) * n;
      for (int j = k + 1; j <= i; ++j) row[j] -= lik * L[static_cast<std::size_t>(j) * n + k];
    }
    __syncthreads();
  }
  // Column j of the inverse: L y = e_j, then L^T z = y (thread per column).
  for (int j = t; j < n; j += T) {
    for (int i = 0; i < n; ++i) {
      double s = i == j ? 1.0 : 0.0;
      if (i > j)
        for (int k = j; k < i; ++k) s -= L[static_cast<std::size_t>(i) * n + k] * W[static_cast<std::size_t>(k) * n + j];
      W[static_cast<std::size_t>(i) * n + j] = i < j ? 0.0 : s / L[static_cast<std::size_t>(i) * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = W[static_cast<std::size_t>(i) * n + j];
      for (int k = i + 1; k < n; ++k) s -= L[static_cast<std::size_t>(k) * n + i] * W[static_cast<std::size_t>(k) * n + j];
      W[static_cast<std::size_t>(i) * n + j] = s / L[static_cast<std::size_t>(i) * n + i];
    }
  }
  if (t == 0) *error = failed ? 1.0 : 0.0;
}

// x = A^-1 b with the dense FP64 inverse: one warp per row, FP64 accumulation.
__global__ void k_dense_solve(int n, const double* __restrict__ W, const float* __restrict__ b,
                              float* __restrict__ x, const int* __restrict__ status) {
  if (status[0] != 0) return;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = warp; i < n; i += warps) {
    double acc = 0.0;
    const double* row = W + static_cast<std::size_t>(i) * n;
    for (int k = lane; k < n; k += 32) acc += row[k] * static_cast<double>(b[k]);
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if (lane == 0) x[i] = static_cast<float>(acc);
  }
}

// FP64 refinement residual: r = b - A x in FP64 (x FP64, A and b FP32), written
// rounded to FP32 for the inner solve, with ||r||^2 reduced in FP64 into out[slot].
__global__ void k_residual64(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                             const float* __restrict__ vals, const double* __restrict__ x,
                             const float* __restrict__ b, float* __restrict__ rf,
                             DeviceReducer red, double* out, int slot) {
  double acc = 0.0;
  ROWS(i, n) {
    double s = static_cast<double>(b[i]);
    const int end = rows[i + 1];
    for (int j = rows[i]; j < end; ++j) s -= static_cast<double>(vals[j]) * x[cols[j]];
    rf[i] = static_cast<float>(s);
    acc += s * s;
  }
  __shared__ double shared[32];
  acc = block_sum(acc, shared);
  const Reducer r{red.partials, red.ticket};
  if (!publish(r, acc, 0, false)) return;
  const double total = gather(r, 0, shared);
  if (threadIdx.x == 0) {
    out[slot] = total;
    *r.ticket = 0;
  }
}

__global__ void k_update64(int n, double* __restrict__ x, const float* __restrict__ e) {
  ROWS(i, n) x[i] += static_cast<double>(e[i]);
}

}  // namespace

namespace launch {

void bf16_pack(int n, const int* rows, const float* vals, unsigned short* v16, float* scale,
               cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_bf16_pack<<<rows_grid(n), kBlock, 0, s>>>(n, rows, vals, v16, scale);
}
void bf16_smooth(int n, const int* rows, const int* cols, const unsigned short* v16,
                 const float* scale, const float* x, const float* b, const float* inv, float* next,
                 const int* status, bool zero_start, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  if (zero_start)
    k_bf16_smooth<true><<<rows_grid(n), kBlock, 0, s>>>(n, rows, cols, v16, scale, x, b, inv, next, status);
  else
    k_bf16_smooth<false><<<rows_grid(n), kBlock, 0, s>>>(n, rows, cols, v16, scale, x, b, inv, next, status);
}
void bf16_residual(int n, const int* rows, const int* cols, const unsigned short* v16,
                   const float* scale, const float* x, const float* b, float* r, const int* status,
                   cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_bf16_residual<<<rows_grid(n), kBlock, 0, s>>>(n, rows, cols, v16, scale, x, b, r, status);
}
void dense_inverse(int n, const int* rows, const int* cols, const float* vals, double* lower,
                   double* inverse, double* error, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  const int threads = std::min(1024, ((n + 31) / 32) * 32);
  k_dense_inverse<<<1, threads, 0, s>>>(n, rows, cols, vals, lower, inverse, error);
}
void dense_solve(int n, const double* inverse, const float* b, float* x, const int* status,
                 cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  const int blocks = std::min(1184, (n * 32 + kBlock - 1) / kBlock);
  k_dense_solve<<<blocks, kBlock, 0, s>>>(n, inverse, b, x, status);
}
void residual64(int n, const int* rows, const int* cols, const float* vals, const double* x,
                const float* b, float* rf, DeviceReducer red, double* out, int slot,
                cudaStream_t s) {
  ++counter;
  k_residual64<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, vals, x, b, rf, red, out, slot);
}
void update64(int n, double* x, const float* e, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_update64<<<rows_grid(n), kBlock, 0, s>>>(n, x, e);
}

}  // namespace launch
}  // namespace kb2
