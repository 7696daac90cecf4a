// Mixed-precision kernels (no reference counterpart): BF16 coarse operators,
// the dense FP64 coarsest-level inverse, and the FP64 refinement residual.
// Compiled with ordinary FMA contraction: these results are checked against the
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
  pdl_entry();
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

// Coarse rows hold about a dozen entries: four lanes share a row, each taking
// every fourth entry, so a warp reads eight rows' contiguous segments instead
// of 32 strided ones, and a row's dependent gathers are a quarter as long.
constexpr int kLanes = 4;
constexpr int kRowsPerWarp = 32 / kLanes;

// This lane's share of sum_j a_ij x_j (BF16 values, FP32 accumulation). The
// row is taken in chunks of kLanes * kPerLane entries; a lane issues all its
// column and value loads of a chunk before any gather, so each warp keeps
// several independent loads in flight (these levels are latency-bound).
constexpr int kPerLane = 3;
__device__ __forceinline__ float bf16_row_part(int i, int lane, const int* __restrict__ rows,
                                               const int* __restrict__ cols,
                                               const unsigned short* __restrict__ v16,
                                               const float* __restrict__ x) {
  float acc = 0.0f;
  const int end = rows[i + 1];
  for (int j0 = rows[i] + lane; j0 < end; j0 += kLanes * kPerLane) {
    int c[kPerLane];
    float a[kPerLane];
#pragma unroll
    for (int u = 0; u < kPerLane; ++u) {
      const int j = j0 + u * kLanes;
      c[u] = j < end ? cols[j] : -1;
      a[u] = j < end ? bf(v16[j]) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < kPerLane; ++u)
      if (c[u] >= 0) acc = fmaf(a[u], x[c[u]], acc);
  }
  return acc;
}
// Sum over the row's four lanes, in lane 0 (every lane of the warp calls it).
__device__ __forceinline__ float row_total(float v) {
  v += __shfl_down_sync(0xffffffffu, v, 2, kLanes);
  v += __shfl_down_sync(0xffffffffu, v, 1, kLanes);
  return v;
}

// Visits rows kLanes lanes at a time; the loop bound is uniform across a warp,
// so every lane reaches the shuffles. body(i, lane, valid).
template <class Body>
__device__ __forceinline__ void for_rows(int n, Body body) {
  const int lane = threadIdx.x & (kLanes - 1);
  const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
  for (int row0 = warp * kRowsPerWarp; row0 < n; row0 += warps * kRowsPerWarp) {
    const int i = row0 + static_cast<int>((threadIdx.x & 31) / kLanes);
    body(i, lane, i < n);
  }
}

// A reduction's grid stays within the partials buffer (kMaxBlocks blocks).
inline int lanes_grid(int n, bool reduction) {
  const long long blocks = (static_cast<long long>(n) * kLanes + kBlock - 1) / kBlock;
  const long long cap = reduction ? static_cast<long long>(kMaxBlocks) : (1LL << 30);
  return static_cast<int>(std::max(1LL, std::min(blocks, cap)));
}

// Damped L1-Jacobi sweep with the BF16 operator (FP32 accumulation).
template <bool kZero>
__global__ void k_bf16_smooth(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                              const unsigned short* __restrict__ v16,
                              const float* __restrict__ scale, const float* __restrict__ x,
                              const float* __restrict__ b, const float* __restrict__ inv,
                              float* __restrict__ next, const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  if (kZero) {
    ROWS(i, n) next[i] = (2.0f / 3.0f) * inv[i] * b[i];
    return;
  }
  for_rows(n, [&](int i, int lane, bool valid) {
    const float acc = row_total(valid ? bf16_row_part(i, lane, rows, cols, v16, x) : 0.0f);
    if (valid && lane == 0) next[i] = x[i] + (2.0f / 3.0f) * inv[i] * (b[i] - scale[i] * acc);
  });
}

__global__ void k_bf16_residual(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                                const unsigned short* __restrict__ v16,
                                const float* __restrict__ scale, const float* __restrict__ x,
                                const float* __restrict__ b, float* __restrict__ r,
                                const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  for_rows(n, [&](int i, int lane, bool valid) {
    const float acc = row_total(valid ? bf16_row_part(i, lane, rows, cols, v16, x) : 0.0f);
    if (valid && lane == 0) r[i] = b[i] - scale[i] * acc;
  });
}

// Coarse b = sum of the fine residual over each aggregate's members, four
// lanes per aggregate with their member loads batched like the row kernels.
__global__ void k_restrict_lanes(int nc, const int* __restrict__ offsets,
                                 const int* __restrict__ members, const float* __restrict__ fine,
                                 float* __restrict__ coarse, const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  for_rows(nc, [&](int g, int lane, bool valid) {
    float acc = 0.0f;
    if (valid) {
      const int end = offsets[g + 1];
      for (int j0 = offsets[g] + lane; j0 < end; j0 += kLanes * kPerLane) {
        int m[kPerLane];
#pragma unroll
        for (int u = 0; u < kPerLane; ++u) {
          const int j = j0 + u * kLanes;
          m[u] = j < end ? members[j] : -1;
        }
#pragma unroll
        for (int u = 0; u < kPerLane; ++u)
          if (m[u] >= 0) acc += fine[m[u]];
      }
    }
    acc = row_total(acc);
    if (valid && lane == 0) coarse[g] = acc;
  });
}

// The last block stores the two FP64 totals as (hi, lo) pairs at
// scalars[offset] and scalars[offset + 2].
__device__ __forceinline__ void finish_dot2(DeviceReducer red, double a, double b,
                                            float* scalars, int offset) {
  __shared__ double shared[32];
  a = block_sum(a, shared);
  b = block_sum(b, shared);
  const Reducer r{red.partials, red.ticket};
  if (!publish(r, a, b, true)) return;
  const double total_a = gather(r, 0, shared);
  const double total_b = gather(r, 1, shared);
  if (threadIdx.x == 0) {
    store_pair(scalars, offset, total_a);
    store_pair(scalars, offset + 2, total_b);
    *r.ticket = 0;
  }
}

// K-cycle inner step on a BF16 level: q = A p and, in the same pass, the two
// products its step length needs -> scalars[0..3]: p.q and w.p (A-conjugate,
// SPD) or q.q and w.q (GCR). Skipped while status[0] != 0.
__global__ void k_bf16_spmv_dot2(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                                 const unsigned short* __restrict__ v16,
                                 const float* __restrict__ scale, const float* __restrict__ p,
                                 const float* __restrict__ w, float* __restrict__ q, bool gcr,
                                 DeviceReducer red, float* scalars,
                                 const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  double a = 0.0, b = 0.0;
  for_rows(n, [&](int i, int lane, bool valid) {
    const float acc = row_total(valid ? bf16_row_part(i, lane, rows, cols, v16, p) : 0.0f);
    if (valid && lane == 0) {
      const float qi = scale[i] * acc;
      q[i] = qi;
      const double d = gcr ? static_cast<double>(qi) : static_cast<double>(p[i]);
      a += d * static_cast<double>(qi);
      b += static_cast<double>(w[i]) * d;
    }
  });
  finish_dot2(red, a, b, scalars, 0);
}

// amg_inner_first with the next reduction fused: x = alpha p, t = b - alpha q
// (or x = p, t = 0 when the level's status is not running), then t.t and b.b
// -> scalars[4..7]. Skipped (reduction included) while status[0] != 0, as
// every reader of those slots is.
__global__ void k_inner_first_dot(int n, const float* __restrict__ b, const float* __restrict__ p,
                                  const float* __restrict__ q, float* __restrict__ x,
                                  float* __restrict__ t, float* scalars,
                                  const int* __restrict__ status, DeviceReducer red) {
  pdl_entry();
  const bool running = status[0] == 0;
  const float alpha = kp_float(kp_load(scalars, 8));
  double tt = 0.0, bb = 0.0;
  ROWS(i, n) {
    const float ti = running ? b[i] - alpha * q[i] : 0.0f;
    x[i] = running ? alpha * p[i] : p[i];
    t[i] = ti;
    tt += static_cast<double>(ti) * static_cast<double>(ti);
    bb += static_cast<double>(b[i]) * static_cast<double>(b[i]);
  }
  if (!running) return;
  finish_dot2(red, tt, bb, scalars, 4);
}

// Dense FP64 Cholesky of the coarsest operator and its explicit inverse, in one
// block (n <= 1024). L is n x n row-major scratch and W the n x n inverse, both
// in global memory (the level is small, so both stay in cache). *error is
// written at the end: 1 if a pivot was not positive (the operator is not SPD;
// such a pivot is replaced by 1 so the kernel ends), else 0. If `ratio` is not
// null, *ratio is the smallest pivot relative to its row's diagonal (0 if one
// failed): close to 0 when the operator is nearly singular.
__global__ void __launch_bounds__(1024)
    k_dense_inverse(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                    const float* __restrict__ vals, double* __restrict__ L,
                    double* __restrict__ W, double* error, double* ratio) {
  pdl_entry();
  const int t = threadIdx.x, T = blockDim.x;
  __shared__ int failed;
  __shared__ double smallest;
  __shared__ double diag0[1024];
  if (t == 0) {
    failed = 0;
    smallest = 1.0;
  }
  for (int k = t; k < n * n; k += T) L[k] = 0.0;
  __syncthreads();
  for (int i = t; i < n; i += T)
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      if (cols[j] <= i) L[static_cast<std::size_t>(i) * n + cols[j]] = vals[j];
      if (cols[j] == i) diag0[i] = vals[j];
    }
  __syncthreads();
  __shared__ double pivot;
  for (int k = 0; k < n; ++k) {
    if (t == 0) {
      double d = L[static_cast<std::size_t>(k) * n + k];
      if (!(d > 0.0)) {
        failed = 1;
        d = 1.0;
      } else {
        smallest = fmin(smallest, d / diag0[k]);
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
  if (t == 0) {
    *error = failed ? 1.0 : 0.0;
    if (ratio) *ratio = failed ? 0.0 : smallest;
  }
}

// The same Cholesky factor and inverse for n <= kSharedDense, on chip and
// with short dependent chains: L and X = L^-1 live in shared memory; each
// elimination step updates the trailing lower triangle in parallel over its
// (i, j) pairs (each element sees the same updates in the same k order as a
// row-by-row update); X is built one elimination step at a time over all
// right-hand sides of the identity at once; W = X^T X (symmetric) is written
// to global memory. `L` (global) is not used.
constexpr int kSharedDense = 112;  // 2 n^2 doubles <= 200 KB
constexpr int kDenseThreads = 256;

// Lower-triangle pair number p -> (i, j), j <= i, rows counted from 0.
__device__ __forceinline__ void triangle_pair(int p, int& i, int& j) {
  i = static_cast<int>((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= p) ++i;
  while (i * (i + 1) / 2 > p) --i;
  j = p - i * (i + 1) / 2;
}

__global__ void __launch_bounds__(kDenseThreads)
    k_dense_inverse_shared(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                           const float* __restrict__ vals, double* __restrict__ W, double* error,
                           double* ratio) {
  pdl_entry();
  extern __shared__ double dense[];
  double* Ls = dense;          // n x n, lower triangle
  double* Xs = dense + n * n;  // n x n, X = L^-1 (lower triangle)
  const int t = threadIdx.x, T = blockDim.x;
  __shared__ int failed;
  __shared__ double smallest, pivot;
  __shared__ double diag0[kSharedDense];
  if (t == 0) {
    failed = 0;
    smallest = 1.0;
  }
  for (int k = t; k < n * n; k += T) {
    Ls[k] = 0.0;
    Xs[k] = (k / n == k % n) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int i = t; i < n; i += T)
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      if (cols[j] <= i) Ls[i * n + cols[j]] = vals[j];
      if (cols[j] == i) diag0[i] = vals[j];
    }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (t == 0) {
      double d = Ls[k * n + k];
      if (!(d > 0.0)) {
        failed = 1;
        d = 1.0;
      } else {
        smallest = fmin(smallest, d / diag0[k]);
      }
      pivot = sqrt(d);
      Ls[k * n + k] = pivot;
    }
    __syncthreads();
    for (int i = k + 1 + t; i < n; i += T) Ls[i * n + k] /= pivot;
    __syncthreads();
    const int m = n - k - 1;  // trailing rows k+1 .. n-1
    for (int p = t; p < m * (m + 1) / 2; p += T) {
      int a, b;
      triangle_pair(p, a, b);
      const int i = k + 1 + a, j = k + 1 + b;
      Ls[i * n + j] -= Ls[i * n + k] * Ls[j * n + k];
    }
    __syncthreads();
  }
  // X = L^-1: step k scales row k of X by 1 / L_kk, then removes L_ik X_k from
  // the rows below (only columns j <= k of X are nonzero at that point).
  for (int k = 0; k < n; ++k) {
    const double inv = 1.0 / Ls[k * n + k];
    for (int j = t; j <= k; j += T) Xs[k * n + j] *= inv;
    __syncthreads();
    const int below = n - k - 1;
    for (int p = t; p < below * (k + 1); p += T) {
      const int i = k + 1 + p / (k + 1), j = p % (k + 1);
      Xs[i * n + j] -= Ls[i * n + k] * Xs[k * n + j];
    }
    __syncthreads();
  }
  // W = X^T X: W_ij = sum_{k >= max(i, j)} X_ki X_kj.
  for (int p = t; p < n * (n + 1) / 2; p += T) {
    int i, j;
    triangle_pair(p, i, j);
    double acc = 0.0;
    for (int k = i; k < n; ++k) acc += Xs[k * n + i] * Xs[k * n + j];
    W[static_cast<std::size_t>(i) * n + j] = acc;
    W[static_cast<std::size_t>(j) * n + i] = acc;
  }
  if (t == 0) {
    *error = failed ? 1.0 : 0.0;
    if (ratio) *ratio = failed ? 0.0 : smallest;
  }
}

// The same for kSharedDense < n <= kPackedDense: only the lower triangle, packed
// (row i at i (i + 1) / 2), fits in shared memory, so L is inverted in place.
// Column j of X = L^-1 (j from the right) needs the already inverted columns
// k > j and column j of L: X_ij = -(sum_{k=j+1..i} X_ik L_kj) / L_jj, one warp
// per row i with the sum split over the lanes; then W = X^T X.
constexpr int kPackedDense = 236;  // (n (n + 1) / 2 + 2 n) doubles <= 227 KB
constexpr int kPackedThreads = 1024;

__device__ __forceinline__ int packed(int i, int j) { return i * (i + 1) / 2 + j; }

__global__ void __launch_bounds__(kPackedThreads)
    k_dense_inverse_packed(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                           const float* __restrict__ vals, double* __restrict__ W, double* error,
                           double* ratio) {
  pdl_entry();
  extern __shared__ double dense[];
  const int total = n * (n + 1) / 2;
  double* P = dense;           // packed lower triangle: L, then X = L^-1
  double* temp = P + total;    // one column's new entries
  double* diag0 = temp + n;    // the input diagonal
  const int t = threadIdx.x, T = blockDim.x, lane = t & 31, warp = t >> 5, warps = T >> 5;
  __shared__ int failed;
  __shared__ double smallest, pivot;
  if (t == 0) {
    failed = 0;
    smallest = 1.0;
  }
  for (int k = t; k < total; k += T) P[k] = 0.0;
  __syncthreads();
  for (int i = t; i < n; i += T)
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      if (cols[j] <= i) P[packed(i, cols[j])] = vals[j];
      if (cols[j] == i) diag0[i] = vals[j];
    }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (t == 0) {
      double d = P[packed(k, k)];
      if (!(d > 0.0)) {
        failed = 1;
        d = 1.0;
      } else {
        smallest = fmin(smallest, d / diag0[k]);
      }
      pivot = sqrt(d);
      P[packed(k, k)] = pivot;
    }
    __syncthreads();
    for (int i = k + 1 + t; i < n; i += T) P[packed(i, k)] /= pivot;
    __syncthreads();
    const int m = n - k - 1;
    for (int p = t; p < m * (m + 1) / 2; p += T) {
      int a, b;
      triangle_pair(p, a, b);
      const int i = k + 1 + a, j = k + 1 + b;
      P[packed(i, j)] -= P[packed(i, k)] * P[packed(j, k)];
    }
    __syncthreads();
  }
  for (int j = n - 1; j >= 0; --j) {
    const double ljj = P[packed(j, j)];  // read before this step's writes
    for (int i = j + 1 + warp; i < n; i += warps) {
      double acc = 0.0;
      for (int k = j + 1 + lane; k <= i; k += 32) acc += P[packed(i, k)] * P[packed(k, j)];
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
      if (lane == 0) temp[i] = acc;
    }
    __syncthreads();
    for (int i = j + 1 + t; i < n; i += T) P[packed(i, j)] = -temp[i] / ljj;
    if (t == 0) P[packed(j, j)] = 1.0 / ljj;
    __syncthreads();
  }
  for (int p = t; p < total; p += T) {
    int i, j;
    triangle_pair(p, i, j);
    double acc = 0.0;
    for (int k = i; k < n; ++k) acc += P[packed(k, i)] * P[packed(k, j)];
    W[static_cast<std::size_t>(i) * n + j] = acc;
    W[static_cast<std::size_t>(j) * n + i] = acc;
  }
  if (t == 0) {
    *error = failed ? 1.0 : 0.0;
    if (ratio) *ratio = failed ? 0.0 : smallest;
  }
}

// x = A^-1 b with the dense FP64 inverse: one warp per row, FP64 accumulation.
__global__ void k_dense_solve(int n, const double* __restrict__ W, const float* __restrict__ b,
                              float* __restrict__ x, const int* __restrict__ status) {
  pdl_entry();
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
  pdl_entry();
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
  pdl_entry();
  ROWS(i, n) x[i] += static_cast<double>(e[i]);
}

__global__ void k_widen(int n, const float* __restrict__ x, double* __restrict__ y) {
  pdl_entry();
  ROWS(i, n) y[i] = static_cast<double>(x[i]);
}

__global__ void k_narrow(int n, const double* __restrict__ y, float* __restrict__ x) {
  pdl_entry();
  ROWS(i, n) x[i] = static_cast<float>(y[i]);
}

}  // namespace

namespace launch {

void bf16_pack(int n, const int* rows, const float* vals, unsigned short* v16, float* scale,
               cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_bf16_pack, rows_grid(n), kBlock, 0, s, n, rows, vals, v16, scale);
}
void bf16_smooth(int n, const int* rows, const int* cols, const unsigned short* v16,
                 const float* scale, const float* x, const float* b, const float* inv, float* next,
                 const int* status, bool zero_start, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  if (zero_start)
    pdl(k_bf16_smooth<true>, rows_grid(n), kBlock, 0, s, n, rows, cols, v16, scale, x, b, inv, next, status);
  else
    pdl(k_bf16_smooth<false>, lanes_grid(n, false), kBlock, 0, s, n, rows, cols, v16, scale, x, b, inv, next, status);
}
void restrict_lanes(int nc, const int* offsets, const int* members, const float* fine,
                    float* coarse, const int* status, cudaStream_t s) {
  if (nc <= 0) return;
  ++counter;
  pdl(k_restrict_lanes, lanes_grid(nc, false), kBlock, 0, s, nc, offsets, members, fine, coarse,
                                                            status);
}
void bf16_spmv_dot2(int n, const int* rows, const int* cols, const unsigned short* v16,
                    const float* scale, const float* p, const float* w, float* q, bool gcr,
                    DeviceReducer red, float* scalars, const int* status, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_bf16_spmv_dot2, lanes_grid(n, true), kBlock, 0, s, n, rows, cols, v16, scale, p, w, q,
                                                          gcr, red, scalars, status);
}
void inner_first_dot(int n, const float* b, const float* p, const float* q, float* x, float* t,
                     float* scalars, const int* status, DeviceReducer red, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_inner_first_dot, grid_for(n), kBlock, 0, s, n, b, p, q, x, t, scalars, status, red);
}
void bf16_residual(int n, const int* rows, const int* cols, const unsigned short* v16,
                   const float* scale, const float* x, const float* b, float* r, const int* status,
                   cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_bf16_residual, lanes_grid(n, false), kBlock, 0, s, n, rows, cols, v16, scale, x, b, r,
                                                          status);
}
void dense_inverse(int n, const int* rows, const int* cols, const float* vals, double* lower,
                   double* inverse, double* error, cudaStream_t s, double* ratio) {
  if (n <= 0) return;
  ++counter;
  if (n <= kSharedDense) {
    const int bytes = 2 * n * n * static_cast<int>(sizeof(double));
    static std::atomic<unsigned long long> raised{0};
    raise_shared_limit(reinterpret_cast<const void*>(k_dense_inverse_shared),
                       2 * kSharedDense * kSharedDense * static_cast<int>(sizeof(double)), raised);
    pdl(k_dense_inverse_shared, 1, kDenseThreads, bytes, s, n, rows, cols, vals, inverse, error,
                                                            ratio);
    return;
  }
  if (n <= kPackedDense) {
    const int bytes = (n * (n + 1) / 2 + 2 * n) * static_cast<int>(sizeof(double));
    static std::atomic<unsigned long long> raised_packed{0};
    raise_shared_limit(
        reinterpret_cast<const void*>(k_dense_inverse_packed),
        (kPackedDense * (kPackedDense + 1) / 2 + 2 * kPackedDense) * static_cast<int>(sizeof(double)),
        raised_packed);
    pdl(k_dense_inverse_packed, 1, kPackedThreads, bytes, s, n, rows, cols, vals, inverse, error,
                                                            ratio);
    return;
  }
  const int threads = std::min(1024, ((n + 31) / 32) * 32);
  pdl(k_dense_inverse, 1, threads, 0, s, n, rows, cols, vals, lower, inverse, error, ratio);
}
void dense_solve(int n, const double* inverse, const float* b, float* x, const int* status,
                 cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  const int blocks = std::min(1184, (n * 32 + kBlock - 1) / kBlock);
  pdl(k_dense_solve, blocks, kBlock, 0, s, n, inverse, b, x, status);
}
void residual64(int n, const int* rows, const int* cols, const float* vals, const double* x,
                const float* b, float* rf, DeviceReducer red, double* out, int slot,
                cudaStream_t s) {
  ++counter;
  pdl(k_residual64, grid_for(n), kBlock, 0, s, n, rows, cols, vals, x, b, rf, red, out, slot);
}
void update64(int n, double* x, const float* e, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_update64, rows_grid(n), kBlock, 0, s, n, x, e);
}
void widen(int n, const float* x, double* y, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_widen, rows_grid(n), kBlock, 0, s, n, x, y);
}
void narrow(int n, const double* y, float* x, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_narrow, rows_grid(n), kBlock, 0, s, n, y, x);
}

}  // namespace launch
}  // namespace kb2
