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

// Dense FP64 Cholesky of the coarsest operator and its explicit inverse for
// kPackedDense < n <= 1024, blocked in 32 x 32 blocks and spread over many
// CTAs (a sequence of launches at refresh time). L is n x n row-major scratch
// in global memory (2 MB at n = 512, L2-resident) and W the n x n inverse.
//   1. L = the lower triangle of A (the strict upper triangle is free; the
//      original diagonal is kept there for the pivot ratio: a_kk at L[k][n-1],
//      a_{n-1,n-1} at L[0][n-2]);
//   2. per 32-column panel: the diagonal block factored in one CTA (shared
//      memory), the rows below solved against it (a thread per row), the
//      trailing lower triangle updated tile by tile (a CTA per 32 x 32 tile);
//   3. X = L^-1 into W's lower triangle: the diagonal blocks inverted in
//      parallel, then block diagonal d = 1, 2, ...: X_ij = -X_ii sum_{k=j}^{i-1}
//      L_ik X_kj for i - j = d, a CTA per block;
//   4. W = X^T X tile by tile into L's buffer, then copied to W.
// Every element is summed in a fixed order, so the result is deterministic.
// *error = 1 if a pivot was not positive (it is replaced by 1 so the kernels
// finish), else 0; with `ratio`, *ratio is the smallest pivot relative to its
// row's original diagonal (0 if one failed).
constexpr int kNb = 32;                         // block size
constexpr int kNbThreads = kNb * kNb;           // one thread per block element

__device__ __forceinline__ std::size_t at(int n, int i, int j) {
  return static_cast<std::size_t>(i) * n + j;
}
// Where row k's original diagonal is kept (strict upper triangle of L).
__device__ __forceinline__ std::size_t diag_slot(int n, int k) {
  return k < n - 1 ? at(n, k, n - 1) : at(n, 0, n - 2);
}

__global__ void k_dense_zero(std::size_t count, double* __restrict__ L) {
  pdl_entry();
  for (std::size_t k = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; k < count;
       k += static_cast<std::size_t>(gridDim.x) * blockDim.x)
    L[k] = 0.0;
}

__global__ void k_dense_scatter(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                                const float* __restrict__ vals, double* __restrict__ L,
                                double* error, double* ratio) {
  pdl_entry();
  ROWS(i, n) {
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      const int c = cols[j];
      if (c <= i) L[at(n, i, c)] = vals[j];
      if (c == i) L[diag_slot(n, i)] = vals[j];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *error = 0.0;
    if (ratio) *ratio = 1.0;
  }
}

// Factor the diagonal block of panel k0 (b = min(32, n - k0) columns) in place.
__global__ void __launch_bounds__(kNbThreads)
    k_dense_panel_factor(int n, int k0, double* __restrict__ L, double* error, double* ratio) {
  pdl_entry();
  __shared__ double D[kNb][kNb + 1];
  const int b = min(kNb, n - k0);
  const int r = threadIdx.x / kNb, c = threadIdx.x % kNb;
  if (r < b && c <= r) D[r][c] = L[at(n, k0 + r, k0 + c)];
  __syncthreads();
  for (int k = 0; k < b; ++k) {
    if (threadIdx.x == 0) {
      double d = D[k][k];
      if (!(d > 0.0)) {
        *error = 1.0;
        if (ratio) *ratio = 0.0;
        d = 1.0;
      } else if (ratio && *error == 0.0) {
        *ratio = fmin(*ratio, d / L[diag_slot(n, k0 + k)]);
      }
      D[k][k] = sqrt(d);
    }
    __syncthreads();
    if (c == k && r > k && r < b) D[r][k] /= D[k][k];
    __syncthreads();
    if (r < b && c > k && c <= r) D[r][c] -= D[r][k] * D[c][k];
    __syncthreads();
  }
  if (r < b && c <= r) L[at(n, k0 + r, k0 + c)] = D[r][c];
}

// The rows below panel k0: x L_kk^T = a for each row's panel slice x.
__global__ void k_dense_panel_solve(int n, int k0, double* __restrict__ L) {
  pdl_entry();
  __shared__ double D[kNb][kNb + 1];
  const int b = min(kNb, n - k0);
  for (int e = threadIdx.x; e < kNb * kNb; e += blockDim.x) {
    const int r = e / kNb, c = e % kNb;
    D[r][c] = r < b && c <= r ? L[at(n, k0 + r, k0 + c)] : 0.0;
  }
  __syncthreads();
  const int i = k0 + b + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x[kNb];
#pragma unroll
  for (int c = 0; c < kNb; ++c) x[c] = c < b ? L[at(n, i, k0 + c)] : 0.0;
#pragma unroll
  for (int c = 0; c < kNb; ++c) {
    if (c >= b) break;
    double v = x[c];
    for (int m = 0; m < c; ++m) v -= x[m] * D[c][m];
    x[c] = v / D[c][c];
  }
#pragma unroll
  for (int c = 0; c < kNb; ++c)
    if (c < b) L[at(n, i, k0 + c)] = x[c];
}

// Trailing update below panel k0: L_ij -= sum_c L_ic L_jc over the panel's
// columns, for j <= i in the rows after the panel. Block (bx, by) of the
// grid is tile (ti, tj) = (by, bx) of the trailing part; tiles above the
// diagonal do nothing.
__global__ void __launch_bounds__(kNbThreads)
    k_dense_panel_update(int n, int k0, double* __restrict__ L) {
  pdl_entry();
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (tj > ti) return;
  __shared__ double Pi[kNb][kNb + 1], Pj[kNb][kNb + 1];
  const int b = min(kNb, n - k0);
  const int base = k0 + b;
  const int r = threadIdx.x / kNb, c = threadIdx.x % kNb;
  const int i0 = base + ti * kNb, j0 = base + tj * kNb;
  Pi[r][c] = i0 + r < n && c < b ? L[at(n, i0 + r, k0 + c)] : 0.0;
  Pj[r][c] = j0 + r < n && c < b ? L[at(n, j0 + r, k0 + c)] : 0.0;
  __syncthreads();
  const int i = i0 + r, j = j0 + c;
  if (i >= n || j >= n || j > i) return;
  double sum = 0.0;
  for (int m = 0; m < b; ++m) sum += Pi[r][m] * Pj[c][m];
  L[at(n, i, j)] -= sum;
}

// X_pp = L_pp^-1 for every diagonal block p (a CTA each), into W.
__global__ void __launch_bounds__(kNbThreads)
    k_dense_block_inverse(int n, const double* __restrict__ L, double* __restrict__ W) {
  pdl_entry();
  __shared__ double D[kNb][kNb + 1], X[kNb][kNb + 1];
  const int k0 = blockIdx.x * kNb;
  const int b = min(kNb, n - k0);
  const int r = threadIdx.x / kNb, c = threadIdx.x % kNb;
  D[r][c] = r < b && c <= r ? L[at(n, k0 + r, k0 + c)] : 0.0;
  X[r][c] = 0.0;
  __syncthreads();
  // Column c of X: L_pp X[:, c] = e_c, forward substitution by thread (0, c).
  if (r == 0 && c < b) {
    for (int i = c; i < b; ++i) {
      double v = i == c ? 1.0 : 0.0;
      for (int m = c; m < i; ++m) v -= D[i][m] * X[m][c];
      X[i][c] = v / D[i][i];
    }
  }
  __syncthreads();
  if (r < b && c <= r) W[at(n, k0 + r, k0 + c)] = X[r][c];
}

// Block diagonal d of X: X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj, i = j + d
// (block indices), a CTA per j.
__global__ void __launch_bounds__(kNbThreads)
    k_dense_block_offdiag(int n, int d, const double* __restrict__ L, double* __restrict__ W) {
  pdl_entry();
  __shared__ double A[kNb][kNb + 1], B[kNb][kNb + 1];
  const int jb = blockIdx.x, ib = jb + d;
  const int i0 = ib * kNb, j0 = jb * kNb;
  const int r = threadIdx.x / kNb, c = threadIdx.x % kNb;
  double sum = 0.0;  // S[r][c]
  for (int kb = jb; kb < ib; ++kb) {
    const int k0 = kb * kNb;
    // A = L_ik (rows i0.., columns k0..), B = X_kj (rows k0.., columns j0..);
    // X_kj is lower triangular when k == j.
    A[r][c] = i0 + r < n ? L[at(n, i0 + r, k0 + c)] : 0.0;
    B[r][c] = k0 + r < n && (kb > jb || c <= r) ? W[at(n, k0 + r, j0 + c)] : 0.0;
    __syncthreads();
    for (int m = 0; m < kNb; ++m) sum += A[r][m] * B[m][c];
    __syncthreads();
  }
  // X_ij = -X_ii S, X_ii lower triangular.
  A[r][c] = i0 + r < n && c <= r ? W[at(n, i0 + r, i0 + c)] : 0.0;
  B[r][c] = sum;
  __syncthreads();
  double x = 0.0;
  for (int m = 0; m <= r; ++m) x -= A[r][m] * B[m][c];
  if (i0 + r < n && j0 + c < n) W[at(n, i0 + r, j0 + c)] = x;
}

// Tile (ti, tj), tj <= ti, of W = X^T X: sum over block rows k >= ti of
// X_k,ti^T X_k,tj (X lower triangular in W), into out (both (i, j) and (j, i)).
__global__ void __launch_bounds__(kNbThreads)
    k_dense_gram(int n, const double* __restrict__ X, double* __restrict__ out) {
  pdl_entry();
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (tj > ti) return;
  __shared__ double A[kNb][kNb + 1], B[kNb][kNb + 1];
  const int nb = (n + kNb - 1) / kNb;
  const int r = threadIdx.x / kNb, c = threadIdx.x % kNb;
  const int i = ti * kNb + r, j = tj * kNb + c;
  double sum = 0.0;
  for (int kb = ti; kb < nb; ++kb) {
    const int k0 = kb * kNb;
    // A[m][r] = X[k0 + m][ti*32 + r], B[m][c] = X[k0 + m][tj*32 + c] (zero above the diagonal).
    const int kr = k0 + r;
    A[r][c] = kr < n && ti * kNb + c < n && ti * kNb + c <= kr ? X[at(n, kr, ti * kNb + c)] : 0.0;
    B[r][c] = kr < n && tj * kNb + c < n && tj * kNb + c <= kr ? X[at(n, kr, tj * kNb + c)] : 0.0;
    __syncthreads();
    for (int m = 0; m < kNb; ++m) sum += A[m][r] * B[m][c];
    __syncthreads();
  }
  if (i < n && j < n) {
    out[at(n, i, j)] = sum;
    out[at(n, j, i)] = sum;
  }
}

__global__ void k_dense_copy(std::size_t count, const double* __restrict__ from,
                             double* __restrict__ to) {
  pdl_entry();
  for (std::size_t k = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; k < count;
       k += static_cast<std::size_t>(gridDim.x) * blockDim.x)
    to[k] = from[k];
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
  // Blocked, over many CTAs (see k_dense_panel_factor and the kernels after it).
  const std::size_t count = static_cast<std::size_t>(n) * n;
  const int nb = (n + kNb - 1) / kNb;
  const int fill = static_cast<int>(std::min<std::size_t>((count + kBlock - 1) / kBlock, 1184));
  counter += 4 * nb + 2;
  pdl(k_dense_zero, fill, kBlock, 0, s, count, lower);
  pdl(k_dense_scatter, (n + kBlock - 1) / kBlock, kBlock, 0, s, n, rows, cols, vals, lower, error,
      ratio);
  for (int p = 0; p < nb; ++p) {
    const int k0 = p * kNb;
    pdl(k_dense_panel_factor, 1, kNbThreads, 0, s, n, k0, lower, error, ratio);
    const int below = n - k0 - kNb;
    if (below > 0) {
      pdl(k_dense_panel_solve, (below + 127) / 128, 128, 0, s, n, k0, lower);
      const int tiles = (below + kNb - 1) / kNb;
      pdl(k_dense_panel_update, dim3(tiles, tiles), kNbThreads, 0, s, n, k0, lower);
    }
  }
  pdl(k_dense_block_inverse, nb, kNbThreads, 0, s, n, static_cast<const double*>(lower), inverse);
  for (int d = 1; d < nb; ++d)
    pdl(k_dense_block_offdiag, nb - d, kNbThreads, 0, s, n, d, static_cast<const double*>(lower),
        inverse);
  pdl(k_dense_gram, dim3(nb, nb), kNbThreads, 0, s, n, static_cast<const double*>(inverse), lower);
  pdl(k_dense_copy, fill, kBlock, 0, s, count, static_cast<const double*>(lower), inverse);
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
