// Reference-parity solver kernels for sm_100a (compiled with --fmad=false).
//
// Each kernel computes exactly the float operations, in exactly the order, of
// the reference kernel it replaces (cited per kernel), so every per-row value is
// bit-identical to the reference's CPU path. Reductions accumulate in FP64 in a
// fixed tree; they are fused into the kernel that produces their operand and the
// last block runs the reference's single-thread scalar update as an epilogue,
// so a PCG iteration is a handful of launches instead of a dozen.
#include "common.cuh"
#include "kernels.hpp"

#include <algorithm>
#include <atomic>
#include <cstdlib>

namespace kb2 {
namespace dev {
bool pdl_enabled() {
  static const bool enabled = [] {
    const char* v = std::getenv("KUTTA_B200_PDL");
    return v == nullptr || v[0] != '0';
  }();
  return enabled;
}
}  // namespace dev
namespace {
using namespace dev;

#define ROWS(i, n) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

__device__ __forceinline__ Reducer as_reducer(DeviceReducer r) { return Reducer{r.partials, r.ticket}; }

// ---- scalar updates, src/kutta/kernels/scalars.kern.h:51-121 -----------------
__device__ void epilogue(Epilogue e, float* sc, int* st) {
  switch (e) {
    case Epilogue::None:
      return;
    case Epilogue::PcgAlpha: {  // solver_pcg_alpha :63-71
      if (st[0] != 0) return;
      const Pair rho = kp_load(sc, 0), pq = kp_load(sc, 2);
      const Pair alpha = kp_div(rho, pq);
      if (!kp_positive(rho) || !kp_positive(pq) || !kp_coefficient(alpha) || kp_zero(alpha))
        st[0] = 2;
      else
        kp_store(sc, 8, alpha);
      return;
    }
    case Epilogue::PcgBeta:
    case Epilogue::PcgBetaFlexible: {  // solver_pcg_beta :72-80
      if (st[0] != 0) return;
      const Pair next = kp_load(sc, 4);
      const Pair numer = e == Epilogue::PcgBetaFlexible
                             ? kp_neg(kp_mul(kp_load(sc, 8), kp_load(sc, 6)))
                             : next;
      const Pair beta = kp_div(numer, kp_load(sc, 0));
      if (!kp_positive(next) || !kp_coefficient(beta) || (kp_zero(beta) && !kp_zero(numer)))
        st[0] = 2;
      else {
        kp_store(sc, 10, beta);
        kp_store(sc, 0, next);
      }
      return;
    }
    case Epilogue::BicgBeta: {  // solver_bicg_beta :81-89
      if (st[0] != 0) return;
      const Pair rho = kp_load(sc, 0), omega = kp_load(sc, 12);
      const Pair beta = kp_mul(kp_div(rho, kp_load(sc, 14)), kp_div(kp_load(sc, 8), omega));
      if (kp_zero(rho) || !kp_finite(rho) || kp_zero(omega) || !kp_coefficient(omega) ||
          !kp_coefficient(beta) || kp_zero(beta))
        st[0] = 2;
      else {
        kp_store(sc, 10, beta);
        st[2] = 0;
      }
      return;
    }
    case Epilogue::BicgAlpha: {  // solver_bicg_alpha :90-97
      if (st[0] != 0) return;
      const Pair rv = kp_load(sc, 2);
      const Pair alpha = kp_div(kp_load(sc, 0), rv);
      if (kp_zero(rv) || !kp_finite(rv) || !kp_coefficient(alpha) || kp_zero(alpha))
        st[0] = 2;
      else
        kp_store(sc, 8, alpha);
      return;
    }
    case Epilogue::BicgS: {  // solver_bicg_s :98-103
      if (st[0] != 0) return;
      ++st[1];
      st[2] = kp_le(kp_load(sc, 16), kp_load(sc, 20)) ? 1 : 0;
      return;
    }
    case Epilogue::BicgOmega: {  // solver_bicg_omega :104-112
      if (st[0] != 0) return;
      if (st[2] != 0) {
        kp_store(sc, 12, kp(0.0f, 0.0f));
        return;
      }
      const Pair tt = kp_load(sc, 2), ts = kp_load(sc, 4);
      const Pair omega = kp_div(ts, tt);
      if (!kp_positive(tt) || !kp_finite(tt) || kp_zero(omega) || !kp_coefficient(omega))
        st[0] = 2;
      else
        kp_store(sc, 12, omega);
      return;
    }
    case Epilogue::CheckPcg:
    case Epilogue::CheckBicg: {  // solver_check :113-121
      if (st[0] != 0) return;
      const bool pcg = e == Epilogue::CheckPcg;
      if (pcg) ++st[1];
      const Pair rr = kp_load(sc, 18);
      if (!kp_finite(rr) || kp_le(rr, kp_load(sc, 20)) || !kp_le(rr, kp_load(sc, 22)) ||
          st[1] % 50 == 0)
        st[0] = 1;
      if (!pcg) kp_store(sc, 14, kp_load(sc, 0));
      return;
    }
  }
}

// Block partial -> grid total -> pair store -> epilogue, in the last block.
__device__ __forceinline__ void finish(const Reducer& red, double a, double b, bool dual,
                                       float* scalars, int offset, int* status, Epilogue epi) {
  __shared__ double shared[32];
  a = block_sum(a, shared);
  if (dual) b = block_sum(b, shared);
  if (!publish(red, a, b, dual)) return;
  const double total_a = gather(red, 0, shared);
  const double total_b = dual ? gather(red, 1, shared) : 0.0;
  if (threadIdx.x == 0) {
    store_pair(scalars, offset, total_a);
    if (dual) store_pair(scalars, offset + 2, total_b);
    epilogue(epi, scalars, status);
    *red.ticket = 0;
  }
}

// ---- CSR row kernels --------------------------------------------------------
// One row per thread: on the 5-entry fine rows this direct form measured
// fastest (74% of the copy peak); staging tiles in shared memory or
// register-chunking the row both measured slower there.

// csr_spmv / csr_spmv_guarded, linalg.kern.h:5-16,111-114.
__global__ void k_spmv(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                       const float* __restrict__ vals, const float* __restrict__ x,
                       float* __restrict__ y, const int* __restrict__ status) {
  pdl_entry();
  if (status && status[0] != 0) return;
  ROWS(i, n) {
    float sum = 0.0f, error = 0.0f;
    const int end = rows[i + 1];
    for (int j = rows[i]; j < end; ++j) kahan_term(sum, error, vals[j], x[cols[j]]);
    y[i] = sum;
  }
}

// csr_spmv_guarded + dot_into(w, q) + a scalar kernel: PCG's p.q and alpha
// (solver.cpp:288-290, w = p) or BiCGStab's rhat.q and alpha (:335-337, w = rhat).
__global__ void k_spmv_dot(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                           const float* __restrict__ vals, const float* __restrict__ p,
                           const float* __restrict__ w, float* __restrict__ q, DeviceReducer red,
                           float* scalars, int offset, int* status, Epilogue epi) {
  pdl_entry();
  if (status[0] != 0) return;
  double acc = 0;
  ROWS(i, n) {
    float sum = 0.0f, error = 0.0f;
    const int end = rows[i + 1];
    for (int j = rows[i]; j < end; ++j) kahan_term(sum, error, vals[j], p[cols[j]]);
    q[i] = sum;
    acc += static_cast<double>(w[i]) * static_cast<double>(sum);
  }
  finish(as_reducer(red), acc, 0, false, scalars, offset, status, epi);
}

// csr_residual / csr_residual_guarded, linalg.kern.h:32-50,115-118.
__global__ void k_residual(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                           const float* __restrict__ vals, const float* __restrict__ x,
                           const float* __restrict__ b, float* __restrict__ r,
                           const int* __restrict__ status) {
  pdl_entry();
  if (status && status[0] != 0) return;
  ROWS(i, n) {
    float sum = b[i], error = 0.0f;
    const int end = rows[i + 1];
    for (int j = rows[i]; j < end; ++j) residual_term(sum, error, vals[j], x[cols[j]]);
    r[i] = sum + error;
  }
}

// amg_smooth_zero's row (linalg.kern.h:162-170): the caller has just cleared x,
// so only a nonfinite b takes the ordinary path, with x = 0.
__device__ __forceinline__ float zero_sweep_row(int i, const int* __restrict__ rows,
                                                const float* __restrict__ vals, float bi,
                                                float inv) {
  if (!nonfinite(bi)) return 0.0f + (2.0f / 3.0f) * inv * (bi + 0.0f);
  float sum = bi, error = 0.0f;
  const int end = rows[i + 1];
  for (int j = rows[i]; j < end; ++j) residual_term(sum, error, vals[j], 0.0f);
  return 0.0f + (2.0f / 3.0f) * inv * (sum + error);
}

// amg_smooth (linalg.kern.h:150-156) and amg_smooth_zero (:162-170).
template <bool kZero>
__global__ void k_smooth(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                         const float* __restrict__ vals, const float* __restrict__ x,
                         const float* __restrict__ b, const float* __restrict__ inv,
                         float* __restrict__ next, const int* __restrict__ status) {
  pdl_entry();
  if (status && status[0] != 0) return;
  ROWS(i, n) {
    if (kZero) {
      next[i] = zero_sweep_row(i, rows, vals, b[i], inv[i]);
      continue;
    }
    float sum = b[i], error = 0.0f;
    const int end = rows[i + 1];
    for (int j = rows[i]; j < end; ++j) residual_term(sum, error, vals[j], x[cols[j]]);
    next[i] = x[i] + (2.0f / 3.0f) * inv[i] * (sum + error);
  }
}

// The fine-level post-sweep of the flexible PCG (mixed solve) with the two
// reductions that follow the preconditioner fused in: next as
// k_smooth<false>, then b.next and next.q (b the Krylov residual r, next the
// preconditioned z, q = A p) into scalars[offset..] with the epilogue, as
// reduce_into(Dot2, r, z, z, q) computes them: the same grid, the same row
// loop and the same products, so the same totals bit for bit.
__global__ void k_smooth_dot2(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                              const float* __restrict__ vals, const float* __restrict__ x,
                              const float* __restrict__ b, const float* __restrict__ inv,
                              float* __restrict__ next, const float* __restrict__ q,
                              DeviceReducer red, float* scalars, int offset, int* status,
                              Epilogue epi) {
  pdl_entry();
  if (status[0] != 0) return;
  double a = 0, c = 0;
  ROWS(i, n) {
    float sum = b[i], error = 0.0f;
    const int end = rows[i + 1];
    for (int j = rows[i]; j < end; ++j) residual_term(sum, error, vals[j], x[cols[j]]);
    const float z = x[i] + (2.0f / 3.0f) * inv[i] * (sum + error);
    next[i] = z;
    a += static_cast<double>(b[i]) * static_cast<double>(z);
    c += static_cast<double>(z) * static_cast<double>(q[i]);
  }
  finish(as_reducer(red), a, c, true, scalars, offset, status, epi);
}

// ---- Packed rows (the mixed solve's fine operator) ---------------------------
// The kernels are bounded to 32 registers a thread (8 blocks of 256 per SM):
// their grids are the CSR kernels' (8 blocks per SM, one resident wave), and
// at more registers part of the grid would wait for a second wave.
// The row's values, absolute columns and diagonal, loaded with 128-bit (and
// 64-bit) loads that stream past the caches: the operator is read once per
// pass, the gathered vectors are what the caches should keep.
template <int W>
struct PackedRow {
  float v[W];
  int c[W];
  float d;
};
template <int W>
__device__ __forceinline__ PackedRow<W> packed_row(int i, const float* __restrict__ vals,
                                                   const short* __restrict__ offsets,
                                                   const float* __restrict__ diag) {
  PackedRow<W> row;
  const float4* v4 = reinterpret_cast<const float4*>(vals) + static_cast<std::size_t>(i) * (W / 4);
#pragma unroll
  for (int q = 0; q < W / 4; ++q) {
    const float4 a = __ldcs(v4 + q);
    row.v[4 * q] = a.x;
    row.v[4 * q + 1] = a.y;
    row.v[4 * q + 2] = a.z;
    row.v[4 * q + 3] = a.w;
  }
  unsigned words[W / 2];
  if constexpr (W == 4) {
    const uint2 o = __ldcs(reinterpret_cast<const uint2*>(offsets) + i);
    words[0] = o.x;
    words[1] = o.y;
  } else {
    const uint4 o = __ldcs(reinterpret_cast<const uint4*>(offsets) + i);
    words[0] = o.x;
    words[1] = o.y;
    words[2] = o.z;
    words[3] = o.w;
  }
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const int off = static_cast<short>((words[k / 2] >> (16 * (k & 1))) & 0xffffu);
    row.c[k] = i + off;
  }
  row.d = __ldcs(diag + i);
  return row;
}

// residual_term with the product's rounding error taken by one FMA instead of
// Dekker's 4097 split: both give the exact error of v x when neither factor
// exceeds 1e30 (the split's guard, kept) and no partial product underflows,
// so the sums agree bit for bit there at a third of the instructions, which
// keeps these streaming kernels memory-bound.
__device__ __forceinline__ void residual_term_fma(float& sum, float& error, float v, float x) {
  const float product = v * x;
  const float term = -product;
  const float next = sum + term;
  error += fabsf(sum) >= fabsf(term) ? (sum - next) + term : (term - next) + sum;
  if (fabsf(v) <= 1.0e30f && fabsf(x) <= 1.0e30f) error -= fmaf(v, x, -product);
  sum = next;
}

// sum = b_i - sum_j a_ij x_j with residual_term_fma, in CSR column order;
// unused slots (column i) are skipped.
template <int W>
__device__ __forceinline__ float packed_residual_row(int i, const PackedRow<W>& row, float bi,
                                                     const float* __restrict__ x) {
  float xv[W];
#pragma unroll
  for (int k = 0; k < W; ++k) xv[k] = x[row.c[k]];
  const float xi = x[i];
  float sum = bi, error = 0.0f;
#pragma unroll
  for (int k = 0; k < W; ++k)
    if (row.c[k] < i) residual_term_fma(sum, error, row.v[k], xv[k]);
  residual_term_fma(sum, error, row.d, xi);
#pragma unroll
  for (int k = 0; k < W; ++k)
    if (row.c[k] > i) residual_term_fma(sum, error, row.v[k], xv[k]);
  return sum + error;
}

template <int W>
__global__ void __launch_bounds__(kBlock, 8) k_packed_residual(int n, const float* __restrict__ vals,
                                  const short* __restrict__ offsets, const float* __restrict__ diag,
                                  const float* __restrict__ x, const float* __restrict__ b,
                                  float* __restrict__ r, const int* __restrict__ status) {
  pdl_entry();
  if (status && status[0] != 0) return;
  ROWS(i, n) {
    const PackedRow<W> row = packed_row<W>(i, vals, offsets, diag);
    r[i] = packed_residual_row<W>(i, row, b[i], x);
  }
}

// k_smooth_dot2 on packed rows.
template <int W>
__global__ void __launch_bounds__(kBlock, 8) k_packed_smooth_dot2(int n, const float* __restrict__ vals,
                                     const short* __restrict__ offsets,
                                     const float* __restrict__ diag, const float* __restrict__ x,
                                     const float* __restrict__ b, const float* __restrict__ inv,
                                     float* __restrict__ next, const float* __restrict__ q,
                                     DeviceReducer red, float* scalars, int offset, int* status,
                                     Epilogue epi) {
  pdl_entry();
  if (status[0] != 0) return;
  double a = 0, c = 0;
  ROWS(i, n) {
    const PackedRow<W> row = packed_row<W>(i, vals, offsets, diag);
    const float bi = b[i];
    const float z = x[i] + (2.0f / 3.0f) * inv[i] * packed_residual_row<W>(i, row, bi, x);
    next[i] = z;
    a += static_cast<double>(bi) * static_cast<double>(z);
    c += static_cast<double>(z) * static_cast<double>(q[i]);
  }
  finish(as_reducer(red), a, c, true, scalars, offset, status, epi);
}

// k_spmv_dot on packed rows (Kahan sum in CSR column order).
template <int W>
__global__ void __launch_bounds__(kBlock, 8) k_packed_spmv_dot(int n, const float* __restrict__ vals,
                                  const short* __restrict__ offsets,
                                  const float* __restrict__ diag, const float* __restrict__ p,
                                  const float* __restrict__ w, float* __restrict__ q,
                                  DeviceReducer red, float* scalars, int offset, int* status,
                                  Epilogue epi) {
  pdl_entry();
  if (status[0] != 0) return;
  double acc = 0;
  ROWS(i, n) {
    const PackedRow<W> row = packed_row<W>(i, vals, offsets, diag);
    float pv[W];
#pragma unroll
    for (int k = 0; k < W; ++k) pv[k] = p[row.c[k]];
    const float pi = p[i];
    float sum = 0.0f, error = 0.0f;
#pragma unroll
    for (int k = 0; k < W; ++k)
      if (row.c[k] < i) kahan_term(sum, error, row.v[k], pv[k]);
    kahan_term(sum, error, row.d, pi);
#pragma unroll
    for (int k = 0; k < W; ++k)
      if (row.c[k] > i) kahan_term(sum, error, row.v[k], pv[k]);
    q[i] = sum;
    acc += static_cast<double>(w[i]) * static_cast<double>(sum);
  }
  finish(as_reducer(red), acc, 0, false, scalars, offset, status, epi);
}

// Values of the packed rows: the row's off-diagonal values in column order,
// then zeros; the diagonal apart.
__global__ void k_pack_rows(int n, int width, const int* __restrict__ rows,
                            const int* __restrict__ diag_index, const float* __restrict__ vals,
                            float* __restrict__ packed, float* __restrict__ packed_diag) {
  pdl_entry();
  ROWS(i, n) {
    float* out = packed + static_cast<std::size_t>(i) * width;
    int k = 0;
    const int d = diag_index[i];
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      if (j != d) out[k++] = vals[j];
    for (; k < width; ++k) out[k] = 0.0f;
    packed_diag[i] = vals[d];
  }
}

// amg_coarse_solve, linalg.kern.h:126-147: whole <=24-row system in one thread.
__global__ void k_coarse_solve(int count, const int* __restrict__ rows,
                               const int* __restrict__ cols, const float* __restrict__ vals,
                               float* __restrict__ x, const float* __restrict__ b,
                               const float* __restrict__ inv, const int* __restrict__ status,
                               int sweeps) {
  pdl_entry();
  if (threadIdx.x != 0 || blockIdx.x != 0 || status[0] != 0) return;
  float current[24], r[24];
  for (int row = 0; row < count; ++row) current[row] = 0.0f;
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    for (int row = 0; row < count; ++row) {
      float sum = b[row], error = 0.0f;
      for (int j = rows[row]; j < rows[row + 1]; ++j)
        residual_term(sum, error, vals[j], current[cols[j]]);
      r[row] = sum + error;
    }
    for (int row = 0; row < count; ++row) current[row] += (2.0f / 3.0f) * inv[row] * r[row];
  }
  for (int row = 0; row < count; ++row) x[row] = current[row];
}

// krylov_diagonal, linalg.kern.h:52-70, with the refresh's max_abs check of the
// invalid flags fused (amg.cpp:236-240).
__global__ void k_diagonal(int n, const int* __restrict__ rows, const int* __restrict__ diag,
                           const float* __restrict__ vals, float* __restrict__ inverse,
                           int use_l1, DeviceReducer red, double* check, int slot) {
  pdl_entry();
  double worst = 0;
  ROWS(i, n) worst = nan_max(worst, diagonal_row(i, rows, diag, vals, inverse, use_l1));
  __shared__ double shared[32];
  worst = block_max(worst, shared);
  const Reducer r = as_reducer(red);
  if (!publish(r, worst, 0, false)) return;
  const double total = gather_max(r, shared);
  if (threadIdx.x == 0) {
    check[slot] = total;
    *r.ticket = 0;
  }
}

// ---- AMG transfer and Galerkin, src/kutta/kernels/amg.kern.h ------------------
// amg_restrict(_guarded) :5-16,84-87: Kahan sum over the aggregate's members.
__global__ void k_restrict(int nc, const int* __restrict__ offsets,
                           const int* __restrict__ members, const float* __restrict__ fine,
                           float* __restrict__ coarse, const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  ROWS(g, nc) {
    float sum = 0.0f, error = 0.0f;
    for (int j = offsets[g]; j < offsets[g + 1]; ++j) {
      const float term = fine[members[j]] - error;
      const float next = sum + term;
      error = (next - sum) - term;
      sum = next;
    }
    coarse[g] = sum;
  }
}

// amg_prolong(_guarded) :18-21,88-91.
__global__ void k_prolong(int nf, const int* __restrict__ aggregate,
                          const float* __restrict__ coarse, float* __restrict__ fine,
                          const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  ROWS(i, nf) {
    const int g = aggregate[i];
    if (g >= 0) fine[i] += coarse[g];
  }
}

// amg_galerkin :27-38: Neumaier sum over the coarse entry's fine entries.
__global__ void k_galerkin(int nnz_c, const int* __restrict__ offsets,
                           const int* __restrict__ entries, const float* __restrict__ fine,
                           float* __restrict__ coarse) {
  pdl_entry();
  ROWS(e, nnz_c) {
    float sum = 0.0f, error = 0.0f;
    for (int j = offsets[e]; j < offsets[e + 1]; ++j) neumaier_term(sum, error, fine[entries[j]]);
    coarse[e] = sum + error;
  }
}

// amg_m_matrix_diagonal :44-58 in two passes with the same roundings in the
// same order: each fine row's surplus (its diagonal plus its off-diagonals,
// upward rounded), independent per row and computed in parallel; then, per
// coarse row, the upward-rounded sum of its members' surpluses in member
// order minus its stored off-diagonals. Splitting the member loop out of the
// per-coarse-row chain shortens the dependent sequence of each thread.
__global__ void k_row_surplus(int n, const int* __restrict__ rows, const int* __restrict__ diag,
                              const float* __restrict__ fine, float* __restrict__ surplus) {
  pdl_entry();
  ROWS(i, n) {
    UpperSum sum{fine[diag[i]], 0.0f};
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      if (j != diag[i]) sum = upper_add(sum, fine[j]);
    surplus[i] = upper_value(sum);
  }
}

__global__ void k_m_matrix_combine(int nc, const int* __restrict__ offsets,
                                   const int* __restrict__ members,
                                   const float* __restrict__ surplus, const int* __restrict__ rows,
                                   const int* __restrict__ diag, float* coarse) {
  pdl_entry();
  ROWS(g, nc) {
    UpperSum diagonal{0.0f, 0.0f};
    for (int m = offsets[g]; m < offsets[g + 1]; ++m)
      diagonal = upper_add(diagonal, surplus[members[m]]);
    for (int j = rows[g]; j < rows[g + 1]; ++j)
      if (j != diag[g]) diagonal = upper_add(diagonal, -coarse[j]);
    coarse[diag[g]] = upper_value(diagonal);
  }
}

// ---- Krylov vector updates, scalars.kern.h:122-152 ---------------------------
// solver_step :122-127 + dot_into(r, r -> 18) + solver_check(pcg) (solver.cpp:291-293).
__global__ void k_pcg_step_dot(int n, float* __restrict__ x, float* __restrict__ r,
                               const float* __restrict__ p, const float* __restrict__ q,
                               DeviceReducer red, float* scalars, int* status) {
  pdl_entry();
  if (status[0] != 0) return;
  const float alpha = kp_float(kp_load(scalars, 8));
  double acc = 0;
  ROWS(i, n) {
    x[i] += alpha * p[i];
    const float ri = r[i] - alpha * q[i];
    r[i] = ri;
    acc += static_cast<double>(ri) * static_cast<double>(ri);
  }
  finish(as_reducer(red), acc, 0, false, scalars, 18, status, Epilogue::CheckPcg);
}

// solver_direction :128-131.
__global__ void k_direction(int n, const float* __restrict__ z, float* __restrict__ p,
                            const float* __restrict__ scalars, const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  const float beta = kp_float(kp_load(scalars, 10));
  ROWS(i, n) p[i] = z[i] + beta * p[i];
}

// solver_bicg_direction :132-137.
__global__ void k_bicg_direction(int n, const float* __restrict__ r, const float* __restrict__ v,
                                 float* __restrict__ p, const float* __restrict__ scalars,
                                 const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  const float beta = kp_float(kp_load(scalars, 10)), omega = kp_float(kp_load(scalars, 12));
  ROWS(i, n) p[i] = r[i] + beta * (p[i] - omega * v[i]);
}

// solver_bicg_difference :138-141.
__global__ void k_bicg_difference(int n, const float* __restrict__ r, const float* __restrict__ q,
                                  float* __restrict__ sv, const float* __restrict__ scalars,
                                  const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  const float alpha = kp_float(kp_load(scalars, 8));
  ROWS(i, n) sv[i] = r[i] - alpha * q[i];
}

// solver_bicg_step :142-149.
__global__ void k_bicg_step(int n, float* __restrict__ x, float* __restrict__ r,
                            const float* __restrict__ z, const float* __restrict__ zs,
                            const float* __restrict__ sv, const float* __restrict__ t,
                            const float* __restrict__ scalars, const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  const float alpha = kp_float(kp_load(scalars, 8)), omega = kp_float(kp_load(scalars, 12));
  const bool s_only = status[2] != 0;
  ROWS(i, n) {
    if (s_only) {
      x[i] += alpha * z[i];
      r[i] = sv[i];
    } else {
      x[i] += alpha * z[i] + omega * zs[i];
      r[i] = sv[i] - omega * t[i];
    }
  }
}

// krylov_multiply(_guarded), linalg.kern.h:72-75,119-122.
__global__ void k_multiply(int n, const float* __restrict__ r, const float* __restrict__ inverse,
                           float* __restrict__ z, const int* __restrict__ status) {
  pdl_entry();
  if (status && status[0] != 0) return;
  ROWS(i, n) z[i] = r[i] * inverse[i];
}

// axpy, blas.kern.h:5.
__global__ void k_axpy(int n, float* __restrict__ y, const float* __restrict__ x, float a) {
  pdl_entry();
  ROWS(i, n) y[i] = y[i] + a * x[i];
}

__global__ void k_fill(int n, float* __restrict__ x, float value) {
  pdl_entry(); ROWS(i, n) x[i] = value; }

// ---- reductions ---------------------------------------------------------------
// Device::reduce_into (device.hpp:186-202) with FP64 accumulation.
__global__ void k_reduce_into(ReduceMode mode, int n, const float* __restrict__ x,
                              const float* __restrict__ y, const float* __restrict__ u,
                              const float* __restrict__ v, DeviceReducer red, float* scalars,
                              int offset, int* status, bool guard, Epilogue epi) {
  pdl_entry();
  if (guard && status[0] != 0) return;
  double a = 0, b = 0;
  const bool dual = mode == ReduceMode::Dot2;
  ROWS(i, n) {
    a += mode == ReduceMode::Sum ? static_cast<double>(x[i])
                                 : static_cast<double>(x[i]) * static_cast<double>(y[i]);
    if (dual) b += static_cast<double>(u[i]) * static_cast<double>(v[i]);
  }
  finish(as_reducer(red), a, b, dual, scalars, offset, status, epi);
}

// Host reductions (Device::sum/dot/max_abs): the FP64 value into out[slot].
__global__ void k_reduce_value(ReduceMode mode, int n, const float* __restrict__ x,
                               const float* __restrict__ y, DeviceReducer red, double* out,
                               int slot) {
  pdl_entry();
  __shared__ double shared[32];
  double a = 0;
  ROWS(i, n) {
    if (mode == ReduceMode::MaxAbs) a = nan_max(a, fabs(static_cast<double>(x[i])));
    else if (mode == ReduceMode::Sum) a += static_cast<double>(x[i]);
    else a += static_cast<double>(x[i]) * static_cast<double>(y[i]);
  }
  const Reducer r = as_reducer(red);
  a = mode == ReduceMode::MaxAbs ? block_max(a, shared) : block_sum(a, shared);
  if (!publish(r, a, 0, false)) return;
  const double total = mode == ReduceMode::MaxAbs ? gather_max(r, shared) : gather(r, 0, shared);
  if (threadIdx.x == 0) {
    out[slot] = total;
    *r.ticket = 0;
  }
}

// solver_limits :51-55 (all 24 slots).
__global__ void k_solver_limits(float* scalars, float th, float tl, float dh, float dl) {
  pdl_entry();
  const int i = threadIdx.x;
  if (i < 24)
    scalars[i] = i == 20 ? th : (i == 21 ? tl : (i == 22 ? dh : (i == 23 ? dl : 0.0f)));
}

// solver_reset :56-62.
__global__ void k_solver_reset(float* scalars, int* status, int iterations) {
  pdl_entry();
  status[0] = 0;
  status[1] = iterations;
  status[2] = 0;
  scalars[8] = 1.0f;
  scalars[9] = 0.0f;
  scalars[12] = 1.0f;
  scalars[13] = 0.0f;
  scalars[14] = 1.0f;
  scalars[15] = 0.0f;
}

// solver_project :150-152.
__global__ void k_project(int n, float* __restrict__ x, const float* __restrict__ sum,
                          float count_hi, float count_lo) {
  pdl_entry();
  const float mean = kp_float(kp_div(kp_load(sum, 0), kp(count_hi, count_lo)));
  ROWS(i, n) x[i] -= mean;
}

// ---- K-cycle inner corrections (scalars.kern.h:154-186) ------------------------
// Per-level scalars: [0] p.q (q.q for GCR), [2] b.p / t.p (b.q / t.q), [4] t.t or
// z.q, [6] b.b, [8] alpha, [10] beta. The level's status: 0 running, 1 keep the
// accepted first correction, 2 fall back to the plain first cycle.
__global__ void k_inner_alpha(float* scalars, int* status, const int* parent, int first) {
  pdl_entry();
  if (first != 0) status[0] = parent[0] == 0 ? 0 : 2;
  if (status[0] != 0) return;
  const Pair denom = kp_load(scalars, 0);
  const Pair alpha = kp_div(kp_load(scalars, 2), denom);
  if (!kp_positive(denom) || !kp_coefficient(alpha) ||
      (kp_zero(alpha) && !kp_zero(kp_load(scalars, 2))))
    status[0] = first != 0 ? 2 : 1;
  else
    kp_store(scalars, 8, alpha);
}

__global__ void k_inner_first(int n, const float* __restrict__ b, const float* __restrict__ p,
                              const float* __restrict__ q, float* __restrict__ x,
                              float* __restrict__ t, const float* __restrict__ scalars,
                              const int* __restrict__ status) {
  pdl_entry();
  const bool running = status[0] == 0;
  const float alpha = kp_float(kp_load(scalars, 8));
  ROWS(i, n) {
    x[i] = running ? alpha * p[i] : p[i];
    t[i] = running ? b[i] - alpha * q[i] : 0.0f;
  }
}

// Adaptive exit: keep the first correction when |t|^2 <= |b|^2 / 16.
__global__ void k_inner_check(const float* scalars, int* status) {
  pdl_entry();
  if (status[0] != 0) return;
  if (kp_le(kp_load(scalars, 4), kp_mul(kp(0.0625f, 0.0f), kp_load(scalars, 6)))) status[0] = 1;
}

__global__ void k_inner_beta(float* scalars, int* status) {
  pdl_entry();
  if (status[0] != 0) return;
  const Pair beta = kp_div(kp_neg(kp_load(scalars, 4)), kp_load(scalars, 0));
  if (!kp_coefficient(beta) || (kp_zero(beta) && !kp_zero(kp_load(scalars, 4))))
    status[0] = 1;
  else
    kp_store(scalars, 10, beta);
}

__global__ void k_inner_step(int n, float* __restrict__ x, const float* __restrict__ p,
                             const float* __restrict__ scalars, const int* __restrict__ status) {
  pdl_entry();
  if (status[0] != 0) return;
  const float alpha = kp_float(kp_load(scalars, 8));
  ROWS(i, n) x[i] += alpha * p[i];
}

inline int blocks(int n) { return grid_for(n); }
// Kernels without a reduction: one row per thread below ~2M rows, where that
// measured fastest; above, the 1184-block grid-stride form measured faster
// (fine-level sweep 65.9 us vs 72.1 us at 5.3M rows).
inline int full_grid(int n) {
  if (n >= (1 << 21)) return grid_for(n);
  return n > 0 ? (n + kBlock - 1) / kBlock : 1;
}
static_assert(kReducePartials == kPartials, "reduction scratch size");

}  // namespace

namespace launch {

std::atomic<long long> counter{0};

void spmv(int n, const int* rows, const int* cols, const float* vals, const float* x, float* y,
          const int* status, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_spmv, full_grid(n), kBlock, 0, s, n, rows, cols, vals, x, y, status);
}
void spmv_dot(int n, const int* rows, const int* cols, const float* vals, const float* p,
              const float* w, float* q, DeviceReducer red, float* scalars, int offset,
              int* status, Epilogue epi, cudaStream_t s) {
  ++counter;
  pdl(k_spmv_dot, blocks(n), kBlock, 0, s, n, rows, cols, vals, p, w, q, red, scalars, offset,
                                          status, epi);
}
void residual(int n, const int* rows, const int* cols, const float* vals, const float* x,
              const float* b, float* r, const int* status, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_residual, full_grid(n), kBlock, 0, s, n, rows, cols, vals, x, b, r, status);
}
void smooth(int n, const int* rows, const int* cols, const float* vals, const float* x,
            const float* b, const float* inv, float* next, const int* status, bool zero_start,
            cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  if (zero_start)
    pdl(k_smooth<true>, full_grid(n), kBlock, 0, s, n, rows, cols, vals, x, b, inv, next, status);
  else
    pdl(k_smooth<false>, full_grid(n), kBlock, 0, s, n, rows, cols, vals, x, b, inv, next, status);
}
void smooth_dot2(int n, const int* rows, const int* cols, const float* vals, const float* x,
                 const float* b, const float* inv, float* next, const float* q, DeviceReducer red,
                 float* scalars, int offset, int* status, Epilogue epi, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_smooth_dot2, blocks(n), kBlock, 0, s, n, rows, cols, vals, x, b, inv, next, q, red,
                                             scalars, offset, status, epi);
}
void pack_rows(int n, int width, const int* rows, const int* cols, const int* diag,
               const float* vals, float* packed, float* packed_diag, cudaStream_t s) {
  (void)cols;
  if (n <= 0) return;
  ++counter;
  pdl(k_pack_rows, full_grid(n), kBlock, 0, s, n, width, rows, diag, vals, packed, packed_diag);
}
void packed_residual(int n, PackedRows a, const float* x, const float* b, float* r,
                     const int* status, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  if (a.width == 4)
    pdl(k_packed_residual<4>, full_grid(n), kBlock, 0, s, n, a.vals, a.offsets, a.diag, x, b, r,
        status);
  else
    pdl(k_packed_residual<8>, full_grid(n), kBlock, 0, s, n, a.vals, a.offsets, a.diag, x, b, r,
        status);
}
void packed_spmv_dot(int n, PackedRows a, const float* p, const float* w, float* q,
                     DeviceReducer red, float* scalars, int offset, int* status, Epilogue epi,
                     cudaStream_t s) {
  ++counter;
  if (a.width == 4)
    pdl(k_packed_spmv_dot<4>, blocks(n), kBlock, 0, s, n, a.vals, a.offsets, a.diag, p, w, q, red,
        scalars, offset, status, epi);
  else
    pdl(k_packed_spmv_dot<8>, blocks(n), kBlock, 0, s, n, a.vals, a.offsets, a.diag, p, w, q, red,
        scalars, offset, status, epi);
}
void packed_smooth_dot2(int n, PackedRows a, const float* x, const float* b, const float* inv,
                        float* next, const float* q, DeviceReducer red, float* scalars,
                        int offset, int* status, Epilogue epi, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  if (a.width == 4)
    pdl(k_packed_smooth_dot2<4>, blocks(n), kBlock, 0, s, n, a.vals, a.offsets, a.diag, x, b, inv,
        next, q, red, scalars, offset, status, epi);
  else
    pdl(k_packed_smooth_dot2<8>, blocks(n), kBlock, 0, s, n, a.vals, a.offsets, a.diag, x, b, inv,
        next, q, red, scalars, offset, status, epi);
}
void coarse_solve(int count, const int* rows, const int* cols, const float* vals, float* x,
                  const float* b, const float* inv, const int* status, int sweeps,
                  cudaStream_t s) {
  ++counter;
  pdl(k_coarse_solve, 1, 32, 0, s, count, rows, cols, vals, x, b, inv, status, sweeps);
}
void diagonal(int n, const int* rows, const int* diag, const float* vals, float* inverse,
              int use_l1, DeviceReducer red, double* check, int slot, cudaStream_t s) {
  ++counter;
  pdl(k_diagonal, blocks(n), kBlock, 0, s, n, rows, diag, vals, inverse, use_l1, red, check, slot);
}
void restrict_(int nc, const int* offsets, const int* members, const float* fine, float* coarse,
               const int* status, cudaStream_t s) {
  if (nc <= 0) return;
  ++counter;
  pdl(k_restrict, blocks(nc), kBlock, 0, s, nc, offsets, members, fine, coarse, status);
}
void prolong(int nf, const int* aggregate, const float* coarse, float* fine, const int* status,
             cudaStream_t s) {
  if (nf <= 0) return;
  ++counter;
  pdl(k_prolong, blocks(nf), kBlock, 0, s, nf, aggregate, coarse, fine, status);
}
void galerkin(int nnz_c, const int* offsets, const int* entries, const float* fine, float* coarse,
              cudaStream_t s) {
  if (nnz_c <= 0) return;
  ++counter;
  pdl(k_galerkin, blocks(nnz_c), kBlock, 0, s, nnz_c, offsets, entries, fine, coarse);
}
void m_matrix_diagonal(int nf, int nc, const int* offsets, const int* members, const int* fine_rows,
                       const int* fine_diag, const float* fine, const int* rows, const int* diag,
                       float* coarse, float* surplus, cudaStream_t s) {
  if (nc <= 0) return;
  ++counter;
  pdl(k_row_surplus, full_grid(nf), kBlock, 0, s, nf, fine_rows, fine_diag, fine, surplus);
  ++counter;
  pdl(k_m_matrix_combine, full_grid(nc), kBlock, 0, s, nc, offsets, members, surplus, rows, diag,
                                                      coarse);
}
void pcg_step_dot(int n, float* x, float* r, const float* p, const float* q, DeviceReducer red,
                  float* scalars, int* status, cudaStream_t s) {
  ++counter;
  pdl(k_pcg_step_dot, blocks(n), kBlock, 0, s, n, x, r, p, q, red, scalars, status);
}
void direction(int n, const float* z, float* p, const float* scalars, const int* status,
               cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_direction, blocks(n), kBlock, 0, s, n, z, p, scalars, status);
}
void bicg_direction(int n, const float* r, const float* v, float* p, const float* scalars,
                    const int* status, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_bicg_direction, blocks(n), kBlock, 0, s, n, r, v, p, scalars, status);
}
void bicg_difference(int n, const float* r, const float* q, float* sv, const float* scalars,
                     const int* status, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_bicg_difference, blocks(n), kBlock, 0, s, n, r, q, sv, scalars, status);
}
void bicg_step(int n, float* x, float* r, const float* z, const float* zs, const float* sv,
               const float* t, const float* scalars, const int* status, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_bicg_step, blocks(n), kBlock, 0, s, n, x, r, z, zs, sv, t, scalars, status);
}
void multiply(int n, const float* r, const float* inverse, float* z, const int* status,
              cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_multiply, blocks(n), kBlock, 0, s, n, r, inverse, z, status);
}
void axpy(int n, float* y, const float* x, float a, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_axpy, blocks(n), kBlock, 0, s, n, y, x, a);
}
void fill(int n, float* x, float value, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_fill, blocks(n), kBlock, 0, s, n, x, value);
}
void reduce_into(ReduceMode mode, int n, const float* x, const float* y, const float* u,
                 const float* v, DeviceReducer red, float* scalars, int offset, int* status,
                 bool guard, Epilogue epi, cudaStream_t s) {
  ++counter;
  pdl(k_reduce_into, blocks(n), kBlock, 0, s, mode, n, x, y, u, v, red, scalars, offset, status,
                                             guard, epi);
}
void reduce_value(ReduceMode mode, int n, const float* x, const float* y, DeviceReducer red,
                  double* out, int slot, cudaStream_t s) {
  ++counter;
  pdl(k_reduce_value, blocks(n), kBlock, 0, s, mode, n, x, y, red, out, slot);
}
void solver_limits(float* scalars, float th, float tl, float dh, float dl, cudaStream_t s) {
  ++counter;
  pdl(k_solver_limits, 1, 32, 0, s, scalars, th, tl, dh, dl);
}
void solver_reset(float* scalars, int* status, int iterations, cudaStream_t s) {
  ++counter;
  pdl(k_solver_reset, 1, 1, 0, s, scalars, status, iterations);
}
void project(int n, float* x, const float* sum, float count_hi, float count_lo, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_project, blocks(n), kBlock, 0, s, n, x, sum, count_hi, count_lo);
}
void inner_alpha(float* scalars, int* status, const int* parent, int first, cudaStream_t s) {
  ++counter;
  pdl(k_inner_alpha, 1, 1, 0, s, scalars, status, parent, first);
}
void inner_first(int n, const float* b, const float* p, const float* q, float* x, float* t,
                 const float* scalars, const int* status, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_inner_first, blocks(n), kBlock, 0, s, n, b, p, q, x, t, scalars, status);
}
void inner_check(const float* scalars, int* status, cudaStream_t s) {
  ++counter;
  pdl(k_inner_check, 1, 1, 0, s, scalars, status);
}
void inner_beta(float* scalars, int* status, cudaStream_t s) {
  ++counter;
  pdl(k_inner_beta, 1, 1, 0, s, scalars, status);
}
void inner_step(int n, float* x, const float* p, const float* scalars, const int* status,
                cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_inner_step, blocks(n), kBlock, 0, s, n, x, p, scalars, status);
}

}  // namespace launch
}  // namespace kb2
