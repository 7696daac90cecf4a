// The finite-volume steps on either side of the pressure solve
// (src/kutta/kernels/fv_flow.kern.h:164-201), compiled without FMA
// contraction so every value rounds as the reference's CPU kernels do:
//
//   fv_pressure_assemble  cell i's CSR row of the pressure-correction matrix
//                         and its right-hand side from the face coefficients
//                         and mass fluxes (:164-183); with `fused`, the row's
//                         inverse L1 diagonal (the refresh's first step,
//                         linalg.kern.h:52-70) and its validity flag follow in
//                         the same pass, from the values the thread just wrote;
//   fv_correct_flux       face flux correction (:185-190);
//   fv_correct_velocity   cell velocity and pressure correction (:192-201).
//
// Row i's values are written only by the thread of row i (the entries of its
// faces and its diagonal are all in row i), so rows are independent.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.hpp"

namespace kb2 {
namespace {
using namespace dev;

#define ROWS(i, n) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

__device__ __forceinline__ float assemble_row(int i, const int* __restrict__ offsets,
                                              const int* __restrict__ faces,
                                              const float* __restrict__ sign,
                                              const int* __restrict__ adjacent,
                                              const int* __restrict__ entry,
                                              const int* __restrict__ rows,
                                              const int* __restrict__ diag,
                                              const float* __restrict__ coefficient,
                                              const float* __restrict__ flux,
                                              float* __restrict__ values, int reference) {
  UpperSum ap{0.0f, 0.0f};
  float b = 0.0f;
  for (int j = offsets[i]; j < offsets[i + 1]; ++j)
    if (adjacent[j] >= 0) values[entry[j]] = 0.0f;
  for (int j = offsets[i]; j < offsets[i + 1]; ++j) {
    const int f = faces[j], nb = adjacent[j];
    const float d = coefficient[f];
    b -= sign[j] * flux[f];
    // Boundary faces and the eliminated reference cell anchor the diagonal.
    if (nb < 0 || nb == reference) ap = upper_add(ap, d);
    if (nb >= 0 && nb != reference && i != reference) values[entry[j]] -= d;
  }
  // The stored off-diagonals once each (faces may share an entry), upward
  // rounded: the row stays weakly diagonally dominant.
  for (int j = rows[i]; j < rows[i + 1]; ++j)
    if (j != diag[i]) ap = upper_add(ap, -values[j]);
  values[diag[i]] = i == reference ? 1.0f : upper_value(ap);
  return i == reference ? 0.0f : b;
}

template <bool kFused>
__global__ void k_fv_pressure_assemble(int n, const int* __restrict__ offsets,
                                       const int* __restrict__ faces,
                                       const float* __restrict__ sign,
                                       const int* __restrict__ adjacent,
                                       const int* __restrict__ entry, const int* __restrict__ rows,
                                       const int* __restrict__ diag,
                                       const float* __restrict__ coefficient,
                                       const float* __restrict__ flux, float* __restrict__ values,
                                       float* __restrict__ rhs, int reference,
                                       float* __restrict__ inverse, DeviceReducer red,
                                       double* check, int slot) {
  double worst = 0;
  ROWS(i, n) {
    rhs[i] = assemble_row(i, offsets, faces, sign, adjacent, entry, rows, diag, coefficient, flux,
                          values, reference);
    if constexpr (kFused) worst = nan_max(worst, diagonal_row(i, rows, diag, values, inverse, 1));
  }
  if constexpr (kFused) {
    __shared__ double shared[32];
    worst = block_max(worst, shared);
    const Reducer r{red.partials, red.ticket};
    if (!publish(r, worst, 0, false)) return;
    const double total = gather_max(r, shared);
    if (threadIdx.x == 0) {
      check[slot] = total;
      *r.ticket = 0;
    }
  }
}

__global__ void k_fv_correct_flux(int n, const int* __restrict__ owner,
                                  const int* __restrict__ neighbour,
                                  const float* __restrict__ correction,
                                  const float* __restrict__ coefficient, float* __restrict__ flux,
                                  int internal) {
  ROWS(i, n) {
    const float pc = correction[owner[i]];
    const float pn = i < internal ? correction[neighbour[i]] : 0.0f;
    flux[i] += coefficient[i] * (pc - pn);
  }
}

__global__ void k_fv_correct_velocity(int n, const float* __restrict__ volume,
                                      const float* __restrict__ inverse,
                                      const float* __restrict__ diagonal,
                                      const float* __restrict__ gx, const float* __restrict__ gy,
                                      const float* __restrict__ gz,
                                      const float* __restrict__ correction, float* __restrict__ u,
                                      float* __restrict__ v, float* __restrict__ w,
                                      float* __restrict__ p, float alpha) {
  ROWS(i, n) {
    const float d = volume[i] * inverse[i];
    u[i] -= d * gx[i];
    v[i] -= d * gy[i];
    w[i] -= d * gz[i];
    // The pressure step is bounded by the local ratio of the physical to the
    // SIMPLEC correction coefficient.
    const float pressure_alpha = fminf(alpha, 0.7f * diagonal[i] * inverse[i]);
    p[i] += pressure_alpha * correction[i];
  }
}

}  // namespace

namespace launch {

void fv_pressure_assemble(int n, const int* offsets, const int* faces, const float* sign,
                          const int* adjacent, const int* entry, const int* rows, const int* diag,
                          const float* coefficient, const float* flux, float* values, float* rhs,
                          int reference, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_fv_pressure_assemble<false><<<grid_for(n), kBlock, 0, s>>>(
      n, offsets, faces, sign, adjacent, entry, rows, diag, coefficient, flux, values, rhs,
      reference, nullptr, DeviceReducer{nullptr, nullptr}, nullptr, 0);
}

void fv_pressure_assemble_l1(int n, const int* offsets, const int* faces, const float* sign,
                             const int* adjacent, const int* entry, const int* rows,
                             const int* diag, const float* coefficient, const float* flux,
                             float* values, float* rhs, int reference, float* inverse,
                             DeviceReducer red, double* check, int slot, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_fv_pressure_assemble<true><<<grid_for(n), kBlock, 0, s>>>(
      n, offsets, faces, sign, adjacent, entry, rows, diag, coefficient, flux, values, rhs,
      reference, inverse, red, check, slot);
}

void fv_correct_flux(int n, const int* owner, const int* neighbour, const float* correction,
                     const float* coefficient, float* flux, int internal, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_fv_correct_flux<<<grid_for(n), kBlock, 0, s>>>(n, owner, neighbour, correction, coefficient,
                                                   flux, internal);
}

void fv_correct_velocity(int n, const float* volume, const float* inverse, const float* diagonal,
                         const float* gx, const float* gy, const float* gz,
                         const float* correction, float* u, float* v, float* w, float* p,
                         float alpha, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_fv_correct_velocity<<<grid_for(n), kBlock, 0, s>>>(n, volume, inverse, diagonal, gx, gy, gz,
                                                       correction, u, v, w, p, alpha);
}

}  // namespace launch
}  // namespace kb2
