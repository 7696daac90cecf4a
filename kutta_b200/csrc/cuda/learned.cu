// Learned preconditioner stage (no reference counterpart): a small
// message-passing network over the matrix graph (the cell-face graph of the
// pressure operator), its backward pass and an Adam step, all in FP32.
//
// Graph features come from the matrix: edge weight w_ij = -a_ij / sqrt(a_ii
// a_jj), node scale s_i = 1 / sqrt(a_ii); with the faces' geometric
// coefficients bound as well, each edge weight is gated by a learned function
// of a geometry feature (k_gnn_gate below).
// Layer l maps H (n x Cin) to H' (n x 32):
//   M = W H  (M_i = sum_j w_ij H_j),   H'_i = relu(Ws H_i + Wn M_i + b);
// the output is z_i = s_i (wo . H3_i). Since w is symmetric, the backward of
// the aggregation is the aggregation itself.
//
// Activations are row-major n x C; a warp handles one row with lane = output
// channel (C <= 32), so a row of H is one 128-byte read.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.hpp"

namespace kb2 {
namespace {
using namespace dev;

constexpr int kHidden = 32;

#define ROWS(i, n) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// Warp-per-row loop (uniform per warp).
#define WARP_ROWS(i, n)                                                                \
  for (int i = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < (n); \
       i += static_cast<int>((gridDim.x * blockDim.x) >> 5))

// Also lift_ij = w_ij s_j, the input aggregation weight of the tensor-core
// forward (which aggregates t rather than s t).
__global__ void k_gnn_graph(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                            const int* __restrict__ diag, const float* __restrict__ vals,
                            float* __restrict__ edge, float* __restrict__ lift,
                            float* __restrict__ node_scale) {
  ROWS(i, n) {
    const float di = vals[diag[i]];
    node_scale[i] = di > 0.0f ? rsqrtf(di) : 0.0f;
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      const int c = cols[j];
      const float dc = vals[diag[c]];
      const float w = (c == i || di <= 0.0f || dc <= 0.0f) ? 0.0f : -vals[j] * rsqrtf(di * dc);
      edge[j] = w;
      lift[j] = dc > 0.0f ? w * rsqrtf(dc) : 0.0f;
    }
  }
}

// Geometry edge feature. With g_ij the face's geometric coefficient
// |A_f| / |c_N - c_P| and G_i = sum_j g_ij, the geometric analogue of w is
// gh_ij = g_ij / sqrt(G_i G_j); rho_ij = log(gh_ij / w_ij) (clamped to
// [-20, 20], 0 where either is not positive) compares the face's share of
// the operator with its share of the geometry: for a diffusion operator, the
// face's diffusivity relative to its cells'. It is symmetric in (i, j).
__global__ void k_gnn_geometry_sums(int n, const int* __restrict__ rows,
                                    const float* __restrict__ geometry, float* __restrict__ G) {
  ROWS(i, n) {
    float s = 0.0f;
    for (int j = rows[i]; j < rows[i + 1]; ++j) s += geometry[j];
    G[i] = s;
  }
}
__global__ void k_gnn_geometry_rho(int n, const int* __restrict__ rows,
                                   const int* __restrict__ cols, const float* __restrict__ geometry,
                                   const float* __restrict__ G, const float* __restrict__ edge_w,
                                   float* __restrict__ rho) {
  ROWS(i, n) {
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      const int c = cols[j];
      const float g = geometry[j], w = edge_w[j];
      const float gg = G[i] * G[c];
      float r = 0.0f;
      if (g > 0.0f && w > 0.0f && gg > 0.0f) r = fminf(fmaxf(logf(g * rsqrtf(gg) / w), -20.0f), 20.0f);
      rho[j] = r;
    }
  }
}
// E = w gamma, gamma = exp(theta_a tanh(theta_b rho)), for the edge and the
// input-lift weights; theta read from the parameters on the device.
__global__ void k_gnn_gate(int nnz, const float* __restrict__ edge_w,
                           const float* __restrict__ lift_w, const float* __restrict__ rho,
                           const float* __restrict__ theta, float* __restrict__ edge,
                           float* __restrict__ lift) {
  const float ta = theta[0], tb = theta[1];
  ROWS(j, nnz) {
    const float gamma = expf(ta * tanhf(tb * rho[j]));
    edge[j] = edge_w[j] * gamma;
    lift[j] = lift_w[j] * gamma;
  }
}
// dL/dE_ij (+)= sum_c dM[i][c] H[j][c], the aggregation M = E H's gradient
// with respect to each edge weight (one warp per row, lane = channel).
__global__ void k_gnn_edge_grad(int n, int C, const int* __restrict__ rows,
                                const int* __restrict__ cols, const float* __restrict__ dM,
                                const float* __restrict__ H, float* __restrict__ dedge,
                                int accumulate) {
  const int lane = threadIdx.x & 31;
  WARP_ROWS(i, n) {
    const float d = lane < C ? dM[static_cast<std::size_t>(i) * C + lane] : 0.0f;
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      float v = lane < C ? d * H[static_cast<std::size_t>(cols[j]) * C + lane] : 0.0f;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) dedge[j] = accumulate ? dedge[j] + v : v;
    }
  }
}
// dE/dtheta_a = E tanh(theta_b rho), dE/dtheta_b = E theta_a (1 - tanh^2) rho.
__global__ void k_gnn_gate_factors(int nnz, const float* __restrict__ edge,
                                   const float* __restrict__ rho, const float* __restrict__ theta,
                                   float* __restrict__ fa, float* __restrict__ fb) {
  const float ta = theta[0], tb = theta[1];
  ROWS(j, nnz) {
    const float th = tanhf(tb * rho[j]);
    fa[j] = edge[j] * th;
    fb[j] = edge[j] * ta * (1.0f - th * th) * rho[j];
  }
}
__global__ void k_gnn_store_gate_grad(const double* __restrict__ dots, float* __restrict__ grad) {
  if (blockIdx.x == 0 && threadIdx.x < 2) grad[threadIdx.x] = static_cast<float>(dots[threadIdx.x]);
}

// M = W H (C channels).
__global__ void k_gnn_aggregate(int n, int C, const int* __restrict__ rows,
                                const int* __restrict__ cols, const float* __restrict__ edge,
                                const float* __restrict__ H, float* __restrict__ M) {
  const int lane = threadIdx.x & 31;
  WARP_ROWS(i, n) {
    float acc = 0.0f;
    const int end = rows[i + 1];
    for (int j = rows[i]; j < end; ++j) {
      const float w = edge[j];
      if (lane < C && w != 0.0f) acc = fmaf(w, H[static_cast<std::size_t>(cols[j]) * C + lane], acc);
    }
    if (lane < C) M[static_cast<std::size_t>(i) * C + lane] = acc;
  }
}

// H'_i = relu(Ws H_i + Wn M_i + b): weights [Cout=32][Cin] held transposed in
// shared memory (lane = output channel reads consecutive words, no bank
// conflicts); the row's inputs are broadcast by shuffles.
__global__ void k_gnn_dense(int n, int Cin, const float* __restrict__ H,
                            const float* __restrict__ M, const float* __restrict__ Ws,
                            const float* __restrict__ Wn, const float* __restrict__ bias,
                            float* __restrict__ out) {
  __shared__ float ws[kHidden * kHidden], wn[kHidden * kHidden], bs[kHidden];
  for (int k = threadIdx.x; k < kHidden * Cin; k += blockDim.x) {
    const int c = k / Cin, j = k % Cin;  // Ws[c][j] -> ws[j][c]
    ws[j * kHidden + c] = Ws[k];
    wn[j * kHidden + c] = Wn[k];
  }
  if (threadIdx.x < kHidden) bs[threadIdx.x] = bias[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  WARP_ROWS(i, n) {
    const float h = lane < Cin ? H[static_cast<std::size_t>(i) * Cin + lane] : 0.0f;
    const float m = lane < Cin ? M[static_cast<std::size_t>(i) * Cin + lane] : 0.0f;
    float acc = bs[lane];
    for (int k = 0; k < Cin; ++k) {
      const float hk = __shfl_sync(0xffffffffu, h, k);
      const float mk = __shfl_sync(0xffffffffu, m, k);
      acc = fmaf(ws[k * kHidden + lane], hk, acc);
      acc = fmaf(wn[k * kHidden + lane], mk, acc);
    }
    out[static_cast<std::size_t>(i) * kHidden + lane] = fmaxf(acc, 0.0f);
  }
}

// RMS of the input features from their sum of squares (FP64, reduced on the
// device); 0 for a zero input.
__device__ __forceinline__ double input_rms(int n, const double* sum2) {
  const double m = sum2[0] / static_cast<double>(n);
  return m > 0.0 ? sqrt(m) : 0.0;
}

// z_i = rho s_i (wo . H_i), rho the input RMS: with the input normalised by rho
// the network is positively homogeneous, G(lambda r) = lambda G(r).
__global__ void k_gnn_output(int n, const float* __restrict__ H, const float* __restrict__ wo,
                             const float* __restrict__ node_scale, const double* __restrict__ sum2,
                             float* __restrict__ z, float beta) {
  const int lane = threadIdx.x & 31;
  const float w = wo[lane];
  const float rho = static_cast<float>(input_rms(n, sum2));
  WARP_ROWS(i, n) {
    float v = w * H[static_cast<std::size_t>(i) * kHidden + lane];
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if (lane == 0) z[i] = (beta != 0.0f ? beta * z[i] : 0.0f) + rho * node_scale[i] * v;
  }
}

// Input features before normalisation: H0_i = s_i r_i.
__global__ void k_gnn_input(int n, const float* __restrict__ r, const float* __restrict__ node_scale,
                            float* __restrict__ H0) {
  ROWS(i, n) H0[i] = node_scale[i] * r[i];
}

// H0 /= rho (the RMS of H0), so the network sees unit-RMS features whatever
// the residual's magnitude.
__global__ void k_gnn_normalize(int n, float* __restrict__ H0, const double* __restrict__ sum2) {
  const double rho = input_rms(n, sum2);
  const float inv = rho > 0.0 ? static_cast<float>(1.0 / rho) : 0.0f;
  ROWS(i, n) H0[i] *= inv;
}

// ---- training -------------------------------------------------------------
// Energy loss of a correction c for the residual t = A e:
//   L = 1 - (c.t)^2 / ((c.Ac)(t.e)),
// the fraction of the error's A-energy left after the best step along c
// (alpha = c.t / c.Ac). dots = {c.t, c.Ac, t.e} in FP64; q = A c.
//   dL/dc = -(2P / (Q E)) t + (2P^2 / (Q^2 E)) q    (P, Q, E = dots).
// Zero gradient and L = 1 when c.Ac or t.e is not positive.
__global__ void k_gnn_energy(int n, const float* __restrict__ t, const float* __restrict__ q,
                             const double* __restrict__ dots, float* __restrict__ dz,
                             float* __restrict__ loss) {
  const double P = dots[0], Q = dots[1], E = dots[2];
  const bool ok = Q > 0.0 && E > 0.0;
  const float gt = ok ? static_cast<float>(-2.0 * P / (Q * E)) : 0.0f;
  const float gq = ok ? static_cast<float>(2.0 * P * P / (Q * Q * E)) : 0.0f;
  if (blockIdx.x == 0 && threadIdx.x == 0) *loss = ok ? static_cast<float>(1.0 - P * P / (Q * E)) : 1.0f;
  ROWS(i, n) dz[i] = fmaf(gt, t[i], gq * q[i]);
}

// Output backward: dH_i = dz_i rho s_i wo, dwo += sum_i dz_i rho s_i H_i.
__global__ void k_gnn_output_back(int n, const float* __restrict__ H, const float* __restrict__ wo,
                                  const float* __restrict__ node_scale,
                                  const double* __restrict__ sum2, const float* __restrict__ dz,
                                  float* __restrict__ dH, float* __restrict__ dwo) {
  const int lane = threadIdx.x & 31;
  const float w = wo[lane];
  const float rho = static_cast<float>(input_rms(n, sum2));
  float g = 0.0f;
  WARP_ROWS(i, n) {
    const float t = dz[i] * rho * node_scale[i];
    const std::size_t k = static_cast<std::size_t>(i) * kHidden + lane;
    dH[k] = t * w;
    g = fmaf(t, H[k], g);
  }
  atomicAdd(dwo + lane, g);
}

// Dense layer backward. G = dOut * (out > 0); dH_i = Ws^T G_i, dM_i = Wn^T G_i;
// dWs += G_i H_i^T, dWn += G_i M_i^T, db += G_i (per-warp sums, then atomics).
__global__ void k_gnn_dense_back(int n, int Cin, const float* __restrict__ H,
                                 const float* __restrict__ M, const float* __restrict__ out,
                                 const float* __restrict__ dOut, const float* __restrict__ Ws,
                                 const float* __restrict__ Wn, float* __restrict__ dH,
                                 float* __restrict__ dM, float* __restrict__ dWs,
                                 float* __restrict__ dWn, float* __restrict__ db) {
  __shared__ float ws[kHidden * kHidden], wn[kHidden * kHidden];
  __shared__ float gws[kHidden * kHidden], gwn[kHidden * kHidden], gb[kHidden];
  for (int k = threadIdx.x; k < kHidden * Cin; k += blockDim.x) {
    ws[k] = Ws[k];
    wn[k] = Wn[k];
    gws[k] = 0.0f;
    gwn[k] = 0.0f;
  }
  if (threadIdx.x < kHidden) gb[threadIdx.x] = 0.0f;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  // Per-lane accumulators for this lane's output channel c = lane.
  float aws[kHidden], awn[kHidden];
#pragma unroll
  for (int k = 0; k < kHidden; ++k) aws[k] = awn[k] = 0.0f;
  float ab = 0.0f;
  WARP_ROWS(i, n) {
    const std::size_t row = static_cast<std::size_t>(i);
    const float o = out[row * kHidden + lane];
    const float g = o > 0.0f ? dOut[row * kHidden + lane] : 0.0f;  // channel c = lane
    const float h = lane < Cin ? H[row * Cin + lane] : 0.0f;
    const float m = lane < Cin ? M[row * Cin + lane] : 0.0f;
    ab += g;
    // dH_i[k] = sum_c Ws[c][k] g_c; lane k gathers over c by shuffles.
    float dh = 0.0f, dm = 0.0f;
#pragma unroll
    for (int c = 0; c < kHidden; ++c) {
      const float gc = __shfl_sync(0xffffffffu, g, c);
      if (lane < Cin) {
        dh = fmaf(ws[c * Cin + lane], gc, dh);
        dm = fmaf(wn[c * Cin + lane], gc, dm);
      }
    }
    if (lane < Cin) {
      dH[row * Cin + lane] = dh;
      dM[row * Cin + lane] = dm;
    }
#pragma unroll
    for (int k = 0; k < kHidden; ++k) {
      if (k < Cin) {
        aws[k] = fmaf(g, __shfl_sync(0xffffffffu, h, k), aws[k]);
        awn[k] = fmaf(g, __shfl_sync(0xffffffffu, m, k), awn[k]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kHidden; ++k)
    if (k < Cin) {
      atomicAdd(&gws[lane * Cin + k], aws[k]);
      atomicAdd(&gwn[lane * Cin + k], awn[k]);
    }
  atomicAdd(&gb[lane], ab);
  __syncthreads();
  for (int k = threadIdx.x; k < kHidden * Cin; k += blockDim.x) {
    atomicAdd(dWs + k, gws[k]);
    atomicAdd(dWn + k, gwn[k]);
  }
  if (threadIdx.x < kHidden) atomicAdd(db + threadIdx.x, gb[threadIdx.x]);
}

// out = a + b (elementwise).
__global__ void k_gnn_add(std::size_t count, const float* __restrict__ a,
                          const float* __restrict__ b, float* __restrict__ out) {
  for (std::size_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count;
       k += static_cast<std::size_t>(gridDim.x) * blockDim.x)
    out[k] = a[k] + b[k];
}

// z += alpha c with alpha = max(0, dots[0] / dots[1]) (dots = c.t, c.A c in
// FP64): the step along c that minimises the A-norm of the error, never
// negative.
__global__ void k_gnn_step(int n, float* __restrict__ z, const float* __restrict__ c,
                           const double* __restrict__ dots) {
  const double den = dots[1];
  const float alpha = den > 0.0 && dots[0] > 0.0 ? static_cast<float>(dots[0] / den) : 0.0f;
  // No step leaves z untouched, also where c is not finite (0 * NaN is NaN).
  if (!(alpha > 0.0f) || !isfinite(alpha)) return;
  ROWS(i, n) z[i] = fmaf(alpha, c[i], z[i]);
}

// The same step on an FP64 vector (the warm start of the mixed solve).
__global__ void k_gnn_step64(int n, double* __restrict__ x, const float* __restrict__ c,
                             const double* __restrict__ dots) {
  const double den = dots[1];
  const double alpha = den > 0.0 && dots[0] > 0.0 ? dots[0] / den : 0.0;
  if (!(alpha > 0.0) || !isfinite(alpha)) return;
  ROWS(i, n) x[i] += alpha * static_cast<double>(c[i]);
}

// Adam with bias correction (step t >= 1).
__global__ void k_gnn_adam(int count, float* __restrict__ w, const float* __restrict__ g,
                           float* __restrict__ m, float* __restrict__ v, float lr, float beta1,
                           float beta2, float eps, float correction1, float correction2) {
  ROWS(k, count) {
    const float gk = g[k];
    m[k] = beta1 * m[k] + (1.0f - beta1) * gk;
    v[k] = beta2 * v[k] + (1.0f - beta2) * gk * gk;
    w[k] -= lr * (m[k] / correction1) / (sqrtf(v[k] / correction2) + eps);
  }
}

int warp_grid(int n) {
  const long long blocks = (static_cast<long long>(n) * 32 + kBlock - 1) / kBlock;
  return static_cast<int>(std::max(1LL, std::min(blocks, static_cast<long long>(kMaxBlocks))));
}

}  // namespace

namespace launch {

void gnn_graph(int n, const int* rows, const int* cols, const int* diag, const float* vals,
               float* edge, float* lift, float* node_scale, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_graph<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, diag, vals, edge, lift, node_scale);
}
void gnn_geometry(int n, const int* rows, const int* cols, const float* geometry,
                  const float* edge_w, float* G, float* rho, cudaStream_t s) {
  if (n <= 0) return;
  counter += 2;
  k_gnn_geometry_sums<<<grid_for(n), kBlock, 0, s>>>(n, rows, geometry, G);
  k_gnn_geometry_rho<<<grid_for(n), kBlock, 0, s>>>(n, rows, cols, geometry, G, edge_w, rho);
}
void gnn_gate(int nnz, const float* edge_w, const float* lift_w, const float* rho,
              const float* theta, float* edge, float* lift, cudaStream_t s) {
  if (nnz <= 0) return;
  ++counter;
  k_gnn_gate<<<grid_for(nnz), kBlock, 0, s>>>(nnz, edge_w, lift_w, rho, theta, edge, lift);
}
void gnn_edge_grad(int n, int C, const int* rows, const int* cols, const float* dM,
                   const float* H, float* dedge, bool accumulate, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_edge_grad<<<warp_grid(n), kBlock, 0, s>>>(n, C, rows, cols, dM, H, dedge,
                                                  accumulate ? 1 : 0);
}
void gnn_gate_factors(int nnz, const float* edge, const float* rho, const float* theta,
                      float* fa, float* fb, cudaStream_t s) {
  if (nnz <= 0) return;
  ++counter;
  k_gnn_gate_factors<<<grid_for(nnz), kBlock, 0, s>>>(nnz, edge, rho, theta, fa, fb);
}
void gnn_store_gate_grad(const double* dots, float* grad, cudaStream_t s) {
  ++counter;
  k_gnn_store_gate_grad<<<1, 32, 0, s>>>(dots, grad);
}
void gnn_input(int n, const float* r, const float* node_scale, float* H0, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_input<<<grid_for(n), kBlock, 0, s>>>(n, r, node_scale, H0);
}
void gnn_normalize(int n, float* H0, const double* sum2, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_normalize<<<grid_for(n), kBlock, 0, s>>>(n, H0, sum2);
}
void gnn_aggregate(int n, int C, const int* rows, const int* cols, const float* edge,
                   const float* H, float* M, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_aggregate<<<warp_grid(n), kBlock, 0, s>>>(n, C, rows, cols, edge, H, M);
}
void gnn_dense(int n, int Cin, const float* H, const float* M, const float* Ws, const float* Wn,
               const float* bias, float* out, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_dense<<<warp_grid(n), kBlock, 0, s>>>(n, Cin, H, M, Ws, Wn, bias, out);
}
void gnn_output(int n, const float* H, const float* wo, const float* node_scale,
                const double* sum2, float* z, float beta, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_output<<<warp_grid(n), kBlock, 0, s>>>(n, H, wo, node_scale, sum2, z, beta);
}
void gnn_energy(int n, const float* t, const float* q, const double* dots, float* dz, float* loss,
                cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_energy<<<grid_for(n), kBlock, 0, s>>>(n, t, q, dots, dz, loss);
}
void gnn_output_back(int n, const float* H, const float* wo, const float* node_scale,
                     const double* sum2, const float* dz, float* dH, float* dwo, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_output_back<<<warp_grid(n), kBlock, 0, s>>>(n, H, wo, node_scale, sum2, dz, dH, dwo);
}
void gnn_dense_back(int n, int Cin, const float* H, const float* M, const float* out,
                    const float* dOut, const float* Ws, const float* Wn, float* dH, float* dM,
                    float* dWs, float* dWn, float* db, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_dense_back<<<warp_grid(n), kBlock, 0, s>>>(n, Cin, H, M, out, dOut, Ws, Wn, dH, dM, dWs,
                                                   dWn, db);
}
void gnn_add(std::size_t count, const float* a, const float* b, float* out, cudaStream_t s) {
  if (count == 0) return;
  ++counter;
  const int blocks = static_cast<int>(std::min<std::size_t>((count + kBlock - 1) / kBlock, kMaxBlocks));
  k_gnn_add<<<blocks, kBlock, 0, s>>>(count, a, b, out);
}
void gnn_step(int n, float* z, const float* c, const double* dots, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_step<<<grid_for(n), kBlock, 0, s>>>(n, z, c, dots);
}
void gnn_step64(int n, double* x, const float* c, const double* dots, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  k_gnn_step64<<<grid_for(n), kBlock, 0, s>>>(n, x, c, dots);
}
void gnn_adam(int count, float* w, const float* g, float* m, float* v, float lr, float beta1,
              float beta2, float eps, float correction1, float correction2, cudaStream_t s) {
  if (count <= 0) return;
  ++counter;
  k_gnn_adam<<<grid_for(count), kBlock, 0, s>>>(count, w, g, m, v, lr, beta1, beta2, eps,
                                                correction1, correction2);
}

}  // namespace launch
}  // namespace kb2
