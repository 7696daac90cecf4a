// Coupled (4x4-block) pressure-velocity solve kernels for sm_100a (compiled
// with --fmad=false, IEEE division): the block Jacobian of momentum and
// continuity in cell unknowns (u, v, w, p~), its damped block-Jacobi smoother,
// the piecewise-constant aggregation Galerkin operators and the transfers of
// src/kutta/kernels/fv_coupled.kern.h. Every per-row and per-coarse-row result
// rounds exactly as the reference kernel's: the same operations in the same
// order, no contraction.
//
// Layout on the device (own design; the reference keeps 4n planes, a 27n
// packed cell array and five incidence planes):
// - block vectors are float4 per cell (u, v, w, p~): one 16-byte load per
//   cell and per neighbour in the row kernels instead of four gathers;
// - setup-time cell data keeps the reference's 27 planes of n floats
//   (slot k of cell i at k n + i: du dv dw cd | Gx Gy Gz | Hx Hy Hz | Q (9) | cs
//   | 7 free), because the assembly kernels fill them slot by slot and the
//   fine Galerkin reads them;
// - the fine operator used every iteration is repacked once per solve into
//   per-cell records, 16-byte aligned: (du, dv, dw, cd), (wc Gx, wc Gy, wc Gz,
//   wc Hx), (wc Hy, wc Hz), the block inverse (iu, iv, iw, schur) and
//   (Hx iu, Hy iv, Hz iw, 0) with Hx = wc Hx, and ELL slots in slot-major
//   order for the internal faces of each cell in cell-face order: (a, gx, gy,
//   gz), h and (neighbour, face) per slot, plus one (sx, sy, sz, rc) record
//   per face. A warp's slot loads are then contiguous 512-byte lines;
// - coarse levels keep the reference's CSR with a, c, G and H per entry and
//   11 planes of n per row (du dv dw cs iu iv iw hx iu hy iv hz iw schur).
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "coupled_kernels.hpp"

namespace kb2 {
namespace {

using dev::grid_for;
using dev::kBlock;
using dev::pdl;
using dev::pdl_entry;

// Neumaier-compensated sum (fv_coupled.kern.h:77-84).
struct Csum {
  float s, e;
};
__device__ __forceinline__ Csum csum_add(Csum a, float b) {
  const float t = a.s + b;
  const float e = fabsf(a.s) >= fabsf(b) ? (a.s - t) + b : (b - t) + a.s;
  return Csum{t, a.e + e};
}
__device__ __forceinline__ float csum_value(Csum a) { return a.s + a.e; }

// Cell c's share of the face velocity it shares with cell i
// (fv_coupled.kern.h:86-91).
__device__ __forceinline__ float share_of(const float* __restrict__ weight, int i, int c) {
  return weight[c] / fmaxf(weight[i] + weight[c], 1.0e-30f);
}

// The arrow block's inverse (fv_coupled.kern.h:51-60), returned as the five
// factors the block solve uses and the Schur denominator.
struct BlockInverse {
  float iu, iv, iw, hu, hv, hw, schur;
};
__device__ __forceinline__ BlockInverse block_prepare(float du, float dv, float dw, float ex,
                                                      float ey, float ez, float hx, float hy,
                                                      float hz, float c) {
  BlockInverse b;
  b.iu = 1.0f / du;
  b.iv = 1.0f / dv;
  b.iw = 1.0f / dw;
  b.schur = fmaxf(c - (hx * ex * b.iu + hy * ey * b.iv + hz * ez * b.iw), 0.5f * c);
  b.hu = hx * b.iu;
  b.hv = hy * b.iv;
  b.hw = hz * b.iw;
  return b;
}
// The block solve (fv_coupled.kern.h:61-66).
__device__ __forceinline__ float4 block_solve(float4 r, float ex, float ey, float ez, float iu,
                                              float iv, float iw, float hu, float hv, float hw,
                                              float schur) {
  const float p = (r.w - hu * r.x - hv * r.y - hw * r.z) / schur;
  return make_float4(iu * (r.x - ex * p), iv * (r.y - ey * p), iw * (r.z - ez * p), p);
}
// next = base + omega d, base = x, or +0 on a zero start (the reference adds
// the zero explicitly, which turns a -0 step into +0).
__device__ __forceinline__ float4 damped(float4 base, float4 d, float omega) {
  return make_float4(base.x + omega * d.x, base.y + omega * d.y, base.z + omega * d.z,
                     base.w + omega * d.w);
}

// ---- Jacobian assembly, once per solve --------------------------------------

// fv_coupled.kern.h:183-189 (coupled_copy_diagonal).
__global__ void k_cpl_copy_diagonal(int n, const int* __restrict__ rows,
                                    const int* __restrict__ diag, const float* __restrict__ values,
                                    const float* __restrict__ physical, float* __restrict__ plane,
                                    float inverse_courant) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int d = diag[i];
    float off = 0.0f;
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      if (j != d) off += fabsf(values[j]);
    const float p = physical[i];
    const float floored = fmaxf(p, off);
    plane[i] = values[d] + (floored - p) + inverse_courant * floored;
  }
}

// fv_coupled.kern.h:112-126 (coupled_face_coefficient), one thread per face.
__global__ void k_cpl_face_coefficient(int nf, int internal, const int* __restrict__ owner,
                                       const int* __restrict__ neighbour,
                                       const int* __restrict__ kind,
                                       const float* __restrict__ diffusion,
                                       const float* __restrict__ volume,
                                       const float* __restrict__ diagonal,
                                       float* __restrict__ coefficient, float scale) {
  pdl_entry();
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    const int c = owner[f];
    float rc = volume[c] / fmaxf(diagonal[c], 1.0e-20f);
    if (f < internal) {
      const int m = neighbour[f];
      rc = 0.5f * (rc + volume[m] / fmaxf(diagonal[m], 1.0e-20f));
    } else {
      const int k = kind[f - internal];
      if (k != 2 && k != 4) {
        coefficient[f] = 0.0f;
        continue;
      }
    }
    coefficient[f] = scale * rc * diffusion[f];
  }
}

// fv_coupled.kern.h:93-108 (coupled_velocity_block): H_ii into planes 7-9.
__global__ void __launch_bounds__(kBlock, 8) k_cpl_velocity_block(int n, int internal, const int* __restrict__ offsets,
                                     const int* __restrict__ faces,
                                     const float* __restrict__ sign,
                                     const int* __restrict__ adjacent,
                                     const int* __restrict__ kind, const float* __restrict__ sx,
                                     const float* __restrict__ sy, const float* __restrict__ sz,
                                     const float* __restrict__ weight, float* __restrict__ cell) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float hx = 0.0f, hy = 0.0f, hz = 0.0f;
    for (int j = offsets[i]; j < offsets[i + 1]; ++j) {
      const int f = faces[j], c = adjacent[j];
      float share = 0.0f;
      if (c >= 0) {
        share = 1.0f - share_of(weight, i, c);
      } else {
        const int k = kind[f - internal];
        if (k == 2 || k == 4) share = 1.0f;
      }
      const float s = share * sign[j];
      hx += s * sx[f];
      hy += s * sy[f];
      hz += s * sz[f];
    }
    cell[7 * static_cast<std::size_t>(n) + i] = hx;
    cell[8 * static_cast<std::size_t>(n) + i] = hy;
    cell[9 * static_cast<std::size_t>(n) + i] = hz;
  }
}

// fv_coupled.kern.h:131-150 (coupled_rhs): the pressure diagonal into plane
// 3 and the block right-hand side.
__global__ void k_cpl_rhs(int n, const int* __restrict__ offsets, const int* __restrict__ faces,
                          const float* __restrict__ sign, const float* __restrict__ coefficient,
                          const float* __restrict__ mass, const float* __restrict__ net,
                          const float* __restrict__ ru, const float* __restrict__ rv,
                          const float* __restrict__ rw, float* __restrict__ cell,
                          float4* __restrict__ b, int reference, float continuity_scale) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Csum c{0.0f, 0.0f};
    float imbalance = 0.0f;
    for (int j = offsets[i]; j < offsets[i + 1]; ++j) {
      const int f = faces[j];
      c = csum_add(c, coefficient[f]);
      imbalance += sign[j] * mass[f];
    }
    if (net) imbalance = net[i];
    const float value = csum_value(c);
    cell[3 * static_cast<std::size_t>(n) + i] = i == reference ? 2.0f * value : value;
    b[i] = make_float4(ru[i], rv[i], rw[i], -continuity_scale * imbalance);
  }
}

struct FineGeometry {
  const int* offsets;
  const int* faces;
  const float* sign;
  const int* adjacent;
  const float *sx, *sy, *sz;
  const float *dx, *dy, *dz;
};

// fv_coupled.kern.h:191-208 (coupled_fine_gsum): |G| row sums, 3n planes.
__global__ void __launch_bounds__(kBlock, 8) k_cpl_fine_gsum(int n, FineGeometry m, const float* __restrict__ cell,
                                float* __restrict__ r, float wc) {
  pdl_entry();
  const std::size_t N = n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float q00 = wc * cell[10 * N + i], q01 = wc * cell[11 * N + i], q02 = wc * cell[12 * N + i];
    const float q10 = wc * cell[13 * N + i], q11 = wc * cell[14 * N + i], q12 = wc * cell[15 * N + i];
    const float q20 = wc * cell[16 * N + i], q21 = wc * cell[17 * N + i], q22 = wc * cell[18 * N + i];
    const float half_wc = 0.5f * wc;
    float gx = fabsf(wc * cell[4 * N + i]), gy = fabsf(wc * cell[5 * N + i]),
          gz = fabsf(wc * cell[6 * N + i]);
    for (int j = m.offsets[i]; j < m.offsets[i + 1]; ++j) {
      if (m.adjacent[j] < 0) continue;
      const int f = m.faces[j];
      const float s = m.sign[j];
      gx += fabsf(half_wc * s * m.sx[f] + q00 * m.dx[j] + q01 * m.dy[j] + q02 * m.dz[j]);
      gy += fabsf(half_wc * s * m.sy[f] + q10 * m.dx[j] + q11 * m.dy[j] + q12 * m.dz[j]);
      gz += fabsf(half_wc * s * m.sz[f] + q20 * m.dx[j] + q21 * m.dy[j] + q22 * m.dz[j]);
    }
    r[i] = gx;
    r[N + i] = gy;
    r[2 * N + i] = gz;
  }
}

// fv_coupled.kern.h:210-223 (coupled_fine_schur): cs into plane 19.
__global__ void k_cpl_fine_schur(int n, FineGeometry m, const float* __restrict__ weight,
                                 const float* __restrict__ r, float* __restrict__ cell, float wc) {
  pdl_entry();
  const std::size_t N = n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float sum = 0.0f;
    for (int j = m.offsets[i]; j < m.offsets[i + 1]; ++j) {
      const int c = m.adjacent[j];
      if (c < 0) continue;
      const int f = m.faces[j];
      sum += wc * share_of(weight, i, c) *
             (fabsf(m.sx[f]) * r[c] / cell[c] + fabsf(m.sy[f]) * r[N + c] / cell[N + c] +
              fabsf(m.sz[f]) * r[2 * N + c] / cell[2 * N + c]);
    }
    cell[19 * N + i] = sum;
  }
}

// Per face: (sx, sy, sz, Rhie-Chow coefficient), the face half of the fine
// row's continuity term.
__global__ void k_cpl_face_records(int nf, const float* __restrict__ sx,
                                   const float* __restrict__ sy, const float* __restrict__ sz,
                                   const float* __restrict__ coefficient,
                                   float4* __restrict__ face) {
  pdl_entry();
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x)
    face[f] = make_float4(sx[f], sy[f], sz[f], coefficient[f]);
}

// fv_coupled.kern.h:229-256 (coupled_fine_coefficients): the block inverse
// and the five directed-edge coefficients, written as the per-cell records
// and the ELL slots of the fine operator.
__global__ void k_cpl_fine_pack(int n, int width, FineGeometry m, const float* __restrict__ mu,
                                const float* __restrict__ diffusion,
                                const float* __restrict__ mass, const float* __restrict__ weight,
                                const float* __restrict__ cell, CoupledFine op, float wc) {
  pdl_entry();
  const std::size_t N = n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float du = cell[i], dv = cell[N + i], dw = cell[2 * N + i], cd = cell[3 * N + i];
    const float ex = wc * cell[4 * N + i], ey = wc * cell[5 * N + i], ez = wc * cell[6 * N + i];
    const float hx = wc * cell[7 * N + i], hy = wc * cell[8 * N + i], hz = wc * cell[9 * N + i];
    const BlockInverse inv = block_prepare(du, dv, dw, ex, ey, ez, hx, hy, hz, cd + cell[19 * N + i]);
    op.diag[i] = make_float4(du, dv, dw, cd);
    op.coupling[i] = make_float4(ex, ey, ez, hx);
    op.coupling_yz[i] = make_float2(hy, hz);
    op.inverse[i] = make_float4(inv.iu, inv.iv, inv.iw, inv.schur);
    op.inverse_h[i] = make_float4(inv.hu, inv.hv, inv.hw, 0.0f);
    const float q00 = wc * cell[10 * N + i], q01 = wc * cell[11 * N + i], q02 = wc * cell[12 * N + i];
    const float q10 = wc * cell[13 * N + i], q11 = wc * cell[14 * N + i], q12 = wc * cell[15 * N + i];
    const float q20 = wc * cell[16 * N + i], q21 = wc * cell[17 * N + i], q22 = wc * cell[18 * N + i];
    const float half_wc = 0.5f * wc;
    int slot = 0;
    for (int j = m.offsets[i]; j < m.offsets[i + 1] && slot < width; ++j) {
      const int c = m.adjacent[j];
      if (c < 0) continue;
      const int f = m.faces[j];
      const float s = m.sign[j];
      const float a = -mu[f] * diffusion[f] + fminf(s * mass[f], 0.0f);
      const float bx = half_wc * s * m.sx[f], by = half_wc * s * m.sy[f], bz = half_wc * s * m.sz[f];
      const float gx = bx + q00 * m.dx[j] + q01 * m.dy[j] + q02 * m.dz[j];
      const float gy = by + q10 * m.dx[j] + q11 * m.dy[j] + q12 * m.dz[j];
      const float gz = bz + q20 * m.dx[j] + q21 * m.dy[j] + q22 * m.dz[j];
      const float h = wc * s * share_of(weight, i, c);
      const std::size_t k = slot * N + i;
      op.edge[k] = make_float4(a, gx, gy, gz);
      op.edge_h[k] = h;
      op.link[k] = make_int2(c, f);
      ++slot;
    }
    for (; slot < width; ++slot) op.link[slot * N + i] = make_int2(-1, 0);
  }
}

// The fine row kernels are bounded to 32 registers (8 resident blocks of 256
// per SM), so the fixed 1,184-block grid runs in one wave: at 40 registers
// the sweep took 142.5 us at 128^3, bounded 122.7 us (0.92 of the measured
// copy bandwidth). The coarse-level and Galerkin kernels are not bounded: the
// spills cost them more than the second wave.
//
// (J x)_i of the fine level (fv_coupled.kern.h:258-278, coupled_fine_row).
__device__ __forceinline__ float4 fine_row(int i, int n, int width, const CoupledFine& op,
                                           const float4* __restrict__ x) {
  const float4 xi = x[i];
  const float4 d = op.diag[i], e = op.coupling[i];
  const float2 h = op.coupling_yz[i];
  float yu = d.x * xi.x + e.x * xi.w;
  float yv = d.y * xi.y + e.y * xi.w;
  float yw = d.z * xi.z + e.z * xi.w;
  float yp = d.w * xi.w + e.w * xi.x + h.x * xi.y + h.y * xi.z;
  const std::size_t N = n;
  for (int s = 0; s < width; ++s) {
    const int2 l = op.link[s * N + i];
    if (l.x < 0) break;
    const float4 g = op.edge[s * N + i];
    const float hs = op.edge_h[s * N + i];
    const float4 sf = op.face[l.y];
    const float4 xc = x[l.x];
    yu += g.x * xc.x + g.y * xc.w;
    yv += g.x * xc.y + g.z * xc.w;
    yw += g.x * xc.z + g.w * xc.w;
    yp += hs * (sf.x * xc.x + sf.y * xc.y + sf.z * xc.z) - sf.w * xc.w;
  }
  return make_float4(yu, yv, yw, yp);
}

__global__ void __launch_bounds__(kBlock, 8) k_cpl_fine_spmv(int n, int width, CoupledFine op,
                                                          const float4* __restrict__ x,
                                                          float4* __restrict__ y) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = fine_row(i, n, width, op, x);
}

__global__ void __launch_bounds__(kBlock, 8) k_cpl_fine_residual(int n, int width, CoupledFine op,
                                                              const float4* __restrict__ x,
                                                              const float4* __restrict__ b,
                                                              float4* __restrict__ r) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 y = fine_row(i, n, width, op, x);
    const float4 bi = b[i];
    r[i] = make_float4(bi.x - y.x, bi.y - y.y, bi.z - y.z, bi.w - y.w);
  }
}

// Damped block Jacobi (fv_coupled.kern.h:294-309, coupled_fine_smooth);
// first: x is zero and is not read.
__global__ void __launch_bounds__(kBlock, 8) k_cpl_fine_smooth(int n, int width, CoupledFine op,
                                                            const float4* __restrict__ x,
                                                            const float4* __restrict__ b,
                                                            float4* __restrict__ next, float omega,
                                                            int first) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 r = b[i];
    float4 base = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (!first) {
      const float4 y = fine_row(i, n, width, op, x);
      r = make_float4(r.x - y.x, r.y - y.y, r.z - y.z, r.w - y.w);
      base = x[i];
    }
    const float4 e = op.coupling[i], iv = op.inverse[i], ih = op.inverse_h[i];
    const float4 d = block_solve(r, e.x, e.y, e.z, iv.x, iv.y, iv.z, ih.x, ih.y, ih.z, iv.w);
    next[i] = damped(base, d, omega);
  }
}

// ---- coarse levels ------------------------------------------------------------

// (J x)_i of a coarse level (fv_coupled.kern.h:376-392, coupled_coarse_row).
// The entries are summed one by one in CSR order, as there. Each entry's
// product terms are formed whether or not it is the diagonal (only the sum
// skips the diagonal), so the loads of four entries at a time are issued
// together: a long row waits for two memory latencies per four entries
// instead of one or two per entry.
struct EntryTerms {
  float u, v, w, p;
};
__device__ __forceinline__ EntryTerms coarse_terms(const CoupledLevel& l, int j, const float4& xm) {
  const std::size_t Z = l.nnz;
  const float a = l.a[j];
  return EntryTerms{a * xm.x + l.g[j] * xm.w, a * xm.y + l.g[Z + j] * xm.w,
                    a * xm.z + l.g[2 * Z + j] * xm.w,
                    l.h[j] * xm.x + l.h[Z + j] * xm.y + l.h[2 * Z + j] * xm.z + l.c[j] * xm.w};
}
__device__ __forceinline__ float4 coarse_row(int i, const CoupledLevel& l,
                                             const float4* __restrict__ x) {
  const std::size_t N = l.n, Z = l.nnz;
  const int k = l.diag[i];
  const float4 xi = x[i];
  float yu = l.d[i] * xi.x + l.g[k] * xi.w;
  float yv = l.d[N + i] * xi.y + l.g[Z + k] * xi.w;
  float yw = l.d[2 * N + i] * xi.z + l.g[2 * Z + k] * xi.w;
  float yp = l.c[k] * xi.w + l.h[k] * xi.x + l.h[Z + k] * xi.y + l.h[2 * Z + k] * xi.z;
  const int end = l.rows[i + 1];
  int j = l.rows[i];
  for (; j + 4 <= end; j += 4) {
    int col[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) col[u] = l.cols[j + u];
    EntryTerms e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) e[u] = coarse_terms(l, j + u, x[col[u]]);
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (j + u != k) {
        yu += e[u].u;
        yv += e[u].v;
        yw += e[u].w;
        yp += e[u].p;
      }
  }
  for (; j < end; ++j) {
    const EntryTerms e = coarse_terms(l, j, x[l.cols[j]]);
    if (j != k) {
      yu += e.u;
      yv += e.v;
      yw += e.w;
      yp += e.p;
    }
  }
  return make_float4(yu, yv, yw, yp);
}

// (J x)_i by one warp, every lane returning the same value: the lanes form
// the terms of 32 entries at a time in parallel, then every lane adds them
// in CSR order, each read from its lane by shuffle, so the sums are
// coarse_row's bit for bit. Called by all 32 lanes of a warp with the same i.
__device__ __forceinline__ float4 coarse_row_warp(int i, const CoupledLevel& l,
                                                  const float4* __restrict__ x, int lane) {
  const std::size_t N = l.n, Z = l.nnz;
  const int k = l.diag[i];
  const float4 xi = x[i];
  float yu = l.d[i] * xi.x + l.g[k] * xi.w;
  float yv = l.d[N + i] * xi.y + l.g[Z + k] * xi.w;
  float yw = l.d[2 * N + i] * xi.z + l.g[2 * Z + k] * xi.w;
  float yp = l.c[k] * xi.w + l.h[k] * xi.x + l.h[Z + k] * xi.y + l.h[2 * Z + k] * xi.z;
  const int end = l.rows[i + 1];
  for (int base = l.rows[i]; base < end; base += 32) {
    const int j = base + lane;
    EntryTerms e{0.0f, 0.0f, 0.0f, 0.0f};
    if (j < end) e = coarse_terms(l, j, x[l.cols[j]]);
    const int count = min(32, end - base);
    for (int u = 0; u < count; ++u) {
      const float tu = __shfl_sync(0xffffffffu, e.u, u);
      const float tv = __shfl_sync(0xffffffffu, e.v, u);
      const float tw = __shfl_sync(0xffffffffu, e.w, u);
      const float tp = __shfl_sync(0xffffffffu, e.p, u);
      if (base + u != k) {
        yu += tu;
        yv += tv;
        yw += tw;
        yp += tp;
      }
    }
  }
  return make_float4(yu, yv, yw, yp);
}

// One damped block-Jacobi update of row i from r = b - (J x)_i (or b when x
// is zero), fv_coupled.kern.h:401-416.
__device__ __forceinline__ float4 coarse_update(const CoupledLevel& l, int i, float4 r,
                                                float4 base, float omega) {
  const std::size_t N = l.n, Z = l.nnz;
  const int k = l.diag[i];
  const float* d = l.d;
  const float4 s = block_solve(r, l.g[k], l.g[Z + k], l.g[2 * Z + k], d[4 * N + i], d[5 * N + i],
                               d[6 * N + i], d[7 * N + i], d[8 * N + i], d[9 * N + i],
                               d[10 * N + i]);
  return damped(base, s, omega);
}

// A warp per row (levels flagged wide): the residual and the sweep.
__global__ void k_cpl_coarse_residual_wide(CoupledLevel l, const float4* __restrict__ x,
                                           const float4* __restrict__ b,
                                           float4* __restrict__ r) {
  pdl_entry();
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < l.n; i += warps) {
    const float4 y = coarse_row_warp(i, l, x, lane);
    if (lane == 0) {
      const float4 bi = b[i];
      r[i] = make_float4(bi.x - y.x, bi.y - y.y, bi.z - y.z, bi.w - y.w);
    }
  }
}
__global__ void k_cpl_coarse_smooth_wide(CoupledLevel l, const float4* __restrict__ x,
                                         const float4* __restrict__ b, float4* __restrict__ next,
                                         float omega, int first) {
  pdl_entry();
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < l.n; i += warps) {
    float4 r = b[i];
    float4 base = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (!first) {
      const float4 y = coarse_row_warp(i, l, x, lane);
      r = make_float4(r.x - y.x, r.y - y.y, r.z - y.z, r.w - y.w);
      base = x[i];
    }
    if (lane == 0) next[i] = coarse_update(l, i, r, base, omega);
  }
}

__global__ void k_cpl_coarse_residual(CoupledLevel l, const float4* __restrict__ x,
                                      const float4* __restrict__ b, float4* __restrict__ r) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < l.n; i += gridDim.x * blockDim.x) {
    const float4 y = coarse_row(i, l, x);
    const float4 bi = b[i];
    r[i] = make_float4(bi.x - y.x, bi.y - y.y, bi.z - y.z, bi.w - y.w);
  }
}

// fv_coupled.kern.h:401-416 (coupled_coarse_smooth).
__global__ void k_cpl_coarse_smooth(CoupledLevel l, const float4* __restrict__ x,
                                    const float4* __restrict__ b, float4* __restrict__ next,
                                    float omega, int first) {
  pdl_entry();
  const std::size_t N = l.n, Z = l.nnz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < l.n; i += gridDim.x * blockDim.x) {
    float4 r = b[i];
    float4 base = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (!first) {
      const float4 y = coarse_row(i, l, x);
      r = make_float4(r.x - y.x, r.y - y.y, r.z - y.z, r.w - y.w);
      base = x[i];
    }
    const int k = l.diag[i];
    const float* d = l.d;
    const float4 s = block_solve(r, l.g[k], l.g[Z + k], l.g[2 * Z + k], d[4 * N + i],
                                 d[5 * N + i], d[6 * N + i], d[7 * N + i], d[8 * N + i],
                                 d[9 * N + i], d[10 * N + i]);
    next[i] = damped(base, s, omega);
  }
}

// The entry of column `col` in coarse row `row` (fv_coupled.kern.h:418-422
// searches linearly). A row's columns are sorted and unique (the contracted
// graph's targets in order, the diagonal in place), so a binary search finds
// the same entry in log2(row length) loads; rows on the small levels of tet
// meshes reach 150 entries.
__device__ __forceinline__ int entry_of(const int* __restrict__ rows, const int* __restrict__ cols,
                                        int row, int col) {
  int lo = rows[row];
  const int end = rows[row + 1];
  int hi = end;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cols[mid] < col)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo < end && cols[lo] == col ? lo : -1;
}

// Adds one off-diagonal contribution to entry e. Every load comes before any
// store, so the eight read-modify-writes overlap instead of each waiting for
// the last store (the arrays are distinct, the compiler cannot know it); each
// sum is the same single addition.
__device__ __forceinline__ void add_entry(const CoupledLevel& l, int e, float a, float c, float gx,
                                          float gy, float gz, float hx, float hy, float hz) {
  const std::size_t Z = l.nnz;
  const float a0 = l.a[e], c0 = l.c[e], gx0 = l.g[e], gy0 = l.g[Z + e], gz0 = l.g[2 * Z + e];
  const float hx0 = l.h[e], hy0 = l.h[Z + e], hz0 = l.h[2 * Z + e];
  l.a[e] = a0 + a;
  l.c[e] = c0 + c;
  l.g[e] = gx0 + gx;
  l.g[Z + e] = gy0 + gy;
  l.g[2 * Z + e] = gz0 + gz;
  l.h[e] = hx0 + hx;
  l.h[Z + e] = hy0 + hy;
  l.h[2 * Z + e] = hz0 + hz;
}

struct Sums {
  Csum u, v, w, c, gx, gy, gz, hx, hy, hz;
};
__device__ __forceinline__ void zero_row(const CoupledLevel& l, int i) {
  const std::size_t Z = l.nnz;
  for (int j = l.rows[i]; j < l.rows[i + 1]; ++j) {
    l.a[j] = 0.0f;
    l.c[j] = 0.0f;
    l.g[j] = 0.0f;
    l.g[Z + j] = 0.0f;
    l.g[2 * Z + j] = 0.0f;
    l.h[j] = 0.0f;
    l.h[Z + j] = 0.0f;
    l.h[2 * Z + j] = 0.0f;
  }
}
__device__ __forceinline__ void store_diagonal(const CoupledLevel& l, int i, int k, const Sums& s) {
  const std::size_t N = l.n, Z = l.nnz;
  l.d[i] = csum_value(s.u);
  l.d[N + i] = csum_value(s.v);
  l.d[2 * N + i] = csum_value(s.w);
  l.c[k] = csum_value(s.c);
  l.g[k] = csum_value(s.gx);
  l.g[Z + k] = csum_value(s.gy);
  l.g[2 * Z + k] = csum_value(s.gz);
  l.h[k] = csum_value(s.hx);
  l.h[Z + k] = csum_value(s.hy);
  l.h[2 * Z + k] = csum_value(s.hz);
}

// Galerkin from the matrix-free fine level (fv_coupled.kern.h:424-488,
// coupled_galerkin_fine): one thread owns one coarse row, so the order of
// every sum is the member order, then the cell-face order.
__global__ void k_cpl_galerkin_fine(CoupledLevel l, CoupledTransfer t, FineGeometry m,
                                    const float* __restrict__ mu, const float* __restrict__ diffusion,
                                    const float* __restrict__ mass,
                                    const float* __restrict__ coefficient,
                                    const float* __restrict__ weight,
                                    const float* __restrict__ cell, int nf_cells, float wc) {
  pdl_entry();
  const std::size_t F = nf_cells, Z = l.nnz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < l.n; i += gridDim.x * blockDim.x) {
    zero_row(l, i);
    Sums s{};
    const float half_wc = 0.5f * wc;
    for (int mm = t.offsets[i]; mm < t.offsets[i + 1]; ++mm) {
      const int q = t.members[mm];
      s.u = csum_add(s.u, cell[q]);
      s.v = csum_add(s.v, cell[F + q]);
      s.w = csum_add(s.w, cell[2 * F + q]);
      s.c = csum_add(s.c, cell[3 * F + q]);
      s.gx = csum_add(s.gx, wc * cell[4 * F + q]);
      s.gy = csum_add(s.gy, wc * cell[5 * F + q]);
      s.gz = csum_add(s.gz, wc * cell[6 * F + q]);
      s.hx = csum_add(s.hx, wc * cell[7 * F + q]);
      s.hy = csum_add(s.hy, wc * cell[8 * F + q]);
      s.hz = csum_add(s.hz, wc * cell[9 * F + q]);
      const float q00 = wc * cell[10 * F + q], q01 = wc * cell[11 * F + q], q02 = wc * cell[12 * F + q];
      const float q10 = wc * cell[13 * F + q], q11 = wc * cell[14 * F + q], q12 = wc * cell[15 * F + q];
      const float q20 = wc * cell[16 * F + q], q21 = wc * cell[17 * F + q], q22 = wc * cell[18 * F + q];
      for (int j = m.offsets[q]; j < m.offsets[q + 1]; ++j) {
        const int other = m.adjacent[j];
        if (other < 0) continue;
        const int f = m.faces[j];
        const float sg = m.sign[j];
        const float uu = -mu[f] * diffusion[f] + fminf(sg * mass[f], 0.0f);
        const float bx = half_wc * sg * m.sx[f], by = half_wc * sg * m.sy[f],
                    bz = half_wc * sg * m.sz[f];
        const float gx = bx + q00 * m.dx[j] + q01 * m.dy[j] + q02 * m.dz[j];
        const float gy = by + q10 * m.dx[j] + q11 * m.dy[j] + q12 * m.dz[j];
        const float gz = bz + q20 * m.dx[j] + q21 * m.dy[j] + q22 * m.dz[j];
        const float pp = -coefficient[f];
        const float share = wc * sg * share_of(weight, q, other);
        const float hx = share * m.sx[f], hy = share * m.sy[f], hz = share * m.sz[f];
        const int target = t.aggregate[other];
        if (target == i) {
          s.u = csum_add(s.u, uu);
          s.v = csum_add(s.v, uu);
          s.w = csum_add(s.w, uu);
          s.gx = csum_add(s.gx, gx);
          s.gy = csum_add(s.gy, gy);
          s.gz = csum_add(s.gz, gz);
          s.hx = csum_add(s.hx, hx);
          s.hy = csum_add(s.hy, hy);
          s.hz = csum_add(s.hz, hz);
          s.c = csum_add(s.c, pp);
        } else {
          // The coarse pattern holds every aggregate a member borders (the
          // contracted graph), so the search always finds it.
          const int e = entry_of(l.rows, l.cols, i, target);
          if (e < 0) continue;
          add_entry(l, e, uu, pp, gx, gy, gz, hx, hy, hz);
        }
      }
    }
    store_diagonal(l, i, l.diag[i], s);
  }
}

// fv_coupled.kern.h:490-524 (coupled_galerkin_coarse).
__global__ void k_cpl_galerkin_coarse(CoupledLevel l, CoupledTransfer t, CoupledLevel f) {
  pdl_entry();
  const std::size_t Z = l.nnz, FN = f.n, FZ = f.nnz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < l.n; i += gridDim.x * blockDim.x) {
    zero_row(l, i);
    Sums s{};
    for (int mm = t.offsets[i]; mm < t.offsets[i + 1]; ++mm) {
      const int row = t.members[mm];
      s.u = csum_add(s.u, f.d[row]);
      s.v = csum_add(s.v, f.d[FN + row]);
      s.w = csum_add(s.w, f.d[2 * FN + row]);
      const int fd = f.diag[row];
      for (int j = f.rows[row]; j < f.rows[row + 1]; ++j) {
        const int target = t.aggregate[f.cols[j]];
        if (j == fd || target == i) {
          if (j != fd) {
            s.u = csum_add(s.u, f.a[j]);
            s.v = csum_add(s.v, f.a[j]);
            s.w = csum_add(s.w, f.a[j]);
          }
          s.gx = csum_add(s.gx, f.g[j]);
          s.gy = csum_add(s.gy, f.g[FZ + j]);
          s.gz = csum_add(s.gz, f.g[2 * FZ + j]);
          s.hx = csum_add(s.hx, f.h[j]);
          s.hy = csum_add(s.hy, f.h[FZ + j]);
          s.hz = csum_add(s.hz, f.h[2 * FZ + j]);
          s.c = csum_add(s.c, f.c[j]);
        } else {
          const int e = entry_of(l.rows, l.cols, i, target);
          if (e < 0) continue;
          add_entry(l, e, f.a[j], f.c[j], f.g[j], f.g[FZ + j], f.g[2 * FZ + j], f.h[j],
                    f.h[FZ + j], f.h[2 * FZ + j]);
        }
      }
    }
    store_diagonal(l, i, l.diag[i], s);
  }
}

// fv_coupled.kern.h:526-534 (coupled_coarse_gsum): into 3n of scratch.
__global__ void k_cpl_coarse_gsum(CoupledLevel l, float* __restrict__ r) {
  pdl_entry();
  const std::size_t N = l.n, Z = l.nnz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < l.n; i += gridDim.x * blockDim.x) {
    float gx = 0.0f, gy = 0.0f, gz = 0.0f;
    for (int j = l.rows[i]; j < l.rows[i + 1]; ++j) {
      gx += fabsf(l.g[j]);
      gy += fabsf(l.g[Z + j]);
      gz += fabsf(l.g[2 * Z + j]);
    }
    r[i] = gx;
    r[N + i] = gy;
    r[2 * N + i] = gz;
  }
}

// fv_coupled.kern.h:536-552 (coupled_coarse_schur): cs and the block inverse.
__global__ void k_cpl_coarse_schur(CoupledLevel l, const float* __restrict__ r) {
  pdl_entry();
  const std::size_t N = l.n, Z = l.nnz;
  float* d = l.d;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < l.n; i += gridDim.x * blockDim.x) {
    const int k = l.diag[i];
    float sum = 0.0f;
    for (int j = l.rows[i]; j < l.rows[i + 1]; ++j) {
      if (j == k) continue;
      const int m = l.cols[j];
      sum += fabsf(l.h[j]) * r[m] / fmaxf(d[m], 1.0e-30f) +
             fabsf(l.h[Z + j]) * r[N + m] / fmaxf(d[N + m], 1.0e-30f) +
             fabsf(l.h[2 * Z + j]) * r[2 * N + m] / fmaxf(d[2 * N + m], 1.0e-30f);
    }
    d[3 * N + i] = sum;
    const BlockInverse b = block_prepare(d[i], d[N + i], d[2 * N + i], l.g[k], l.g[Z + k],
                                         l.g[2 * Z + k], l.h[k], l.h[Z + k], l.h[2 * Z + k],
                                         l.c[k] + sum);
    d[4 * N + i] = b.iu;
    d[5 * N + i] = b.iv;
    d[6 * N + i] = b.iw;
    d[7 * N + i] = b.hu;
    d[8 * N + i] = b.hv;
    d[9 * N + i] = b.hw;
    d[10 * N + i] = b.schur;
  }
}

// fv_coupled.kern.h:554-567: restriction sums members in member order;
// prolongation adds the aggregate's correction.
__global__ void __launch_bounds__(kBlock, 8) k_cpl_restrict(int nc, const int* __restrict__ offsets,
                               const int* __restrict__ members, const float4* __restrict__ fine,
                               float4* __restrict__ coarse) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
    float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int m = offsets[i]; m < offsets[i + 1]; ++m) {
      const float4 v = fine[members[m]];
      s.x += v.x;
      s.y += v.y;
      s.z += v.z;
      s.w += v.w;
    }
    coarse[i] = s;
  }
}
__global__ void __launch_bounds__(kBlock, 8) k_cpl_prolong(int nf, const int* __restrict__ aggregate,
                              const float4* __restrict__ coarse, float4* __restrict__ fine) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
    const float4 c = coarse[aggregate[i]];
    float4 v = fine[i];
    v.x += c.x;
    v.y += c.y;
    v.z += c.z;
    v.w += c.w;
    fine[i] = v;
  }
}

// ---- the small coarse levels in one launch --------------------------------------
//
// The V-cycle below a level of at most CoupledTail::kMaxRows rows, in one
// block of 1024 threads: each sweep, residual, restriction and prolongation
// is a block-stride loop over the level's rows with the arithmetic of the
// kernels above, separated by __syncthreads (no inter-block waits). The
// ping-pong roles of each level's x and tmp follow the host's: the kernel
// starts from the pointers it is given and swaps them as the separate
// launches would. On a 128^3 box this replaces about 25 launches of 3-6 us
// per V-cycle by one. Rows stay one per thread here even on levels flagged
// wide: with 32 warps for the whole level, a warp per row measured slower
// (388 against 252 us per launch on a 875-row level with 152-entry rows).
__device__ __forceinline__ void tail_smooth(const CoupledLevel& l, float4*& x, float4*& tmp,
                                            const float4* __restrict__ b, int sweeps, bool first,
                                            float omega) {
  for (int s = 0; s < sweeps; ++s) {
    const bool zero = first && s == 0;
    for (int i = threadIdx.x; i < l.n; i += blockDim.x) {
      float4 r = b[i];
      float4 base = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (!zero) {
        const float4 y = coarse_row(i, l, x);
        r = make_float4(r.x - y.x, r.y - y.y, r.z - y.z, r.w - y.w);
        base = x[i];
      }
      tmp[i] = coarse_update(l, i, r, base, omega);
    }
    __syncthreads();
    float4* swap = x;
    x = tmp;
    tmp = swap;
  }
}

__global__ void __launch_bounds__(1024) k_cpl_tail(CoupledTail t) {
  pdl_entry();
  float4* x[CoupledTail::kMaxLevels];
  float4* tmp[CoupledTail::kMaxLevels];
  for (int k = 0; k < t.levels; ++k) {
    x[k] = t.x[k];
    tmp[k] = t.tmp[k];
  }
  const int last = t.levels - 1;
  for (int k = 0; k < last; ++k) {
    const CoupledLevel& l = t.op[k];
    tail_smooth(l, x[k], tmp[k], t.b[k], t.pre, true, t.omega);
    for (int i = threadIdx.x; i < l.n; i += blockDim.x) {
      const float4 y = coarse_row(i, l, x[k]);
      const float4 bi = t.b[k][i];
      tmp[k][i] = make_float4(bi.x - y.x, bi.y - y.y, bi.z - y.z, bi.w - y.w);
    }
    __syncthreads();
    const CoupledTransfer& tr = t.down[k];
    for (int i = threadIdx.x; i < t.op[k + 1].n; i += blockDim.x) {
      float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      for (int m = tr.offsets[i]; m < tr.offsets[i + 1]; ++m) {
        const float4 v = tmp[k][tr.members[m]];
        s.x += v.x;
        s.y += v.y;
        s.z += v.z;
        s.w += v.w;
      }
      t.b[k + 1][i] = s;
    }
    __syncthreads();
  }
  tail_smooth(t.op[last], x[last], tmp[last], t.b[last], t.coarsest, true, t.omega);
  for (int k = last - 1; k >= 0; --k) {
    const CoupledTransfer& tr = t.down[k];
    for (int i = threadIdx.x; i < t.op[k].n; i += blockDim.x) {
      const float4 c = x[k + 1][tr.aggregate[i]];
      float4 v = x[k][i];
      v.x += c.x;
      v.y += c.y;
      v.z += c.z;
      v.w += c.w;
      x[k][i] = v;
    }
    __syncthreads();
    tail_smooth(t.op[k], x[k], tmp[k], t.b[k], t.post, false, t.omega);
  }
}

// ---- the update of the flow fields --------------------------------------------

// fv_coupled.kern.h:571-578 (coupled_update).
__global__ void k_cpl_update(int n, const float4* __restrict__ delta, float* __restrict__ u,
                             float* __restrict__ v, float* __restrict__ w, float* __restrict__ p,
                             float alpha_u, float alpha_p) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 d = delta[i];
    u[i] += alpha_u * d.x;
    v[i] += alpha_u * d.y;
    w[i] += alpha_u * d.z;
    p[i] += alpha_p * d.w;
  }
}

// Knuth's two-sum and the slack-held pair addition (prelude.h:103-149,
// kpair_add).
struct Pair2 {
  float hi, lo;
};
__device__ __forceinline__ Pair2 two_sum(float a, float b) {
  const float sum = a + b;
  const float part = sum - a;
  return Pair2{sum, (a - (sum - part)) + (b - part)};
}
__device__ __forceinline__ Pair2 pair_add(float hi, float lo, float d, float slack) {
  const float low = lo + d;
  if (fabsf(low) <= slack) return Pair2{hi, low};
  const Pair2 s = two_sum(hi, d);
  return two_sum(s.hi, s.lo + lo);
}

// fv_coupled.kern.h:582-591 (coupled_paired_update).
__global__ void k_cpl_paired_update(int n, const float4* __restrict__ delta, float* __restrict__ u,
                                    float* __restrict__ v, float* __restrict__ w,
                                    float* __restrict__ p, float* __restrict__ u_lo,
                                    float* __restrict__ v_lo, float* __restrict__ w_lo,
                                    float* __restrict__ p_lo, float alpha_u, float alpha_p,
                                    float velocity_slack, float pressure_slack) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 d = delta[i];
    Pair2 x = pair_add(u[i], u_lo[i], alpha_u * d.x, velocity_slack);
    u[i] = x.hi;
    u_lo[i] = x.lo;
    x = pair_add(v[i], v_lo[i], alpha_u * d.y, velocity_slack);
    v[i] = x.hi;
    v_lo[i] = x.lo;
    x = pair_add(w[i], w_lo[i], alpha_u * d.z, velocity_slack);
    w[i] = x.hi;
    w_lo[i] = x.lo;
    x = pair_add(p[i], p_lo[i], alpha_p * d.w, pressure_slack);
    p[i] = x.hi;
    p_lo[i] = x.lo;
  }
}

// The closed-domain gauge (fv_coupled.kern.h:592-620): the reference cell's
// value is picked into `value` by one thread, then subtracted everywhere.
__global__ void k_cpl_pick(const float* __restrict__ p, const float* __restrict__ p_lo,
                           float* __restrict__ value, int index) {
  pdl_entry();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    value[0] = p[index];
    value[1] = p_lo ? p_lo[index] : 0.0f;
  }
}
__global__ void k_cpl_gauge(int n, const float* __restrict__ value, float* __restrict__ p) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] -= value[0];
}
__global__ void k_cpl_paired_gauge(int n, const float* __restrict__ value, float* __restrict__ p,
                                   float* __restrict__ p_lo, float pressure_slack) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Pair2 x = pair_add(p[i], p_lo[i], -(value[0] + value[1]), pressure_slack);
    p[i] = x.hi;
    p_lo[i] = x.lo;
  }
}

FineGeometry geometry(const CoupledMeshDevice& m) {
  return FineGeometry{m.offsets, m.faces, m.sign, m.adjacent, m.sx, m.sy, m.sz, m.dx, m.dy, m.dz};
}

}  // namespace

namespace launch {

void cpl_copy_diagonal(int n, const int* rows, const int* diag, const float* values,
                       const float* physical, float* plane, float inverse_courant, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_cpl_copy_diagonal, grid_for(n), kBlock, 0, s, n, rows, diag, values, physical, plane,
      inverse_courant);
}

void cpl_assemble(const CoupledMeshDevice& m, const CoupledSolveInputs& in, float* cell,
                  float* coefficient, float4* b, float* scratch, CoupledFine op, float wc,
                  float coefficient_scale, float continuity_scale, int reference,
                  cudaStream_t s) {
  const int n = m.n, nf = m.n_faces;
  if (n <= 0) return;
  const FineGeometry g = geometry(m);
  counter += 7;
  pdl(k_cpl_face_coefficient, grid_for(nf), kBlock, 0, s, nf, m.n_internal, m.owner,
      m.neighbour, m.kind, m.diffusion, m.volume, in.physical_diagonal, coefficient,
      coefficient_scale);
  pdl(k_cpl_velocity_block, grid_for(n), kBlock, 0, s, n, m.n_internal, m.offsets, m.faces,
      m.sign, m.adjacent, m.kind, m.sx, m.sy, m.sz, in.face_weights, cell);
  pdl(k_cpl_rhs, grid_for(n), kBlock, 0, s, n, m.offsets, m.faces, m.sign,
      static_cast<const float*>(coefficient), in.mass, in.net_outflow, in.ru, in.rv, in.rw, cell,
      b, reference, continuity_scale);
  pdl(k_cpl_fine_gsum, grid_for(n), kBlock, 0, s, n, g, static_cast<const float*>(cell), scratch,
      wc);
  pdl(k_cpl_fine_schur, grid_for(n), kBlock, 0, s, n, g, in.face_weights,
      static_cast<const float*>(scratch), cell, wc);
  pdl(k_cpl_face_records, grid_for(nf), kBlock, 0, s, nf, m.sx, m.sy, m.sz,
      static_cast<const float*>(coefficient), const_cast<float4*>(op.face));
  pdl(k_cpl_fine_pack, grid_for(n), kBlock, 0, s, n, m.width, g, in.viscosity, m.diffusion,
      in.mass, in.face_weights, static_cast<const float*>(cell), op, wc);
}

void cpl_galerkin_fine(const CoupledLevel& l, const CoupledTransfer& t, const CoupledMeshDevice& m,
                       const CoupledSolveInputs& in, const float* coefficient, const float* cell,
                       float wc, cudaStream_t s) {
  if (l.n <= 0) return;
  ++counter;
  pdl(k_cpl_galerkin_fine, grid_for(l.n), kBlock, 0, s, l, t, geometry(m), in.viscosity,
      m.diffusion, in.mass, coefficient, in.face_weights, cell, m.n, wc);
}

void cpl_galerkin_coarse(const CoupledLevel& l, const CoupledTransfer& t, const CoupledLevel& f,
                         cudaStream_t s) {
  if (l.n <= 0) return;
  ++counter;
  pdl(k_cpl_galerkin_coarse, grid_for(l.n), kBlock, 0, s, l, t, f);
}

void cpl_coarse_prepare(const CoupledLevel& l, float* scratch, cudaStream_t s) {
  if (l.n <= 0) return;
  counter += 2;
  pdl(k_cpl_coarse_gsum, grid_for(l.n), kBlock, 0, s, l, scratch);
  pdl(k_cpl_coarse_schur, grid_for(l.n), kBlock, 0, s, l, static_cast<const float*>(scratch));
}

void cpl_fine_spmv(int n, const CoupledFine& op, int width, const float4* x, float4* y,
                   cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_cpl_fine_spmv, grid_for(n), kBlock, 0, s, n, width, op, x, y);
}

void cpl_fine_residual(int n, const CoupledFine& op, int width, const float4* x, const float4* b,
                       float4* r, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_cpl_fine_residual, grid_for(n), kBlock, 0, s, n, width, op, x, b, r);
}

void cpl_fine_smooth(int n, const CoupledFine& op, int width, const float4* x, const float4* b,
                     float4* next, float omega, bool first, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_cpl_fine_smooth, grid_for(n), kBlock, 0, s, n, width, op, x, b, next, omega,
      first ? 1 : 0);
}

void cpl_coarse_residual(const CoupledLevel& l, const float4* x, const float4* b, float4* r,
                         cudaStream_t s) {
  if (l.n <= 0) return;
  ++counter;
  if (l.wide)
    pdl(k_cpl_coarse_residual_wide, grid_for(32LL * l.n), kBlock, 0, s, l, x, b, r);
  else
    pdl(k_cpl_coarse_residual, grid_for(l.n), kBlock, 0, s, l, x, b, r);
}

void cpl_coarse_smooth(const CoupledLevel& l, const float4* x, const float4* b, float4* next,
                       float omega, bool first, cudaStream_t s) {
  if (l.n <= 0) return;
  ++counter;
  if (l.wide)
    pdl(k_cpl_coarse_smooth_wide, grid_for(32LL * l.n), kBlock, 0, s, l, x, b, next, omega,
        first ? 1 : 0);
  else
    pdl(k_cpl_coarse_smooth, grid_for(l.n), kBlock, 0, s, l, x, b, next, omega, first ? 1 : 0);
}

void cpl_restrict(int nc, const int* offsets, const int* members, const float4* fine,
                  float4* coarse, cudaStream_t s) {
  if (nc <= 0) return;
  ++counter;
  pdl(k_cpl_restrict, grid_for(nc), kBlock, 0, s, nc, offsets, members, fine, coarse);
}

void cpl_prolong(int nf, const int* aggregate, const float4* coarse, float4* fine,
                 cudaStream_t s) {
  if (nf <= 0) return;
  ++counter;
  pdl(k_cpl_prolong, grid_for(nf), kBlock, 0, s, nf, aggregate, coarse, fine);
}

void cpl_update(int n, const float4* delta, float* u, float* v, float* w, float* p, float alpha_u,
                float alpha_p, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_cpl_update, grid_for(n), kBlock, 0, s, n, delta, u, v, w, p, alpha_u, alpha_p);
}

void cpl_paired_update(int n, const float4* delta, float* u, float* v, float* w, float* p,
                       float* u_lo, float* v_lo, float* w_lo, float* p_lo, float alpha_u,
                       float alpha_p, float velocity_slack, float pressure_slack, cudaStream_t s) {
  if (n <= 0) return;
  ++counter;
  pdl(k_cpl_paired_update, grid_for(n), kBlock, 0, s, n, delta, u, v, w, p, u_lo, v_lo, w_lo,
      p_lo, alpha_u, alpha_p, velocity_slack, pressure_slack);
}

void cpl_tail(const CoupledTail& t, cudaStream_t s) {
  if (t.levels <= 0) return;
  ++counter;
  pdl(k_cpl_tail, 1, 1024, 0, s, t);
}

void cpl_gauge(int n, float* p, float* p_lo, float pressure_slack, float* value, int index,
               cudaStream_t s) {
  if (n <= 0) return;
  counter += 2;
  pdl(k_cpl_pick, 1, 32, 0, s, static_cast<const float*>(p), static_cast<const float*>(p_lo),
      value, index);
  if (p_lo)
    pdl(k_cpl_paired_gauge, grid_for(n), kBlock, 0, s, n, static_cast<const float*>(value), p,
        p_lo, pressure_slack);
  else
    pdl(k_cpl_gauge, grid_for(n), kBlock, 0, s, n, static_cast<const float*>(value), p);
}

}  // namespace launch
}  // namespace kb2
