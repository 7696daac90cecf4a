// Host launchers for the Coupled (4x4-block) solve kernels
// (src/kutta/kernels/fv_coupled.kern.h). Device pointers and sizes only;
// every launcher enqueues on `s` and never synchronises.
#pragma once

#include <cuda_runtime.h>

#include "kernels.hpp"

namespace kb2 {

// The mesh, stencil and least-squares arrays the kernels read, on the device.
struct CoupledMeshDevice {
  int n = 0, n_faces = 0, n_internal = 0;
  int width = 0;  // most internal faces of one cell (ELL slots of the fine operator)
  const int* owner = nullptr;
  const int* neighbour = nullptr;
  const int* offsets = nullptr;   // cell -> its cell-face entries (n + 1)
  const int* faces = nullptr;     // per entry
  const float* sign = nullptr;    // per entry, +1 owner / -1 neighbour
  const int* adjacent = nullptr;  // per entry: the other cell, or -(boundary face + 1)
  const int* kind = nullptr;      // per boundary face
  const float *sx = nullptr, *sy = nullptr, *sz = nullptr;  // face area vectors
  const float *dx = nullptr, *dy = nullptr, *dz = nullptr;  // least-squares rows per entry
  const float* diffusion = nullptr;  // per face
  const float* volume = nullptr;     // per cell
};

// The per-solve flow inputs (device pointers; net_outflow may be null).
struct CoupledSolveInputs {
  const float *ru = nullptr, *rv = nullptr, *rw = nullptr;
  const float* mass = nullptr;
  const float* viscosity = nullptr;
  const float* physical_diagonal = nullptr;
  const float* face_weights = nullptr;
  const float* net_outflow = nullptr;
};

// The fine operator's per-cell records and ELL slots (slot-major: slot s of
// cell i at s n + i); see coupled_kernels.cu.
struct CoupledFine {
  float4* diag;         // (du, dv, dw, cd)
  float4* coupling;     // (wc Gx, wc Gy, wc Gz, wc Hx)
  float2* coupling_yz;  // (wc Hy, wc Hz)
  float4* inverse;      // (iu, iv, iw, schur)
  float4* inverse_h;    // (Hx iu, Hy iv, Hz iw, 0)
  float4* edge;         // per slot: (a, gx, gy, gz)
  float* edge_h;        // per slot: h
  int2* link;           // per slot: (neighbour, face), neighbour -1 past the row's end
  const float4* face;   // per face: (sx, sy, sz, Rhie-Chow coefficient)
};

// One coarse level: CSR with a, c per entry, G and H as 3 nnz [x | y | z],
// and 11 planes of n per row (du dv dw cs iu iv iw hx iu hy iv hz iw schur).
struct CoupledLevel {
  int n = 0, nnz = 0;
  const int* rows = nullptr;
  const int* cols = nullptr;
  const int* diag = nullptr;
  float *a = nullptr, *c = nullptr, *g = nullptr, *h = nullptr, *d = nullptr;
  // Rows long enough (a hub aggregate bordering a hundred others) that the
  // separately launched row kernels give each row a warp instead of a
  // thread; the results are the same bits either way.
  int wide = 0;
};

// Level k -> k+1: aggregate of each fine row, member lists of each coarse row.
struct CoupledTransfer {
  const int* aggregate = nullptr;
  const int* offsets = nullptr;
  const int* members = nullptr;
};

// The V-cycle of the small coarse levels (by default each at most kMaxRows
// rows; the kernel itself takes any size, its block looping over the rows) as
// one single-block launch: levels 0 .. levels-1 of the tail, the first receiving
// its right-hand side from the level above; x/tmp are each level's current
// ping-pong roles.
struct CoupledTail {
  static constexpr int kMaxLevels = 12;
  static constexpr int kMaxRows = 1024;
  int levels = 0;
  int pre = 1, post = 2, coarsest = 8;
  float omega = 0.7f;
  CoupledLevel op[kMaxLevels];
  CoupledTransfer down[kMaxLevels];  // down[k]: tail level k -> k + 1
  float4* x[kMaxLevels];
  float4* tmp[kMaxLevels];
  float4* b[kMaxLevels];
};

namespace launch {

// Plane = the cell data's slot k (momentum diagonal of component k).
void cpl_copy_diagonal(int n, const int* rows, const int* diag, const float* values,
                       const float* physical, float* plane, float inverse_courant, cudaStream_t s);
// Face coefficients, H_ii, pressure diagonal and right-hand side b (float4
// per cell), the smoother's Schur bound, the face records and the packed fine
// operator. scratch: 3n floats.
void cpl_assemble(const CoupledMeshDevice& m, const CoupledSolveInputs& in, float* cell,
                  float* coefficient, float4* b, float* scratch, CoupledFine op, float wc,
                  float coefficient_scale, float continuity_scale, int reference, cudaStream_t s);
void cpl_galerkin_fine(const CoupledLevel& l, const CoupledTransfer& t, const CoupledMeshDevice& m,
                       const CoupledSolveInputs& in, const float* coefficient, const float* cell,
                       float wc, cudaStream_t s);
void cpl_galerkin_coarse(const CoupledLevel& l, const CoupledTransfer& t, const CoupledLevel& f,
                         cudaStream_t s);
// |G| row sums into scratch (3n), then cs and the block inverse.
void cpl_coarse_prepare(const CoupledLevel& l, float* scratch, cudaStream_t s);

void cpl_fine_spmv(int n, const CoupledFine& op, int width, const float4* x, float4* y,
                   cudaStream_t s);
void cpl_fine_residual(int n, const CoupledFine& op, int width, const float4* x, const float4* b,
                       float4* r, cudaStream_t s);
void cpl_fine_smooth(int n, const CoupledFine& op, int width, const float4* x, const float4* b,
                     float4* next, float omega, bool first, cudaStream_t s);
void cpl_coarse_residual(const CoupledLevel& l, const float4* x, const float4* b, float4* r,
                         cudaStream_t s);
void cpl_coarse_smooth(const CoupledLevel& l, const float4* x, const float4* b, float4* next,
                       float omega, bool first, cudaStream_t s);
void cpl_restrict(int nc, const int* offsets, const int* members, const float4* fine,
                  float4* coarse, cudaStream_t s);
void cpl_prolong(int nf, const int* aggregate, const float4* coarse, float4* fine,
                 cudaStream_t s);

void cpl_tail(const CoupledTail& t, cudaStream_t s);

void cpl_update(int n, const float4* delta, float* u, float* v, float* w, float* p, float alpha_u,
                float alpha_p, cudaStream_t s);
void cpl_paired_update(int n, const float4* delta, float* u, float* v, float* w, float* p,
                       float* u_lo, float* v_lo, float* w_lo, float* p_lo, float alpha_u,
                       float alpha_p, float velocity_slack, float pressure_slack, cudaStream_t s);
// p -= p[index] (or, with p_lo, the pair's value at index, slack-held);
// value: 2 floats of device scratch.
void cpl_gauge(int n, float* p, float* p_lo, float pressure_slack, float* value, int index,
               cudaStream_t s);

}  // namespace launch
}  // namespace kb2
