// Host launchers for the sm_100a solver kernels. Plain pointers and sizes;
// every launcher enqueues on `stream` and never synchronises.
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

namespace kb2 {

// Scalar epilogues run by the last block of a fused reduction, after the
// reduced value is stored as a (hi, lo) pair: the single-thread scalar kernels
// of src/kutta/kernels/scalars.kern.h:51-121.
enum class Epilogue : int {
  None = 0,
  PcgAlpha,         // solver_pcg_alpha
  CheckPcg,         // solver_check(pcg = 1)
  CheckBicg,        // solver_check(pcg = 0)
  PcgBeta,          // solver_pcg_beta(flexible = 0)
  PcgBetaFlexible,  // solver_pcg_beta(flexible = 1)
  BicgBeta,         // solver_bicg_beta
  BicgAlpha,        // solver_bicg_alpha
  BicgS,            // solver_bicg_s
  BicgOmega,        // solver_bicg_omega
};

// Reduction modes of Device::reduce_into / host reductions.
enum class ReduceMode : int { Sum = 0, Dot = 1, Dot2 = 2, MaxAbs = 3 };

// Doubles of reduction scratch per reducer: two partials per block for at most
// 148 SMs x 8 blocks.
constexpr int kReducePartials = 2 * 148 * 8;

struct DeviceReducer {
  double* partials;   // 2 * kMaxBlocks doubles
  unsigned* ticket;   // zero-initialised counter
};

namespace launch {

// Kernels launched by this library since load (every launcher increments it).
extern std::atomic<long long> counter;

// ---- CSR row kernels (one row per thread, grid-stride) -------------------
// y = A x, Kahan-compensated (csr_spmv). status may be null (unguarded).
void spmv(int n, const int* rows, const int* cols, const float* vals, const float* x, float* y,
          const int* status, cudaStream_t s);
// q = A p and w.q -> scalars[offset] as a pair, then `epi` (guarded by status).
void spmv_dot(int n, const int* rows, const int* cols, const float* vals, const float* p,
              const float* w, float* q, DeviceReducer red, float* scalars, int offset,
              int* status, Epilogue epi, cudaStream_t s);
// The mixed solve's packed copy of the fine operator ("packed rows"): per
// row i the diagonal value diag[i] and `width` (4 or 8) off-diagonal slots,
// values vals[width i + k] and int16 column offsets offsets[width i + k] =
// col - i in column order, unused slots with offset 0 and value 0. A row is
// 6 width + 4 bytes instead of CSR's 8 (entries) + 4 bytes: on a tet mesh 28
// instead of 44. The kernels below visit a row's terms in CSR column order
// (negative offsets, the diagonal, positive offsets) with the CSR kernels'
// arithmetic, grids and reductions, so every result equals the CSR kernel's
// bit for bit.
struct PackedRows {
  int width;
  const float* vals;
  const short* offsets;
  const float* diag;
};
// Values of the packed rows from CSR values (pattern fixed at packing setup).
void pack_rows(int n, int width, const int* rows, const int* cols, const int* diag,
               const float* vals, float* packed, float* packed_diag, cudaStream_t s);
void packed_residual(int n, PackedRows a, const float* x, const float* b, float* r,
                     const int* status, cudaStream_t s);
void packed_spmv_dot(int n, PackedRows a, const float* p, const float* w, float* q,
                     DeviceReducer red, float* scalars, int offset, int* status, Epilogue epi,
                     cudaStream_t s);
void packed_smooth_dot2(int n, PackedRows a, const float* x, const float* b, const float* inv,
                        float* next, const float* q, DeviceReducer red, float* scalars,
                        int offset, int* status, Epilogue epi, cudaStream_t s);
// r = b - A x, Neumaier + Dekker compensated (csr_residual). status may be null.
void residual(int n, const int* rows, const int* cols, const float* vals, const float* x,
              const float* b, float* r, const int* status, cudaStream_t s);
// next = x + (2/3) inv (b - A x)  (amg_smooth); zero_start: x treated as the
// zero vector without reading it (amg_smooth_zero).
void smooth(int n, const int* rows, const int* cols, const float* vals, const float* x,
            const float* b, const float* inv, float* next, const int* status, bool zero_start,
            cudaStream_t s);
// The fine post-sweep with the flexible PCG's r.z and z.q (b = r, next = z)
// reduced into scalars[offset..] and the epilogue run, as reduce_into(Dot2).
void smooth_dot2(int n, const int* rows, const int* cols, const float* vals, const float* x,
                 const float* b, const float* inv, float* next, const float* q, DeviceReducer red,
                 float* scalars, int offset, int* status, Epilogue epi, cudaStream_t s);
// <=24-row coarsest level, `sweeps` Jacobi sweeps in one thread (amg_coarse_solve).
void coarse_solve(int count, const int* rows, const int* cols, const float* vals, float* x,
                  const float* b, const float* inv, const int* status, int sweeps,
                  cudaStream_t s);
// Inverse (L1) diagonal and invalid flags (krylov_diagonal); the max of the
// flags is written to check[slot] as a double (no host wait).
void diagonal(int n, const int* rows, const int* diag, const float* vals, float* inverse,
              int use_l1, DeviceReducer red, double* check, int slot, cudaStream_t s);

// ---- AMG transfer and Galerkin --------------------------------------------
void restrict_(int nc, const int* offsets, const int* members, const float* fine, float* coarse,
               const int* status, cudaStream_t s);
void prolong(int nf, const int* aggregate, const float* coarse, float* fine, const int* status,
             cudaStream_t s);
void galerkin(int nnz_c, const int* offsets, const int* entries, const float* fine, float* coarse,
              cudaStream_t s);
// amg_m_matrix_diagonal: surplus holds nf floats of scratch.
void m_matrix_diagonal(int nf, int nc, const int* offsets, const int* members, const int* fine_rows,
                       const int* fine_diag, const float* fine, const int* rows, const int* diag,
                       float* coarse, float* surplus, cudaStream_t s);

// ---- Krylov vector updates (guarded by status) ----------------------------
// x += a p; r -= a q; then r.r -> scalars[18] and solver_check(pcg = 1).
void pcg_step_dot(int n, float* x, float* r, const float* p, const float* q, DeviceReducer red,
                  float* scalars, int* status, cudaStream_t s);
void direction(int n, const float* z, float* p, const float* scalars, const int* status,
               cudaStream_t s);
void bicg_direction(int n, const float* r, const float* v, float* p, const float* scalars,
                    const int* status, cudaStream_t s);
void bicg_difference(int n, const float* r, const float* q, float* sv, const float* scalars,
                     const int* status, cudaStream_t s);
void bicg_step(int n, float* x, float* r, const float* z, const float* zs, const float* sv,
               const float* t, const float* scalars, const int* status, cudaStream_t s);
void multiply(int n, const float* r, const float* inverse, float* z, const int* status,
              cudaStream_t s);
void axpy(int n, float* y, const float* x, float a, cudaStream_t s);
void fill(int n, float* x, float value, cudaStream_t s);

// ---- reductions -----------------------------------------------------------
// Sum / Dot / Dot2 of the first n entries, FP64, written as pair(s) into
// scalars[offset..]; then `epi`. guard: skip entirely when status[0] != 0
// (every consumer of these slots is itself guarded).
void reduce_into(ReduceMode mode, int n, const float* x, const float* y, const float* u,
                 const float* v, DeviceReducer red, float* scalars, int offset, int* status,
                 bool guard, Epilogue epi, cudaStream_t s);
// Host reductions: FP64 value into out[slot] (device double array).
void reduce_value(ReduceMode mode, int n, const float* x, const float* y, DeviceReducer red,
                  double* out, int slot, cudaStream_t s);

// ---- mixed precision (no reference counterpart) ---------------------------
// Coarse operator as BF16 times a per-row FP32 scale (max |a_ij|).
void bf16_pack(int n, const int* rows, const float* vals, unsigned short* v16, float* scale,
               cudaStream_t s);
void bf16_smooth(int n, const int* rows, const int* cols, const unsigned short* v16,
                 const float* scale, const float* x, const float* b, const float* inv, float* next,
                 const int* status, bool zero_start, cudaStream_t s);
void bf16_residual(int n, const int* rows, const int* cols, const unsigned short* v16,
                   const float* scale, const float* x, const float* b, float* r, const int* status,
                   cudaStream_t s);
// Restriction for the mixed V-cycle: plain FP32 sums, four lanes per aggregate.
void restrict_lanes(int nc, const int* offsets, const int* members, const float* fine,
                    float* coarse, const int* status, cudaStream_t s);
// K-cycle inner step on a BF16 level: q = A p with p.q and w.p (gcr: q.q and
// w.q) -> scalars[0..3], skipped while status[0] != 0.
void bf16_spmv_dot2(int n, const int* rows, const int* cols, const unsigned short* v16,
                    const float* scale, const float* p, const float* w, float* q, bool gcr,
                    DeviceReducer red, float* scalars, const int* status, cudaStream_t s);
// inner_first fused with the t.t, b.b reduction -> scalars[4..7].
void inner_first_dot(int n, const float* b, const float* p, const float* q, float* x, float* t,
                     float* scalars, const int* status, DeviceReducer red, cudaStream_t s);
// Dense FP64 Cholesky of an n <= 1024 CSR operator and its explicit inverse
// (n x n, row-major, into `inverse`; `lower` is n x n scratch); *error = 1 if
// the operator is not SPD.
// With `ratio`, also the smallest pivot relative to its diagonal (0 if not SPD).
void dense_inverse(int n, const int* rows, const int* cols, const float* vals, double* lower,
                   double* inverse, double* error, cudaStream_t s, double* ratio = nullptr);
// x = inverse * b (FP64 accumulation).
void dense_solve(int n, const double* inverse, const float* b, float* x, const int* status,
                 cudaStream_t s);
// rf = float(b - A x) with x FP64, ||b - A x||^2 (FP64) into out[slot].
void residual64(int n, const int* rows, const int* cols, const float* vals, const double* x,
                const float* b, float* rf, DeviceReducer red, double* out, int slot,
                cudaStream_t s);
// x += e.
void update64(int n, double* x, const float* e, cudaStream_t s);
// y = double(x), and x = float(y) rounded to nearest: the FP32 form of the
// mixed solve's x.
void widen(int n, const float* x, double* y, cudaStream_t s);
void narrow(int n, const double* y, float* x, cudaStream_t s);

// ---- mixed V-cycle tail: the small coarse levels in one cluster launch ------
// Rows of a tail level are split in power-of-two chunks of (1 << shift) rows,
// chunk k owned by CTA k of the cluster. xg, rg, bg are the level's vectors in
// global memory (the first tail level's b is its input and xg its output).
constexpr int kMaxTailLevels = 8;
constexpr int kTailSharedBytes = 200 * 1024;  // dynamic shared memory per CTA, at most
struct TailLevel {
  int n, shift;  // rows; each CTA owns the rows [rank << shift, (rank + 1) << shift)
  const int* rows;
  const int* cols;
  const unsigned short* v16;
  const float* scale;
  const float* inv;
  // transfer to the next tail level (unused on the coarsest)
  const int* aggregate;
  const int* offsets;
  const int* members;
  float* xg;  // first tail level: the result (global memory)
  float* bg;  // first tail level: the right-hand side (global memory)
  // Float offsets into each CTA's dynamic shared memory: full copies of the
  // iterate and of the spare vector (residual, or the next sweep's iterate),
  // n each, and the owned chunk of the right-hand side (1 << shift).
  int xs, rs, bs;
};
struct TailPlan {
  int levels, pre, post, coarse_sweeps, cluster, smem_bytes;
  const double* dense;     // coarsest dense FP64 inverse, or null for sweeps
  TailLevel level[kMaxTailLevels];
};
// Whether a cluster of `cluster` CTAs (16 or 8) with this much shared memory
// per CTA can run the tail on the current device (sets the kernel's
// shared-memory and cluster-size attributes).
bool tail_cluster_fits(int cluster, int smem_bytes);
// level[0].xg = V-cycle of the tail levels applied to level[0].bg; skipped
// while status[0] != 0.
void tail_cycle(const TailPlan& plan, const int* status, cudaStream_t s);

// ---- learned preconditioner stage (learned.cu) ------------------------------
// Edge weights w_ij = -a_ij / sqrt(a_ii a_jj) (0 on the diagonal), lift_ij =
// w_ij / sqrt(a_jj) and node scales 1 / sqrt(a_ii) from the matrix values.
void gnn_graph(int n, const int* rows, const int* cols, const int* diag, const float* vals,
               float* edge, float* lift, float* node_scale, cudaStream_t s);
// Geometry gate: G_i = sum_j g_ij, rho_ij = log((g_ij / sqrt(G_i G_j)) /
// w_ij) clamped to [-20, 20] (0 where not positive); then E = w gamma and
// lift = lift_w gamma with gamma = exp(theta[0] tanh(theta[1] rho)).
void gnn_geometry(int n, const int* rows, const int* cols, const float* geometry,
                  const float* edge_w, float* G, float* rho, cudaStream_t s);
void gnn_gate(int nnz, const float* edge_w, const float* lift_w, const float* rho,
              const float* theta, float* edge, float* lift, cudaStream_t s);
// dedge_ij (+)= sum_c dM[i][c] H[j][c] (C <= 32 channels).
void gnn_edge_grad(int n, int C, const int* rows, const int* cols, const float* dM,
                   const float* H, float* dedge, bool accumulate, cudaStream_t s);
// fa = dE/dtheta[0], fb = dE/dtheta[1] per edge; grad[0..1] = dots[0..1].
void gnn_gate_factors(int nnz, const float* edge, const float* rho, const float* theta,
                      float* fa, float* fb, cudaStream_t s);
void gnn_store_gate_grad(const double* dots, float* grad, cudaStream_t s);
// H0 = node_scale * r; then H0 /= rho, rho = sqrt(sum2[0] / n) (the RMS of
// H0, reduced on the device in between).
void gnn_input(int n, const float* r, const float* node_scale, float* H0, cudaStream_t s);
void gnn_normalize(int n, float* H0, const double* sum2, cudaStream_t s);
// M = W H for C <= 32 channels (row-major n x C).
void gnn_aggregate(int n, int C, const int* rows, const int* cols, const float* edge,
                   const float* H, float* M, cudaStream_t s);
// out = relu(Ws H + Wn M + b), Cin -> 32 channels.
void gnn_dense(int n, int Cin, const float* H, const float* M, const float* Ws, const float* Wn,
               const float* bias, float* out, cudaStream_t s);
// z = beta z + rho node_scale * (H wo).
void gnn_output(int n, const float* H, const float* wo, const float* node_scale,
                const double* sum2, float* z, float beta, cudaStream_t s);
// Energy loss 1 - P^2 / (Q E) of a correction c for t = A e, dots = {P = c.t,
// Q = c.Ac, E = t.e}, q = A c: dz = dL/dc, loss[0] = L.
void gnn_energy(int n, const float* t, const float* q, const double* dots, float* dz, float* loss,
                cudaStream_t s);
void gnn_output_back(int n, const float* H, const float* wo, const float* node_scale,
                     const double* sum2, const float* dz, float* dH, float* dwo, cudaStream_t s);
void gnn_dense_back(int n, int Cin, const float* H, const float* M, const float* out,
                    const float* dOut, const float* Ws, const float* Wn, float* dH, float* dM,
                    float* dWs, float* dWn, float* db, cudaStream_t s);
void gnn_add(std::size_t count, const float* a, const float* b, float* out, cudaStream_t s);
// The same backward as gnn_dense_back for a 32-wide input (Cin = 32) on the
// tensor cores (learned_tc.cu): [dH | dM] = G [Ws | Wn] per 128-row tile, and
// [dWs^T; dWn^T; db] = [H | M | 1]^T G accumulated in tensor memory, BF16
// operands and FP32 accumulation; dWs, dWn, db are added to (not
// overwritten). partials: gnn_back_partials_floats() floats of scratch;
// *fault is set if a tile's MMA did not complete.
int gnn_back_partials_floats();
void gnn_dense_back_tc(int n, const float* H, const float* M, const float* out,
                       const float* dOut, const float* Ws, const float* Wn, float* dH, float* dM,
                       float* dWs, float* dWn, float* db, float* partials, int* fault,
                       cudaStream_t s);
// z += max(0, dots[0] / dots[1]) c.
void gnn_step(int n, float* z, const float* c, const double* dots, cudaStream_t s);
void gnn_step64(int n, double* x, const float* c, const double* dots, cudaStream_t s);
void gnn_adam(int count, float* w, const float* g, float* m, float* v, float lr, float beta1,
              float beta2, float eps, float correction1, float correction2, cudaStream_t s);

// Tensor-core forward (learned_tc.cu). lift: uv = (s t, sum_j lift_ij t_j),
// sum2[0] = |s t|^2 (fixed-order reduction). layer_a: BF16 rows hout (n x 32)
// = relu([H1 | W H1] [Ws | Wn]^T + b), H1 from uv and the first layer's
// (ws1, wn1, b1) = first[0..95]. layer_b: z = beta z + rho s (wo .
// relu([H | W H] [Ws | Wn]^T + b)) for the BF16 rows hin. A CTA whose MMA
// does not complete sets fault[0] and returns.
void gnn_lift(int n, const int* rows, const int* cols, const float* lift, const float* t,
              const float* node_scale, float2* uv, DeviceReducer red, double* sum2,
              cudaStream_t s);
void gnn_layer_a(int n, const int* rows, const int* cols, const float* edge, const float2* uv,
                 const float* first, const float* ws, const float* wn, const float* bias,
                 const double* sum2, unsigned short* hout, int* fault, long long first_polls,
                 cudaStream_t s);
// first_polls: polls of each tile's first wait for its MMA before the CTA
// gives up (< 0: the built-in bound); the drain wait after giving up always
// takes the full bound, so the MMA completes before tensor memory is freed.
void gnn_layer_b(int n, const int* rows, const int* cols, const float* edge,
                 const unsigned short* hin, const float* ws, const float* wn, const float* bias,
                 const float* wo, const float* node_scale, const double* sum2, float* z,
                 float beta, int* fault, long long first_polls, cudaStream_t s);

// ---- finite-volume steps around the pressure solve (fv_kernels.cu) ---------
// fv_pressure_assemble (fv_flow.kern.h:164-183); the _l1 form also writes
// the rows' inverse L1 diagonal and the max invalid flag into check[slot].
void fv_pressure_assemble(int n, const int* offsets, const int* faces, const float* sign,
                          const int* adjacent, const int* entry, const int* rows, const int* diag,
                          const float* coefficient, const float* flux, float* values, float* rhs,
                          int reference, cudaStream_t s);
void fv_pressure_assemble_l1(int n, const int* offsets, const int* faces, const float* sign,
                             const int* adjacent, const int* entry, const int* rows,
                             const int* diag, const float* coefficient, const float* flux,
                             float* values, float* rhs, int reference, float* inverse,
                             DeviceReducer red, double* check, int slot, cudaStream_t s);
void fv_correct_flux(int n, const int* owner, const int* neighbour, const float* correction,
                     const float* coefficient, float* flux, int internal, cudaStream_t s);
void fv_correct_velocity(int n, const float* volume, const float* inverse, const float* diagonal,
                         const float* gx, const float* gy, const float* gz,
                         const float* correction, float* u, float* v, float* w, float* p,
                         float alpha, cudaStream_t s);

// ---- AMG setup on the device (setup_kernels.cu) -----------------------------
// out[0..n] = exclusive scan of in[0..n) (out[n] = total); block_sums holds
// scan_scratch(n) ints.
void exclusive_scan(int n, const int* in, int* out, int* block_sums, cudaStream_t s);
int scan_scratch(int n);
// flag[0] = 1 if some entry (i, j) has no entry (j, i).
void pattern_symmetric(int n, const int* rows, const int* cols, int* flag, cudaStream_t s);
// Pairing: candidate counts and initial states, preference lists (keys is
// scratch of the same length), and one Jacobi sweep of the greedy pass
// (owner: n ints of scratch; changed[0] = 1 if a row's state moved).
void pair_count(int n, const int* rows, const int* cols, const float* vals, double threshold,
                int exclude_isolated, int* count, int* state, cudaStream_t s);
void pair_fill(int n, const int* rows, const int* cols, const float* vals, double threshold,
               const int* offsets, unsigned long long* keys, int* pref, cudaStream_t s);
void pair_sweep(int n, const int* offsets, const int* pref, int* owner, const int* state,
                int* next, int* changed, cudaStream_t s);
void pair_leaders(int n, const int* state, int* flag, cudaStream_t s);
void pair_assign(int n, const int* state, const int* owner, const int* id, int* aggregate,
                 cudaStream_t s);
// Singleton absorption (mixed hierarchy): sizes, one Jacobi sweep, used marks.
void aggregate_sizes(int n, const int* aggregate, int* size, cudaStream_t s);
void absorb_sweep(int n, const int* rows, const int* cols, const int* diag, const float* vals,
                  double threshold, double coupling, const int* map0, const int* size0,
                  const int* cur, int* next, int* changed, cudaStream_t s);
void mark_used(int n, const int* aggregate, int* used, cudaStream_t s);
// map[i] = table[map[i]] where map[i] >= 0.
void compose(int n, int* map, const int* table, cudaStream_t s);
// Coarse pattern and entry map of an aggregation.
void coarsen_count(int n, const int* rows, const int* cols, const int* aggregate, int* size,
                   int* triples, cudaStream_t s);
void place_members(int n, const int* aggregate, const int* offsets, int* cursor, int* members,
                   cudaStream_t s);
void sort_members(int nc, const int* offsets, int* members, cudaStream_t s);
void coarsen_triples(int nc, const int* rows, const int* cols, const int* aggregate,
                     const int* member_offsets, const int* members, const int* triple_offsets,
                     int m_matrix, int4* triples, int* unique, cudaStream_t s);
void coarsen_fill(int nc, const int* triple_offsets, const int4* triples, const int* coarse_rows,
                  int* coarse_cols, int* coarse_diag, int* entry_offsets, int* entries,
                  cudaStream_t s);

// ---- single-thread scalar kernels -------------------------------------------
void solver_limits(float* scalars, float th, float tl, float dh, float dl, cudaStream_t s);
void solver_reset(float* scalars, int* status, int iterations, cudaStream_t s);
// x -= mean(x) using the pair sum at sum[0..1] (solver_project).
void project(int n, float* x, const float* sum, float count_hi, float count_lo, cudaStream_t s);

// ---- K-cycle inner corrections (amg_inner_*, scalars.kern.h:154-186) --------
// alpha = scalars[2] / scalars[0] -> scalars[8]; first != 0 also restarts the
// level status from the parent's.
void inner_alpha(float* scalars, int* status, const int* parent, int first, cudaStream_t s);
// x = alpha p, t = b - alpha q (running) or x = p, t = 0 (fallback).
void inner_first(int n, const float* b, const float* p, const float* q, float* x, float* t,
                 const float* scalars, const int* status, cudaStream_t s);
void inner_check(const float* scalars, int* status, cudaStream_t s);
// beta = -scalars[4] / scalars[0] -> scalars[10].
void inner_beta(float* scalars, int* status, cudaStream_t s);
// x += alpha p.
void inner_step(int n, float* x, const float* p, const float* scalars, const int* status,
                cudaStream_t s);

}  // namespace launch
}  // namespace kb2
