/*
 * kutta_b200: B200-native (sm_100a) pressure-correction linear solve.
 *
 * Plain C ABI. Every entry point takes plain pointers and sizes; device
 * pointers are CUDA device addresses on the current device, host pointers are
 * ordinary host memory. `stream` is a cudaStream_t passed as void* (NULL means
 * the legacy default stream). Every call returns a b2_status; on failure the
 * message is available from b2_last_error() (thread-local).
 *
 * The ABI replaces the reference's C++ linear-solver boundary
 * (src/kutta/linalg/solver.hpp, amg.hpp, csr.hpp); each declaration names the
 * reference interface it stands in for.
 */
#ifndef KUTTA_B200_H
#define KUTTA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. KUTTA's usage errors (KUTTA_REQUIRE -> kutta::Error,
 * src/kutta/core/types.hpp:42-46) map to B2_INVALID_ARGUMENT; nonfinite input
 * vectors (KUTTA_REQUIRE_FINITE -> kutta::NonfiniteError, types.hpp:48-52) map
 * to B2_NONFINITE. Numerical non-convergence is NOT an error: it returns B2_OK
 * with stats.converged = 0, as the reference does (solver.cpp:166-175). */
typedef enum {
  B2_OK = 0,
  B2_INVALID_ARGUMENT = 1,
  B2_NONFINITE = 2,
  B2_DEVICE_ERROR = 3,
  B2_TIMEOUT = 4,
  B2_OUT_OF_MEMORY = 5,
  B2_INTERNAL = 6
} b2_status;

/* SolverKind, src/kutta/linalg/solver.hpp:32-38 (same order and meaning). */
typedef enum {
  B2_JACOBI = 0,
  B2_PCG_JACOBI = 1,
  B2_BICGSTAB_JACOBI = 2,
  B2_AMG_PCG = 3,
  B2_AMG_BICGSTAB = 4
} b2_solver_kind;

/* NullSpace / OperatorStructure, solver.hpp:40-41. AmgCycle, amg.hpp:9. */
typedef enum { B2_NULLSPACE_NONE = 0, B2_NULLSPACE_CONSTANT = 1 } b2_nullspace;
typedef enum { B2_STRUCTURE_GENERAL = 0, B2_STRUCTURE_SYMMETRIC_M_MATRIX = 1 } b2_structure;
typedef enum { B2_CYCLE_V = 0, B2_CYCLE_K = 1 } b2_cycle;
/* Where the AMG hierarchy is built (no reference counterpart; the results are
 * the same bit for bit). B2_SETUP_DEVICE runs the pairing, coarsening and
 * Galerkin product on the GPU when the pattern is structurally symmetric, and
 * falls back to the host setup otherwise. */
typedef enum { B2_SETUP_HOST = 0, B2_SETUP_DEVICE = 1 } b2_setup;

typedef struct b2_workspace b2_workspace;
typedef struct b2_solver b2_solver;
typedef struct b2_hierarchy b2_hierarchy;

/* AmgOptions (amg.hpp:8-20) plus SolverOptions (solver.hpp:66-72) in one
 * struct. `workspace` may be NULL (private Krylov vectors). */
typedef struct {
  int cycle;               /* b2_cycle; default V */
  int pre_sweeps;          /* default 5 */
  int post_sweeps;         /* default 5 */
  int coarse_sweeps;       /* default 32 */
  int coarse_rows;         /* default 24 */
  int max_levels;          /* default 24 */
  int aggregation_passes;  /* default 3 */
  double strength_threshold; /* default 0.25 */
  int nullspace;           /* b2_nullspace; default none */
  int structure;           /* b2_structure; default general */
  b2_workspace* workspace; /* KrylovWorkspace (solver.hpp:47-64) or NULL */
  int setup;               /* b2_setup; default device */
} b2_options;

/* SolveControl, solver.hpp:18-23. */
typedef struct {
  double rel_tol;               /* default 1e-2 */
  double abs_tol;               /* default 1e-12 */
  int max_iter;                 /* default 200 */
  int residual_check_interval;  /* default 8 */
} b2_control;

/* SolveStats, solver.hpp:25-30. */
typedef struct {
  int iterations;
  int converged;
  double initial_residual;
  double final_residual;
} b2_stats;

/* Defaults of AmgOptions{} (amg.hpp:8-20) and SolveControl{} (solver.hpp:18-23). */
void b2_options_default(b2_options* options);
void b2_control_default(b2_control* control);

/* Message of the last failed call on this thread; returns its full length. */
size_t b2_last_error(char* buffer, size_t length);

/* KrylovWorkspace(rows), solver.hpp:47-64: Krylov vectors shared by solvers of
 * one size whose calls never run concurrently. Allocated on first use. */
int b2_workspace_create(int rows, b2_workspace** out);
void b2_workspace_destroy(b2_workspace* workspace);

/* make_solver(kind, dev, a, SolverOptions) (solver.hpp:85-88; amg.cpp:384-406)
 * when options == NULL or `use_amg_options` == 0, make_amg_solver(kind, dev, a,
 * AmgOptions) (amg.hpp:26-27; amg.cpp:345-382) otherwise. The host CSR is the
 * reference's CsrMatrixHost (csr.hpp:16-28): row_ptr[n+1], col[nnz] sorted per
 * row, diag[n] the index of (i,i), val[nnz] as double. The option, CSR,
 * M-matrix, workspace-size and (Jacobi kinds) diagonal checks run on the host
 * before any device work, in the reference's order and with its messages;
 * the hierarchy is then built where options->setup says (B2_SETUP_DEVICE:
 * on the current device, for structurally symmetric patterns). */
int b2_solver_create(int kind, int n, int nnz, const int32_t* row_ptr, const int32_t* col,
                     const int32_t* diag, const double* val, const b2_options* options,
                     int use_amg_options, b2_solver** out);

/* LinearSolver::refresh(dev, a), solver.hpp:77. d_val: the device matrix
 * values (nnz floats, same pattern as at create). */
int b2_solver_refresh(b2_solver* solver, const float* d_val, void* stream);

/* LinearSolver::solve(dev, a, x, b, control), solver.hpp:78-79. d_x holds the
 * initial guess and receives the solution; d_b is the right-hand side; both n
 * floats on the device and not aliased. d_val as for refresh. */
int b2_solver_solve(b2_solver* solver, const float* d_val, float* d_x, const float* d_b,
                    const b2_control* control, b2_stats* stats, void* stream);

/* LinearSolver::describe(), solver.hpp:80. Returns the full length. */
size_t b2_solver_describe(const b2_solver* solver, char* buffer, size_t length);

/* ~LinearSolver(), solver.hpp:76. NULL is accepted. */
void b2_solver_destroy(b2_solver* solver);

/* spmv(dev, a, x, y) and residual(dev, a, x, b, r), csr.hpp:40-48 (kernels
 * csr_spmv / csr_residual, linalg.kern.h:5-50): the same compensated float
 * arithmetic on device CSR arrays. */
int b2_csr_spmv(int n, int nnz, const int32_t* d_row_ptr, const int32_t* d_col,
                const float* d_val, const float* d_x, float* d_y, void* stream);
int b2_csr_residual(int n, int nnz, const int32_t* d_row_ptr, const int32_t* d_col,
                    const float* d_val, const float* d_x, const float* d_b, float* d_r,
                    void* stream);

/* Measurement (no reference counterpart; the reference's bench counts its
 * launches through its InstrumentedDevice, tests/linalg/instrumented_device.hpp).
 * With profiling on, every fine-level smoother sweep of a solve is bracketed by
 * CUDA events on the solve stream, and the algorithmic bytes of every kernel
 * the solve launches are tallied (stored operands, each read or written once). */
typedef struct {
  long long launches;        /* kernels this solver launched since profiling was enabled */
  long long fine_sweeps;     /* fine-level amg_smooth launches timed */
  double fine_sweep_ms;      /* their total device time */
  double fine_sweep_bytes;   /* algorithmic bytes of one fine-level sweep */
  double algorithmic_bytes;  /* all kernels of the profiled solves */
  long long solves;
} b2_profile;
/* Profiling (no reference counterpart): with enable = 1 the solver times its
 * fine-level sweeps with CUDA events and counts its launches and algorithmic
 * bytes until profiling is disabled; b2_solver_profile_read returns the totals. */
int b2_solver_profile(b2_solver* solver, int enable);
int b2_solver_profile_read(b2_solver* solver, b2_profile* out);
/* Process-wide count of kernels launched by this library. */
long long b2_kernel_launches(void);

/* One damped L1-Jacobi sweep (amg_smooth / amg_smooth_zero,
 * src/kutta/kernels/linalg.kern.h:150-170): next = x + (2/3) inv (b - A x). */
int b2_amg_smooth(int n, const int32_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                  const float* d_x, const float* d_b, const float* d_inverse, float* d_next,
                  int zero_start, void* stream);

/* ---- Mixed-precision solve (no reference counterpart) --------------------
 * The same pressure system solved to a tolerance below the FP32 floor: FP64
 * iterative refinement (true residual b - A x and inner products in FP64, the
 * solution kept in FP64) around an inner FP32 PCG whose V-cycle stores the
 * coarse operators in BF16 with symmetric per-row scales and solves the
 * coarsest level with a dense FP64 Cholesky factorisation. The hierarchy
 * pairs rows like the reference's aggregation and lets rows left unpaired join
 * their strongest paired neighbour, so coarsening reaches the dense size. */
typedef struct {
  b2_options amg;            /* cycle (default K), sweeps (default 1,1), threshold,
                                passes, structure (coarse_rows ignored) */
  int absorb_singletons;     /* default 1 */
  int dense_rows;            /* coarsen until a level has <= this many rows (default 112;
                                at most 1024). Up to 236 rows the dense coarsest inverse
                                is formed in one CTA's shared memory; above, by a blocked
                                Cholesky and block inverse over many CTAs (0.66 ms at
                                384 rows, 0.91 ms at 512 on a B200) */
  int coarse_bf16;           /* default 1: levels >= 1 stored as BF16 x row scales */
  double inner_rel_tol;      /* residual reduction per refinement step (default 1e-3) */
  int inner_max_iter;        /* inner PCG iterations per refinement step (default 300) */
  int max_refinements;       /* default 30 */
  int fused_coarse;          /* default 0: 1 runs the coarse levels below 16,384 rows as one
                                thread-block-cluster launch per V-cycle (BF16, no
                                nullspace, below any K-cycle inner steps); with
                                programmatic dependent launch their separate kernels
                                measured faster on the pressure matrices here */
  int k_cycle_levels;        /* with amg.cycle = K: coarse levels 1..k take the inner
                                Krylov step, the rest a V-cycle; 0 = every level
                                (default 1) */
  int cuda_graphs;           /* default 1: each batch of inner iterations between host
                                status checks, and each preconditioner application, is
                                captured once as a CUDA graph and replayed (same kernels,
                                same results); the solve stream may be the legacy default
                                stream, capture uses an internal stream */
  int packed_rows;           /* default 1: the fine level's residual, post-sweep and SpMV
                                read a packed copy of the operator (per row the diagonal
                                and up to 8 off-diagonal values with 16-bit column
                                offsets), the same results bit for bit, rebuilt from the
                                device values at every refresh; used when every row fits.
                                The fine level then follows the values of the last
                                refresh, as the coarse levels always do */
} b2_mixed_options;

typedef struct {
  int refinements;           /* outer FP64 refinement steps */
  int iterations;            /* inner PCG iterations, all steps */
  int converged;
  double initial_residual;   /* ||b - A x0||, FP64 */
  double final_residual;     /* ||b - A x||, FP64, of the returned FP64 x */
  int learned_fallback;      /* 1: a refinement stalled with the learned cycle stage
                                attached, and the solve finished with the AMG cycle
                                alone (the stage stays attached for later solves) */
} b2_mixed_stats;

typedef struct b2_mixed b2_mixed;

/* The defaults listed beside each field above. */
void b2_mixed_options_default(b2_mixed_options* options);
int b2_mixed_create(int n, int nnz, const int32_t* row_ptr, const int32_t* col,
                    const int32_t* diag, const double* val, const b2_mixed_options* options,
                    b2_mixed** out);
int b2_mixed_refresh(b2_mixed* solver, const float* d_val, void* stream);
/* d_x: n doubles, initial guess in, FP64 solution out. d_b: n floats. */
int b2_mixed_solve(b2_mixed* solver, const float* d_val, double* d_x, const float* d_b,
                   const b2_control* control, b2_mixed_stats* stats, void* stream);
/* The same solve with d_x as n floats, the form of LinearSolver::solve
 * (solver.hpp:78-79): d_x is widened into an FP64 copy the solver keeps,
 * solved, and rounded to nearest on return; final_residual is that of the
 * FP64 solution. A rounded x is back at the FP32 floor (about 1e-7 relative
 * on the pressure matrices here), so tighter targets need b2_mixed_solve. */
int b2_mixed_solve_f32(b2_mixed* solver, const float* d_val, float* d_x, const float* d_b,
                       const b2_control* control, b2_mixed_stats* stats, void* stream);
size_t b2_mixed_describe(const b2_mixed* solver, char* buffer, size_t length);
void b2_mixed_destroy(b2_mixed* solver);
/* The mixed solve's coarsest-level step on its own: the dense FP64 Cholesky
 * factorisation of a small SPD CSR operator (n <= 1024) and its explicit
 * inverse, computed in one thread block. d_inverse: n*n doubles, row-major.
 * *d_not_spd (a device double) is written 1.0 if a pivot was not positive,
 * else 0.0. Enqueued on `stream`; the n*n factor scratch is allocated and
 * released stream-ordered (cudaMallocAsync / cudaFreeAsync). */
int b2_dense_inverse(int n, const int32_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                     double* d_inverse, double* d_not_spd, void* stream);

/* b2_dense_inverse for callers that cannot allocate device memory (no
 * counterpart in the reference): hosts that give the solver a fixed device
 * memory budget, real-time loops that must not take the allocator's locks or
 * risk running out of memory mid-step, and work queued while another
 * component records the stream. The same computation, with the n*n factor
 * scratch taken from a 2 MiB array built into the library (so n <= 512; larger
 * n is rejected with B2_INVALID_ARGUMENT). It calls no allocator. Calls with
 * n > 236 factor through the array, which all calls on a device share: such
 * calls that overlap on the GPU race, so the caller orders them. Calls with
 * n <= 236 factor in shared memory and never touch the array. The first call
 * on each device looks the array's address up (and may load the library's
 * device code); make it before any stream capture. A device reset
 * (cudaDeviceReset) can move the array: do not call this entry point on a
 * device after resetting it. */
int b2_dense_inverse_noalloc(int n, const int32_t* d_row_ptr, const int32_t* d_col,
                             const float* d_val, double* d_inverse, double* d_not_spd,
                             void* stream);

/* As b2_solver_profile / _read, for the inner solve plus the FP64 refinement. */
int b2_mixed_profile(b2_mixed* solver, int enable);
int b2_mixed_profile_read(b2_mixed* solver, b2_profile* out);
/* Host-only mixed hierarchy (as b2_hierarchy_build). */
int b2_mixed_hierarchy_build(int n, int nnz, const int32_t* row_ptr, const int32_t* col,
                             const int32_t* diag, const double* val,
                             const b2_mixed_options* options, b2_hierarchy** out);

/* ---- Learned preconditioner stage (no reference counterpart) --------------
 * A message-passing network over the graph of the fine matrix (3 layers,
 * hidden width 32; edge features w_ij = -a_ij / sqrt(a_ii a_jj), node scale
 * 1 / sqrt(a_ii)) mapping a residual r to a correction direction G(r). The
 * input is normalised by its RMS and the output scaled back, so
 * G(lambda r) = lambda G(r) for lambda > 0. Trained with b2_gnn_train_step on
 * (residual t, error e) pairs with A e = t, one Adam step per call, on the
 * energy loss 1 - (c.t)^2 / ((c.Ac)(t.e)) for c = G(t): the fraction of the
 * error's A-energy left after the best step along c. */
typedef struct b2_gnn b2_gnn;
/* A stage with weights drawn from `seed`; b2_gnn_set_weights loads trained
 * ones (b2_gnn_parameter_count floats; the count without the geometry gate's
 * two parameters is accepted too, giving theta = (0, 0.25): a gate of 1). */
int b2_gnn_create(uint64_t seed, b2_gnn** out);
void b2_gnn_destroy(b2_gnn* g);
int b2_gnn_parameter_count(void);
/* Binds the graph of a device CSR matrix (n rows); keep the arrays alive while
 * bound and bind again after its values change. */
int b2_gnn_bind(b2_gnn* g, int n, const int32_t* d_row_ptr, const int32_t* d_col,
                const int32_t* d_diag, const float* d_val, void* stream);
/* The geometry of the matrices bound from now on (takes effect at the next
 * bind, including a mixed solver's refresh): d_geometry holds, per entry of
 * the bound CSR pattern, the face's geometric coefficient |A_f| / |c_N - c_P|
 * (0 on the diagonal), or is NULL for none. Each edge weight w_ij is then
 * gated, E_ij = w_ij exp(theta_0 tanh(theta_1 rho_ij)) with rho_ij =
 * log((g_ij / sqrt(G_i G_j)) / w_ij), G_i = sum_j g_ij: an edge feature from
 * the face coefficient and the geometry, theta the last two weights. Keep the
 * array alive while bound. */
int b2_gnn_set_geometry(b2_gnn* g, const float* d_geometry);
/* d_z = beta d_z + G(d_r), beta 0 or 1: the tensor-core forward (BF16
 * operands, FP32 accumulation); waits for the stream to report a device
 * fault of the stage. */
int b2_gnn_apply(b2_gnn* g, const float* d_r, float* d_z, float beta, void* stream);
/* Testing hook for the forward's bounded waits: each tensor-core tile polls
 * its MMA's completion at most `polls` times (polls < 0 restores the built-in
 * bound, 4,194,304) before its block gives up. A block that gives up records
 * the fault, waits for its MMA once more with the full bound, frees its
 * tensor memory and returns; b2_gnn_apply then returns B2_TIMEOUT and clears
 * the fault. polls = 0 takes that path with a healthy MMA. */
int b2_gnn_set_wait_limit(b2_gnn* g, long long polls);
/* One training step on (d_t, d_e), A e = t for the bound matrix; *loss is the
 * energy loss before the step. The forward keeps FP32 activations; in the
 * backward the two 32-wide layers' products ([dH | dM] = G [Ws | Wn] and the
 * weight gradients [H | M | 1]^T G) run on the tensor cores (BF16 operands,
 * FP32 accumulation), then one Adam step. */
int b2_gnn_train_step(b2_gnn* g, const float* d_t, const float* d_e, float learning_rate,
                      float* loss, void* stream);
/* The energy loss's gradient with respect to the b2_gnn_parameter_count()
 * weights at their current values, for (d_t, d_e) as in b2_gnn_train_step,
 * without a step: tensor_cores = 1 computes the 32-wide layers' backward as
 * b2_gnn_train_step does, 0 in FP32 on CUDA cores. *loss (may be NULL)
 * receives the loss. */
int b2_gnn_gradient(b2_gnn* g, const float* d_t, const float* d_e, int tensor_cores,
                    float* host_gradient, size_t count, float* loss, void* stream);
int b2_gnn_get_weights(const b2_gnn* g, float* host, size_t count);
int b2_gnn_set_weights(b2_gnn* g, const float* host, size_t count);
/* Attaches g (NULL detaches) to a mixed solver; it is bound to the solver's
 * matrix at once if refreshed, and again at every refresh. g must outlive the
 * attachment. `mode` is a bit set:
 *   B2_LEARNED_CYCLE: after each AMG cycle, with z = M(r), t = r - A z and
 *     c = G(t), z += alpha c for the energy-minimising alpha =
 *     max(0, c.t / c.Ac), so the stage never makes the error larger in the
 *     A-norm (the flexible inner PCG absorbs the variable preconditioner);
 *   B2_LEARNED_WARM_START: before the refinement loop, the initial guess x0
 *     takes a safeguarded step along c = G(r), r = b - A x0, of the length
 *     max(0, r.Ac / Ac.Ac) that minimises the new residual (the solve stops
 *     on the residual), so the warm start never raises it. */
#define B2_LEARNED_CYCLE 1
#define B2_LEARNED_WARM_START 2
int b2_mixed_set_learned(b2_mixed* solver, b2_gnn* g, int mode);
/* One application of the mixed solver's preconditioner (the AMG cycle, and
 * the learned stage when attached in B2_LEARNED_CYCLE mode) to d_r, into d_z,
 * with the values d_val the solver was refreshed with. */
int b2_mixed_precondition(b2_mixed* solver, const float* d_val, const float* d_r, float* d_z,
                          void* stream);

/* ---- Finite-volume steps around the pressure solve --------------------------
 * The reference's kernels on either side of the solve, same arguments and
 * the same float results bit for bit (src/kutta/kernels/fv_flow.kern.h:
 * 164-201; called at src/kutta/fv/steady_solver.cpp:1334, 1345, 1364). All
 * arrays are device pointers; cell-face slots run over offsets[n_cells].
 *   fv_pressure_assemble: row i of the pressure-correction matrix (values in
 *     the CSR pattern rows/diag, entry[j] the position of (i, adjacent[j]))
 *     and rhs[i], from per-face coefficients and mass fluxes; `reference` is
 *     an eliminated cell (unit row, column removed) or -1.
 *   fv_correct_flux: flux[f] += coefficient[f] (p'_owner - p'_neighbour) for
 *     the n_faces faces (neighbour read for f < internal only).
 *   fv_correct_velocity: u, v, w -= volume inverse grad p'; p += min(alpha,
 *     0.7 diagonal inverse) p'. */
int b2_fv_pressure_assemble(int n_cells, const int32_t* d_offsets, const int32_t* d_faces,
                            const float* d_sign, const int32_t* d_adjacent, const int32_t* d_entry,
                            const int32_t* d_row_ptr, const int32_t* d_diag,
                            const float* d_coefficient, const float* d_flux, float* d_values,
                            float* d_rhs, int reference, void* stream);
int b2_fv_correct_flux(int n_faces, const int32_t* d_owner, const int32_t* d_neighbour,
                       const float* d_correction, const float* d_coefficient, float* d_flux,
                       int internal, void* stream);
int b2_fv_correct_velocity(int n_cells, const float* d_volume, const float* d_inverse,
                           const float* d_diagonal, const float* d_gx, const float* d_gy,
                           const float* d_gz, const float* d_correction, float* d_u, float* d_v,
                           float* d_w, float* d_p, float alpha, void* stream);
/* fv_pressure_assemble fused with the solver's refresh: one pass over the
 * cells writes the matrix values (into d_values, the solver's pattern), the
 * right-hand side and the fine level's L1 inverse diagonal; the coarse levels
 * then refresh as b2_solver_refresh / b2_mixed_refresh does. d_values is the
 * matrix to pass to the next solve. AMG solvers only. */
int b2_solver_assemble_refresh(b2_solver* solver, const int32_t* d_offsets,
                               const int32_t* d_faces, const float* d_sign,
                               const int32_t* d_adjacent, const int32_t* d_entry,
                               const float* d_coefficient, const float* d_flux, float* d_values,
                               float* d_rhs, int reference, void* stream);
int b2_mixed_assemble_refresh(b2_mixed* solver, const int32_t* d_offsets, const int32_t* d_faces,
                              const float* d_sign, const int32_t* d_adjacent,
                              const int32_t* d_entry, const float* d_coefficient,
                              const float* d_flux, float* d_values, float* d_rhs, int reference,
                              void* stream);

/* Hierarchy introspection (the captured-hierarchy checks of the reference's
 * tests/linalg/test_solvers.cpp:487-555 read the same data back from launches).
 * Level 0 is the input matrix. Copies are synchronous device-to-host reads on
 * `stream`; any output pointer may be NULL. */
int b2_solver_levels(const b2_solver* solver);
int b2_solver_level_shape(const b2_solver* solver, int level, int* n, int* nnz);
int b2_solver_level_copy(const b2_solver* solver, int level, int32_t* row_ptr, int32_t* col,
                         float* val, float* inverse_l1, int32_t* aggregate, void* stream);
/* The level's diagonal positions diag[n] and its transfer to level + 1 (none
 * on the coarsest): member_offsets[n_c + 1], members (at most n), entry_offsets
 * [nnz_c + 1] and entries (at most nnz), the last two the Galerkin entry map
 * (coarse entry e sums the level's entries entries[entry_offsets[e] ..
 * entry_offsets[e+1])). Synchronous reads on `stream`; any pointer may be NULL. */
int b2_solver_level_transfer(const b2_solver* solver, int level, int32_t* diag,
                             int32_t* member_offsets, int32_t* members, int32_t* entry_offsets,
                             int32_t* entries, void* stream);

/* Host-only AMG setup (no GPU needed): the aggregation hierarchy that
 * b2_solver_create builds (Aggregation ctor, amg.cpp:200-226: pairs :25-75,
 * coarsen :77-158, aggregate :160-174). Levels as above; values are the
 * host-assembled coarse operators and L1 inverse diagonals. */
int b2_hierarchy_build(int n, int nnz, const int32_t* row_ptr, const int32_t* col,
                       const int32_t* diag, const double* val, const b2_options* options,
                       int spd, b2_hierarchy** out);
int b2_hierarchy_levels(const b2_hierarchy* h);
int b2_hierarchy_level_shape(const b2_hierarchy* h, int level, int* n, int* nnz);
int b2_hierarchy_level_copy(const b2_hierarchy* h, int level, int32_t* row_ptr, int32_t* col,
                            float* val, float* inverse_l1, int32_t* aggregate);
void b2_hierarchy_free(b2_hierarchy* h);

/* ---- Coupled (4x4-block) pressure-velocity solve ---------------------------
 * kutta::fv::CoupledSolver (src/kutta/fv/coupled_solver.hpp:61-101): momentum
 * and continuity in one block system per outer iteration, solved in delta
 * form by block BiCGStab with a block aggregation-AMG V-cycle (damped block
 * Jacobi smoothing). Unknowns per cell: (du, dv, dw, dp~), dp~ = dp / wc,
 * wc = density x velocity_scale.
 *
 * The reference's constructor takes its DeviceMesh, Stencil, PolyMesh,
 * MeshGeometry, boundary kinds and pressure least-squares fit
 * (coupled_solver.hpp:69-74); b2_coupled_mesh carries the arrays of those it
 * reads, as HOST arrays (setup runs on the host, as the reference's does). */
typedef struct {
  int n_cells, n_faces, n_internal;  /* internal faces first, owner < neighbour */
  const int32_t* owner;              /* n_faces */
  const int32_t* neighbour;          /* n_internal */
  const int32_t* cell_face_offsets;  /* n_cells + 1: DeviceMesh::cell_face_offsets */
  const int32_t* cell_faces;         /* per entry */
  const float* cell_face_sign;       /* per entry: +1 owner, -1 neighbour */
  const int32_t* adjacent;           /* per entry: Stencil::adjacent (other cell or
                                        -(boundary face + 1)) */
  const float *area_x, *area_y, *area_z;  /* n_faces: DeviceMesh::area */
  const double* face_area;           /* 3 n_faces, (x, y, z) per face: MeshGeometry */
  const double* cell_centroid;       /* 3 n_cells: MeshGeometry */
  const float *owner_to_face_x, *owner_to_face_y, *owner_to_face_z;  /* n_faces */
  const float *neighbour_to_face_x, *neighbour_to_face_y,
      *neighbour_to_face_z;          /* n_internal */
  const float *lsq_x, *lsq_y, *lsq_z;  /* per entry: BoundaryLeastSquares::rows() */
  const float *boundary_delta_x, *boundary_delta_y,
      *boundary_delta_z;             /* per boundary face: ::boundary_delta */
  const float* lsq_inverse;          /* 6 n_cells planes (xx xy xz yy yz zz):
                                        ::inverse_values() */
  const float* diffusion;            /* n_faces: Stencil::diffusion */
  const float* volume;               /* n_cells: DeviceMesh::volume */
  const int32_t* boundary_kind;      /* per boundary face: fv_flow.kern.h:3-4 */
  const int32_t* pattern_row_ptr;    /* Stencil::pattern (the momentum rows' CSR */
  const int32_t* pattern_col;        /* pattern, diagonal included) */
  const int32_t* pattern_diag;
  const int32_t* low_order;          /* n_cells flags (low-order pressure faces) or NULL */
} b2_coupled_mesh;

/* CoupledOptions, coupled_solver.hpp:26-38. recompute selects the reference's
 * memory-limited operator (CoupledEdgeStorage::Recompute); its results equal
 * the cached operator's, and this library always caches. */
typedef struct {
  int pre_sweeps, post_sweeps, coarsest_sweeps; /* defaults 1, 2, 8 */
  float smoother_damping;                       /* default 0.7 */
  double courant;                               /* default 200 */
  int coarsest_rows;                            /* default 48 */
  int aggregation_passes;                       /* default 3 */
  int recompute;                                /* default 0 */
} b2_coupled_options;

/* CoupledResiduals, coupled_solver.hpp:41-55: device arrays. d_net_outflow
 * may be NULL (the net outflow is then summed from d_mass). */
typedef struct {
  const float *d_ru, *d_rv, *d_rw;  /* momentum residuals b - A u, n_cells each */
  const float* d_mass;              /* n_faces, kg/s out of owner */
  const float* d_viscosity;         /* n_faces */
  const float* d_physical_diagonal; /* n_cells */
  const float* d_face_weights;      /* n_cells */
  const float* d_net_outflow;       /* n_cells or NULL */
  double density, velocity_scale;
} b2_coupled_residuals;

typedef struct b2_coupled b2_coupled;
typedef struct b2_coupled_setup b2_coupled_setup;

void b2_coupled_options_default(b2_coupled_options* options);
/* CoupledSolver::CoupledSolver (coupled_solver.cpp:464-470). reference >= 0
 * anchors a closed domain's pressure in that cell. Host arrays are read
 * during the call only. */
int b2_coupled_create(const b2_coupled_mesh* mesh, int reference,
                      const b2_coupled_options* options, void* stream, b2_coupled** out);
/* CoupledSolver::capture_diagonal (coupled_solver.cpp:472-477): one momentum
 * component's assembled CSR (device, over the stencil pattern) and its
 * physical diagonal (device, n_cells). */
int b2_coupled_capture_diagonal(b2_coupled* solver, int component, const int32_t* d_row_ptr,
                                const int32_t* d_diag, const float* d_val,
                                const float* d_physical, void* stream);
/* CoupledSolver::solve (coupled_solver.cpp:479-512): assembles the Jacobian and
 * right-hand side, then solves for the update; stats as SolveStats. */
int b2_coupled_solve(b2_coupled* solver, const b2_coupled_residuals* residuals,
                     const b2_control* control, b2_stats* stats, void* stream);
/* CoupledSolver::update (coupled_solver.cpp:514-522): u += alpha_u du,
 * p += alpha_p wc dp~, then the closed-domain gauge. Device arrays. */
int b2_coupled_update(b2_coupled* solver, float* d_u, float* d_v, float* d_w, float* d_p,
                      double alpha_u, double alpha_p, void* stream);
/* The float-pair form (coupled_solver.cpp:524-535, CoupledPairs). */
int b2_coupled_paired_update(b2_coupled* solver, float* d_u, float* d_v, float* d_w, float* d_p,
                             float* d_u_lo, float* d_v_lo, float* d_w_lo, float* d_p_lo,
                             double alpha_u, double alpha_p, float velocity_slack,
                             float pressure_slack, void* stream);
/* CoupledSolver::bytes / describe (coupled_solver.cpp:537-546). */
size_t b2_coupled_bytes(const b2_coupled* solver);
size_t b2_coupled_describe(const b2_coupled* solver, char* buffer, size_t length);
void b2_coupled_destroy(b2_coupled* solver);

/* Introspection of the last solve, synchronous reads on `stream` into host
 * arrays (any pointer may be NULL). what: 0 the solution, 1 the right-hand
 * side (each 4 n_cells floats as planes [u | v | w | p~]), 2 the cell data
 * (27 n_cells floats, the reference's packed planes: du dv dw cd | G | H |
 * Q | cs | iu iv iw hx iu hy iv hz iw schur), 3 the face coefficients
 * (n_faces). Returns the float count. */
long long b2_coupled_copy(const b2_coupled* solver, int what, float* out, void* stream);
/* Levels (the fine level is 0) and a coarse level's operator: rows[n + 1],
 * cols[nnz], diag[n], a[nnz], c[nnz], g[3 nnz], h[3 nnz], d[11 n], and the
 * aggregate of each row of level - 1 (level - 1 rows). */
int b2_coupled_levels(const b2_coupled* solver);
int b2_coupled_level_shape(const b2_coupled* solver, int level, int* n, int* nnz);
int b2_coupled_level_copy(const b2_coupled* solver, int level, int32_t* rows, int32_t* cols,
                          int32_t* diag, float* a, float* c, float* g, float* h, float* d,
                          int32_t* aggregate, void* stream);
/* The fine block operator on device vectors of float4 per cell (u, v, w, p~):
 * op 0 y = J x, 1 y = b - J x, 2 one damped block-Jacobi sweep from x, 3 the
 * same from x = 0 (x not read). Uses the Jacobian of the last solve. */
int b2_coupled_apply(b2_coupled* solver, int op, const float* d_x, const float* d_b, float* d_y,
                     void* stream);

/* The same on coarse level `level` >= 1 (float4 per coarse row): op 1 y =
 * b - J x, 2 / 3 one sweep from x / from x = 0; op 4 y = the restriction of
 * level - 1's x (member sums), op 5 y += the prolongation of x to level - 1
 * (y has level - 1 rows). */
int b2_coupled_level_apply(b2_coupled* solver, int level, int op, const float* d_x,
                           const float* d_b, float* d_y, void* stream);

/* Host-only Coupled setup (no GPU needed): the pressure-force sensitivities
 * and the aggregation hierarchy b2_coupled_create builds
 * (coupled_solver.cpp:27-46 pair_rows, :49-85 members_of and contract, :132-289). */
int b2_coupled_setup_build(const b2_coupled_mesh* mesh, const b2_coupled_options* options,
                           b2_coupled_setup** out);
int b2_coupled_setup_levels(const b2_coupled_setup* setup);
int b2_coupled_setup_level_shape(const b2_coupled_setup* setup, int level, int* n, int* nnz);
/* Level >= 1: rows, cols, diag; every level but the coarsest: its aggregate
 * (level rows), member offsets (next level rows + 1) and members. */
int b2_coupled_setup_level_copy(const b2_coupled_setup* setup, int level, int32_t* rows,
                                int32_t* cols, int32_t* diag, int32_t* aggregate,
                                int32_t* member_offsets, int32_t* members);
/* 27 n_cells floats: G in planes 4-6, Q in planes 10-18, zero elsewhere. */
int b2_coupled_setup_cell(const b2_coupled_setup* setup, float* out);
int b2_coupled_setup_width(const b2_coupled_setup* setup);
void b2_coupled_setup_free(b2_coupled_setup* setup);

#ifdef __cplusplus
}
#endif
#endif /* KUTTA_B200_H */
