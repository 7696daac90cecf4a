/*
 * TEST INFRASTRUCTURE (the oracle). A CPU restatement, in C, of the reference's
 * pressure-solve path: aggregation-AMG setup and refresh, the V-cycle, the
 * Krylov drivers with float-pair device scalars, serial FP64 reductions, plus
 * an FP64 CG oracle. Parity: pinned bit-for-bit against the reference's own CPU
 * path built from its sources (oracle/_ref) and against the golden fixtures in
 * tests/golden/. Only tests, __graft_entry__.smoke() and bench.py's CPU
 * baseline may load it; the product never does.
 */
#ifndef KUTTA_ORACLE_H
#define KUTTA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int kind;          /* 0 Jacobi, 1 PcgJacobi, 2 BicgstabJacobi, 3 AmgPcg, 4 AmgBicgstab */
  int cycle;         /* 0 V (K is not restated) */
  int pre_sweeps, post_sweeps, coarse_sweeps, coarse_rows, max_levels, passes;
  double threshold;
  int nullspace;     /* 1: constant nullspace */
  int m_matrix;      /* 1: SymmetricMMatrix */
  int absorb;        /* 1: singleton absorption (the mixed solve's hierarchy) */
} ko_options;

typedef struct { double rel_tol, abs_tol; int max_iter, interval; } ko_control;
typedef struct { int iterations, converged; double initial_residual, final_residual; } ko_stats;

typedef struct ko_solver ko_solver;

/* make_solver / make_amg_solver; NULL on error (message in err). */
ko_solver* ko_create(int n, int nnz, const int* row_ptr, const int* col, const int* diag,
                     const double* val, const ko_options* o, char* err, int errlen);
/* LinearSolver::refresh with float device values; 0 or -1 (message in err). */
int ko_refresh(ko_solver* s, const float* val, char* err, int errlen);
/* LinearSolver::solve; x in/out. 0, -1 (Error) or -2 (NonfiniteError). */
int ko_solve(ko_solver* s, const float* val, float* x, const float* b, const ko_control* c,
             ko_stats* st, char* err, int errlen);
int ko_describe(const ko_solver* s, char* out, int len);
int ko_levels(const ko_solver* s);
void ko_level_shape(const ko_solver* s, int level, int* n, int* nnz);
void ko_level_copy(const ko_solver* s, int level, int* row_ptr, int* col, float* val, float* l1,
                   int* aggregate);
void ko_destroy(ko_solver* s);

/* Kernel restatements (one call = one launch over all indices). */
void ko_spmv(int n, const int* rows, const int* cols, const float* vals, const float* x, float* y);
void ko_residual(int n, const int* rows, const int* cols, const float* vals, const float* x,
                 const float* b, float* r);
void ko_smooth(int n, const int* rows, const int* cols, const float* vals, const float* x,
               const float* b, const float* inv, float* next, const int* status, int zero_start);
void ko_coarse_solve(const int* rows, const int* cols, const float* vals, float* x,
                     const float* b, const float* inv, const int* status, int count, int sweeps);
void ko_diagonal(int n, const int* rows, const int* diag, const float* vals, float* inverse,
                 float* invalid, int use_l1);
void ko_restrict(int nc, const int* offsets, const int* members, const float* fine, float* coarse);
void ko_prolong(int nf, const int* aggregate, const float* coarse, float* fine);
void ko_galerkin(int nnz_c, const int* offsets, const int* entries, const float* fine, float* coarse);
/* Scalar kernels by name index: 0 pcg_alpha, 1 pcg_beta, 2 pcg_beta flexible,
 * 3 bicg_beta, 4 bicg_alpha, 5 bicg_s, 6 bicg_omega, 7 check pcg, 8 check bicg,
 * 9 reset (arg = iterations). */
void ko_scalar(int op, float* scalars, int* status, int arg);
void ko_solver_step(int n, float* x, float* r, const float* p, const float* q,
                    const float* scalars, const int* status);

/* Finite-volume steps around the pressure solve, src/kutta/kernels/
 * fv_flow.kern.h: fv_pressure_assemble (:164-183), fv_correct_flux (:185-190),
 * fv_correct_velocity (:192-201). */
void ko_fv_pressure_assemble(int n, const int* offsets, const int* faces, const float* sign,
                             const int* adjacent, const int* entry, const int* rows,
                             const int* diag, const float* coefficient, const float* flux,
                             float* values, float* rhs, int reference);
void ko_fv_correct_flux(int n, const int* owner, const int* neighbour, const float* correction,
                        const float* coefficient, float* flux, int internal);
void ko_fv_correct_velocity(int n, const float* volume, const float* inverse,
                            const float* diagonal, const float* gx, const float* gy,
                            const float* gz, const float* correction, float* u, float* v,
                            float* w, float* p, float alpha);

/* FP64 oracle: CG in double on the double-valued matrix, multi-threaded, from
 * x = 0 to ||b - A x|| <= rel_tol ||b||. Returns iterations, or -1. */
int ko_cg64(int n, const int* row_ptr, const int* col, const double* val, const double* b,
            double* x, double rel_tol, int max_iter, int threads);
/* ||b - A x||_2 in double for a float x (the true residual). */
double ko_true_residual(int n, const int* row_ptr, const int* col, const double* val,
                        const double* b, const float* x);

#ifdef __cplusplus
}
#endif
#endif
