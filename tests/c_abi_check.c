/* Test infrastructure: a plain C99 caller of include/kutta_b200.h. It checks
 * that the header is C, that the library links from C, and that calls which
 * fail before any device work report their status and message as declared.
 * Prints "ok" and exits 0 on success. */
#include <stdio.h>
#include <string.h>

#include "kutta_b200.h"

static int fail(const char* what) {
  char message[256];
  b2_last_error(message, sizeof message);
  printf("FAILED: %s (last error: %s)\n", what, message);
  return 1;
}

int main(void) {
  b2_options o;
  b2_control c;
  b2_mixed_options m;
  b2_solver* s = NULL;
  char message[256];
  const int32_t row_ptr[3] = {0, 2, 4}, col[4] = {0, 1, 0, 1}, diag[2] = {0, 3};
  const double val[4] = {2.0, -1.0, -1.0, 2.0};

  b2_options_default(&o);
  if (o.cycle != B2_CYCLE_V || o.pre_sweeps != 5 || o.post_sweeps != 5 ||
      o.coarse_sweeps != 32 || o.coarse_rows != 24 || o.max_levels != 24 ||
      o.aggregation_passes != 3 || o.strength_threshold != 0.25 ||
      o.nullspace != B2_NULLSPACE_NONE || o.structure != B2_STRUCTURE_GENERAL ||
      o.workspace != NULL || o.setup != B2_SETUP_DEVICE)
    return fail("b2_options_default");
  b2_control_default(&c);
  if (c.rel_tol != 1e-2 || c.abs_tol != 1e-12 || c.max_iter != 200 ||
      c.residual_check_interval != 8)
    return fail("b2_control_default");
  b2_mixed_options_default(&m);
  if (m.dense_rows != 112 || m.absorb_singletons != 1 || m.amg.cycle != B2_CYCLE_K)
    return fail("b2_mixed_options_default");

  /* make_amg_solver with a Jacobi kind: rejected before any device work. */
  if (b2_solver_create(B2_PCG_JACOBI, 2, 4, row_ptr, col, diag, val, &o, 1, &s) !=
          B2_INVALID_ARGUMENT || s != NULL)
    return fail("kind check");
  b2_last_error(message, sizeof message);
  if (strcmp(message, "AMG: expected an AMG solver kind") != 0) return fail("kind message");

  /* An invalid option, then a CSR error, each with the reference's message. */
  o.aggregation_passes = 9;
  if (b2_solver_create(B2_AMG_PCG, 2, 4, row_ptr, col, diag, val, &o, 1, &s) !=
      B2_INVALID_ARGUMENT)
    return fail("options check");
  b2_last_error(message, sizeof message);
  if (strcmp(message, "AMG: invalid options") != 0) return fail("options message");
  {
    const int32_t bad_diag[2] = {1, 3};
    b2_options_default(&o);
    if (b2_solver_create(B2_AMG_PCG, 2, 4, row_ptr, col, bad_diag, val, &o, 1, &s) !=
        B2_INVALID_ARGUMENT)
      return fail("CSR check");
    b2_last_error(message, sizeof message);
    if (strcmp(message, "CSR: missing or incorrect diagonal") != 0) return fail("CSR message");
  }

  /* Null handles and the empty no-op. */
  if (b2_solver_refresh(NULL, NULL, NULL) != B2_INVALID_ARGUMENT) return fail("null refresh");
  if (b2_mixed_solve_f32(NULL, NULL, NULL, NULL, NULL, NULL, NULL) != B2_INVALID_ARGUMENT)
    return fail("null mixed solve");
  if (b2_csr_spmv(0, 0, NULL, NULL, NULL, NULL, NULL, NULL) != B2_OK) return fail("empty spmv");
  b2_solver_destroy(NULL);
  b2_mixed_destroy(NULL);
  printf("ok\n");
  return 0;
}
