/*
 * TEST INFRASTRUCTURE (the oracle): CPU restatement in C of the reference's
 * pressure-solve path. See kutta_oracle.h. Every function cites the reference
 * file:line (paths within the reference project) whose algorithm it restates.
 * Compiled with -ffp-contract=off so float expressions round as written, like
 * the reference's CPU build; the only fused multiply-add is the explicit fmaf of
 * the pair product (src/kutta/kernels/scalars.kern.h:18-22).
 */
#include "kutta_oracle.h"

#include <math.h>
#include <setjmp.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------ errors ---- */
static __thread jmp_buf* g_jump;
static __thread char g_msg[512];
static __thread int g_code;
static void fail(int code, const char* msg) {
  g_code = code;
  snprintf(g_msg, sizeof g_msg, "%s", msg);
  longjmp(*g_jump, 1);
}
#define REQUIRE(c, m) do { if (!(c)) fail(-1, m); } while (0)

static void* xmalloc(size_t bytes) {
  void* p = malloc(bytes ? bytes : 1);
  if (!p) fail(-1, "oracle: out of memory");
  return p;
}
static void* xcalloc(size_t n, size_t s) {
  void* p = calloc(n ? n : 1, s ? s : 1);
  if (!p) fail(-1, "oracle: out of memory");
  return p;
}

/* ------------------------------------------------- prelude arithmetic ---- */
/* kadd_up / kupper_sum, src/kutta/kernels/prelude.h:82-100. */
static float add_up(float a, float b) {
  float sum = a + b, part = sum - a;
  float error = (a - (sum - part)) + (b - part);
  return error > 0.0f ? nextafterf(sum, INFINITY) : sum;
}
typedef struct { float sum, error; } upper;
static upper upper_add(upper a, float b) {
  float sum = a.sum + b, part = sum - a.sum;
  float error = (a.sum - (sum - part)) + (b - part);
  upper r = {sum, add_up(a.error, error)};
  return r;
}
static float upper_value(upper a) { return add_up(a.sum, a.error); }

/* Float-pair scalars, src/kutta/kernels/scalars.kern.h:3-42. */
typedef struct { float hi, lo; } pair;
static pair kp(float hi, float lo) { pair p = {hi, lo}; return p; }
static pair kp_load(const float* p, int o) { return kp(p[o], p[o + 1]); }
static pair kp_add(pair a, pair b) {
  float s = a.hi + b.hi;
  if (s - s != 0.0f) return kp(s, 0.0f);
  float v = s - a.hi;
  float e = (a.hi - (s - v)) + (b.hi - v);
  e = e + a.lo + b.lo;
  float h = s + e;
  return kp(h, e - (h - s));
}
static pair kp_neg(pair a) { return kp(-a.hi, -a.lo); }
static pair kp_mul(pair a, pair b) {
  float h = a.hi * b.hi;
  float l = fmaf(a.hi, b.hi, -h) + a.hi * b.lo + a.lo * b.hi;
  return kp_add(kp(h, 0.0f), kp(l, 0.0f));
}
static pair kp_div(pair a, pair b) {
  float q = a.hi / b.hi;
  pair r = kp_add(a, kp_neg(kp_mul(kp(q, 0.0f), b)));
  return kp_add(kp(q, 0.0f), kp((r.hi + r.lo) / b.hi, 0.0f));
}
static void kp_store(float* out, int o, pair p) { out[o] = p.hi; out[o + 1] = p.lo; }
static float kp_float(pair a) { return a.hi + a.lo; }
static int kp_positive(pair a) { return a.hi > 0.0f || (a.hi == 0.0f && a.lo > 0.0f); }
static int kp_finite(pair a) { return a.hi - a.hi == 0.0f && a.lo - a.lo == 0.0f; }
static int kp_zero(pair a) { return a.hi == 0.0f && a.lo == 0.0f; }
static int kp_le(pair a, pair b) { return a.hi < b.hi || (a.hi == b.hi && a.lo <= b.lo); }
static int kp_coefficient(pair a) {
  float v = kp_float(a);
  return kp_finite(a) && v - v == 0.0f && (v != 0.0f || kp_zero(a));
}

/* ---------------------------------------------------------- kernels ---- */
/* csr_spmv, src/kutta/kernels/linalg.kern.h:5-16. */
void ko_spmv(int n, const int* rows, const int* cols, const float* vals, const float* x, float* y) {
  for (int i = 0; i < n; ++i) {
    float sum = 0.0f, error = 0.0f;
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      float term = vals[j] * x[cols[j]] - error;
      float next = sum + term;
      error = (next - sum) - term;
      sum = next;
    }
    y[i] = sum;
  }
}
/* csr_product_error, linalg.kern.h:21-30. */
static float product_error(float a, float b, float product) {
  if (fabsf(a) > 1.0e30f || fabsf(b) > 1.0e30f) return 0.0f;
  float ca = 4097.0f * a, cb = 4097.0f * b;
  float ah = ca - (ca - a), bh = cb - (cb - b);
  float al = a - ah, bl = b - bh;
  return ((ah * bh - product) + ah * bl + al * bh) + al * bl;
}
/* csr_row_residual, linalg.kern.h:32-45. */
static float row_residual(int i, const int* rows, const int* cols, const float* vals,
                          const float* x, const float* b) {
  float sum = b[i], error = 0.0f;
  for (int j = rows[i]; j < rows[i + 1]; ++j) {
    float product = vals[j] * x[cols[j]];
    float term = -product;
    float next = sum + term;
    error += fabsf(sum) >= fabsf(term) ? (sum - next) + term : (term - next) + sum;
    error -= product_error(vals[j], x[cols[j]], product);
    sum = next;
  }
  return sum + error;
}
/* csr_residual, linalg.kern.h:47-50. */
void ko_residual(int n, const int* rows, const int* cols, const float* vals, const float* x,
                 const float* b, float* r) {
  for (int i = 0; i < n; ++i) r[i] = row_residual(i, rows, cols, vals, x, b);
}
/* amg_smooth :150-156 and amg_smooth_zero :162-170 (x is the cleared vector). */
void ko_smooth(int n, const int* rows, const int* cols, const float* vals, const float* x,
               const float* b, const float* inv, float* next, const int* status, int zero_start) {
  if (status[0] != 0) return;
  for (int i = 0; i < n; ++i) {
    if (zero_start && !(b[i] - b[i] != 0.0f)) {
      next[i] = 0.0f + (2.0f / 3.0f) * inv[i] * (b[i] + 0.0f);
      continue;
    }
    float r = row_residual(i, rows, cols, vals, x, b);
    next[i] = x[i] + (2.0f / 3.0f) * inv[i] * r;
  }
}
/* amg_coarse_solve, linalg.kern.h:126-147. */
void ko_coarse_solve(const int* rows, const int* cols, const float* vals, float* x,
                     const float* b, const float* inv, const int* status, int count, int sweeps) {
  if (status[0] != 0) return;
  float current[24], r[24];
  for (int row = 0; row < count; ++row) current[row] = 0.0f;
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    for (int row = 0; row < count; ++row) r[row] = row_residual(row, rows, cols, vals, current, b);
    for (int row = 0; row < count; ++row) current[row] += (2.0f / 3.0f) * inv[row] * r[row];
  }
  for (int row = 0; row < count; ++row) x[row] = current[row];
}
/* krylov_diagonal, linalg.kern.h:52-70. */
void ko_diagonal(int n, const int* rows, const int* diag, const float* vals, float* inverse,
                 float* invalid, int use_l1) {
  for (int i = 0; i < n; ++i) {
    float d = vals[diag[i]], off = 0.0f, bad = 0.0f;
    for (int j = rows[i]; j < rows[i + 1]; ++j) {
      float v = vals[j];
      if (v - v != 0.0f) bad = 1.0f;
      if (j != diag[i]) off += fabsf(v);
    }
    float inv = d != 0.0f ? 1.0f / d : 0.0f;
    float l1 = fmaxf(fabsf(d), 0.5f * (fabsf(d) + off));
    inverse[i] = use_l1 != 0 ? (l1 != 0.0f ? 1.0f / l1 : 0.0f) : inv;
    invalid[i] = (bad != 0.0f || inv - inv != 0.0f || l1 - l1 != 0.0f)
                     ? 2.0f : (use_l1 != 0 && d < 0.0f ? 3.0f : (d == 0.0f ? 1.0f : 0.0f));
  }
}
/* amg_restrict, src/kutta/kernels/amg.kern.h:5-16. */
void ko_restrict(int nc, const int* offsets, const int* members, const float* fine, float* coarse) {
  for (int g = 0; g < nc; ++g) {
    float sum = 0.0f, error = 0.0f;
    for (int j = offsets[g]; j < offsets[g + 1]; ++j) {
      float term = fine[members[j]] - error;
      float next = sum + term;
      error = (next - sum) - term;
      sum = next;
    }
    coarse[g] = sum;
  }
}
/* amg_prolong, amg.kern.h:18-21. */
void ko_prolong(int nf, const int* aggregate, const float* coarse, float* fine) {
  for (int i = 0; i < nf; ++i)
    if (aggregate[i] >= 0) fine[i] += coarse[aggregate[i]];
}
/* amg_galerkin, amg.kern.h:27-38. */
void ko_galerkin(int nnz_c, const int* offsets, const int* entries, const float* fine, float* coarse) {
  for (int e = 0; e < nnz_c; ++e) {
    float sum = 0.0f, error = 0.0f;
    for (int j = offsets[e]; j < offsets[e + 1]; ++j) {
      float term = fine[entries[j]];
      float next = sum + term;
      error += fabsf(sum) >= fabsf(term) ? (sum - next) + term : (term - next) + sum;
      sum = next;
    }
    coarse[e] = sum + error;
  }
}
/* fv_pressure_assemble, fv_flow.kern.h:164-183: zero the row's face entries,
 * subtract each internal face coefficient from its entry (faces may share
 * one), accumulate the right-hand side from the signed fluxes; the diagonal
 * is the upward-rounded sum of boundary and reference anchors and of the
 * negated stored off-diagonals. The reference cell keeps a unit row. */
void ko_fv_pressure_assemble(int n, const int* offsets, const int* faces, const float* sign,
                             const int* adjacent, const int* entry, const int* rows,
                             const int* diag, const float* coefficient, const float* flux,
                             float* values, float* rhs, int reference) {
  for (int i = 0; i < n; ++i) {
    upper ap = {0.0f, 0.0f};
    float b = 0.0f;
    for (int j = offsets[i]; j < offsets[i + 1]; ++j)
      if (adjacent[j] >= 0) values[entry[j]] = 0.0f;
    for (int j = offsets[i]; j < offsets[i + 1]; ++j) {
      const int f = faces[j], nb = adjacent[j];
      const float d = coefficient[f];
      const float term = sign[j] * flux[f];
      b = b - term;
      if (nb < 0 || nb == reference) ap = upper_add(ap, d);
      if (nb >= 0 && nb != reference && i != reference) values[entry[j]] = values[entry[j]] - d;
    }
    for (int j = rows[i]; j < rows[i + 1]; ++j)
      if (j != diag[i]) ap = upper_add(ap, -values[j]);
    values[diag[i]] = i == reference ? 1.0f : upper_value(ap);
    rhs[i] = i == reference ? 0.0f : b;
  }
}
/* fv_correct_flux, fv_flow.kern.h:185-190. */
void ko_fv_correct_flux(int n, const int* owner, const int* neighbour, const float* correction,
                        const float* coefficient, float* flux, int internal) {
  for (int i = 0; i < n; ++i) {
    const float pc = correction[owner[i]];
    const float pn = i < internal ? correction[neighbour[i]] : 0.0f;
    const float step = coefficient[i] * (pc - pn);
    flux[i] = flux[i] + step;
  }
}
/* fv_correct_velocity, fv_flow.kern.h:192-201. */
void ko_fv_correct_velocity(int n, const float* volume, const float* inverse,
                            const float* diagonal, const float* gx, const float* gy,
                            const float* gz, const float* correction, float* u, float* v,
                            float* w, float* p, float alpha) {
  for (int i = 0; i < n; ++i) {
    const float d = volume[i] * inverse[i];
    const float du = d * gx[i], dv = d * gy[i], dw = d * gz[i];
    u[i] = u[i] - du;
    v[i] = v[i] - dv;
    w[i] = w[i] - dw;
    const float bound = 0.7f * diagonal[i];
    const float ratio = bound * inverse[i];
    const float pa = fminf(alpha, ratio);
    const float dp = pa * correction[i];
    p[i] = p[i] + dp;
  }
}
/* amg_m_matrix_diagonal, amg.kern.h:44-58. */
static void m_matrix_diagonal(int nc, const int* offsets, const int* members, const int* fine_rows,
                              const int* fine_diag, const float* fine, const int* rows,
                              const int* diag, float* coarse) {
  for (int g = 0; g < nc; ++g) {
    upper d = {0.0f, 0.0f};
    for (int m = offsets[g]; m < offsets[g + 1]; ++m) {
      int row = members[m];
      upper surplus = {fine[fine_diag[row]], 0.0f};
      for (int j = fine_rows[row]; j < fine_rows[row + 1]; ++j)
        if (j != fine_diag[row]) surplus = upper_add(surplus, fine[j]);
      d = upper_add(d, upper_value(surplus));
    }
    for (int j = rows[g]; j < rows[g + 1]; ++j)
      if (j != diag[g]) d = upper_add(d, -coarse[j]);
    coarse[diag[g]] = upper_value(d);
  }
}

/* Scalar kernels, src/kutta/kernels/scalars.kern.h:51-121. */
void ko_scalar(int op, float* sc, int* st, int arg) {
  if (op == 9) { /* solver_reset :56-62 */
    st[0] = 0; st[1] = arg; st[2] = 0;
    sc[8] = 1.0f; sc[9] = 0.0f; sc[12] = 1.0f; sc[13] = 0.0f; sc[14] = 1.0f; sc[15] = 0.0f;
    return;
  }
  if (st[0] != 0) return;
  switch (op) {
    case 0: { /* solver_pcg_alpha :63-71 */
      pair rho = kp_load(sc, 0), pq = kp_load(sc, 2), alpha = kp_div(rho, pq);
      if (!kp_positive(rho) || !kp_positive(pq) || !kp_coefficient(alpha) || kp_zero(alpha)) st[0] = 2;
      else kp_store(sc, 8, alpha);
      break;
    }
    case 1: case 2: { /* solver_pcg_beta :72-80 */
      pair next = kp_load(sc, 4);
      pair numer = op == 2 ? kp_neg(kp_mul(kp_load(sc, 8), kp_load(sc, 6))) : next;
      pair beta = kp_div(numer, kp_load(sc, 0));
      if (!kp_positive(next) || !kp_coefficient(beta) || (kp_zero(beta) && !kp_zero(numer))) st[0] = 2;
      else { kp_store(sc, 10, beta); kp_store(sc, 0, next); }
      break;
    }
    case 3: { /* solver_bicg_beta :81-89 */
      pair rho = kp_load(sc, 0), omega = kp_load(sc, 12);
      pair beta = kp_mul(kp_div(rho, kp_load(sc, 14)), kp_div(kp_load(sc, 8), omega));
      if (kp_zero(rho) || !kp_finite(rho) || kp_zero(omega) || !kp_coefficient(omega) ||
          !kp_coefficient(beta) || kp_zero(beta)) st[0] = 2;
      else { kp_store(sc, 10, beta); st[2] = 0; }
      break;
    }
    case 4: { /* solver_bicg_alpha :90-97 */
      pair rv = kp_load(sc, 2), alpha = kp_div(kp_load(sc, 0), rv);
      if (kp_zero(rv) || !kp_finite(rv) || !kp_coefficient(alpha) || kp_zero(alpha)) st[0] = 2;
      else kp_store(sc, 8, alpha);
      break;
    }
    case 5: /* solver_bicg_s :98-103 */
      ++st[1];
      st[2] = kp_le(kp_load(sc, 16), kp_load(sc, 20)) ? 1 : 0;
      break;
    case 6: { /* solver_bicg_omega :104-112 */
      if (st[2] != 0) { kp_store(sc, 12, kp(0.0f, 0.0f)); break; }
      pair tt = kp_load(sc, 2), ts = kp_load(sc, 4), omega = kp_div(ts, tt);
      if (!kp_positive(tt) || !kp_finite(tt) || kp_zero(omega) || !kp_coefficient(omega)) st[0] = 2;
      else kp_store(sc, 12, omega);
      break;
    }
    case 7: case 8: { /* solver_check :113-121 */
      int pcg = op == 7;
      if (pcg) ++st[1];
      pair rr = kp_load(sc, 18);
      if (!kp_finite(rr) || kp_le(rr, kp_load(sc, 20)) || !kp_le(rr, kp_load(sc, 22)) || st[1] % 50 == 0)
        st[0] = 1;
      if (!pcg) kp_store(sc, 14, kp_load(sc, 0));
      break;
    }
    default: break;
  }
}
/* solver_step, scalars.kern.h:122-127. */
void ko_solver_step(int n, float* x, float* r, const float* p, const float* q,
                    const float* scalars, const int* status) {
  if (status[0] != 0) return;
  float alpha = kp_float(kp_load(scalars, 8));
  for (int i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
}

/* Serial double reductions of the CPU backend, src/kutta/runtime/cpu/cpu_device.cpp:37-89. */
static double dsum(const float* x, int n) { double s = 0; for (int i = 0; i < n; ++i) s += x[i]; return s; }
static double ddot(const float* x, const float* y, int n) {
  double s = 0;
  for (int i = 0; i < n; ++i) s += (double)x[i] * (double)y[i];
  return s;
}
static double dmax_abs(const float* x, int n) {
  double m = 0;
  for (int i = 0; i < n; ++i) { double v = fabs((double)x[i]); if (v > m || isnan(v)) m = v; }
  return m;
}
static void store_pair(float* p, double value) {
  p[0] = (float)value;
  p[1] = isfinite(p[0]) ? (float)(value - (double)p[0]) : 0.0f;
}

/* ------------------------------------------------------------ setup ---- */
typedef struct { int n, nnz; int *row_ptr, *col, *diag; double* val; } hcsr; /* CsrMatrixHost */
typedef struct { int *aggregate, *member_offsets, *members, *entry_offsets, *entries; int n_members, n_entries; } transfer;

static void hcsr_free(hcsr* a) { free(a->row_ptr); free(a->col); free(a->diag); free(a->val); memset(a, 0, sizeof *a); }
static void transfer_free(transfer* t) {
  free(t->aggregate); free(t->member_offsets); free(t->members); free(t->entry_offsets); free(t->entries);
  memset(t, 0, sizeof *t);
}
static int find_entry(const hcsr* a, int row, int column) { /* lower_bound */
  int lo = a->row_ptr[row], hi = a->row_ptr[row + 1];
  while (lo < hi) { int mid = (lo + hi) / 2; if (a->col[mid] < column) lo = mid + 1; else hi = mid; }
  return lo;
}

/* pairs(), src/kutta/linalg/amg.cpp:25-75. */
static int* pairs(const hcsr* a, double threshold, int exclude_isolated, int absorb) {
  int n = a->n;
  int* offsets = xcalloc((size_t)n + 1, sizeof(int));
  int* sources = xmalloc(sizeof(int) * (size_t)a->nnz);
  for (int j = 0; j < a->nnz; ++j) ++offsets[a->col[j] + 1];
  for (int i = 0; i < n; ++i) offsets[i + 1] += offsets[i];
  int* cursor = xmalloc(sizeof(int) * (size_t)(n + 1));
  memcpy(cursor, offsets, sizeof(int) * (size_t)(n + 1));
  for (int i = 0; i < n; ++i)
    for (int j = a->row_ptr[i]; j < a->row_ptr[i + 1]; ++j) sources[cursor[a->col[j]]++] = i;
  free(cursor);
  int* map = xmalloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; ++i) map[i] = -1;
  int next = 0;
  for (int i = 0; i < n; ++i) {
    if (map[i] != -1) continue;
    double strongest = 0;
    int partner = -1;
    double weight_best = 0;
    for (int visit = 0; visit < 2; ++visit) {  /* the two neighbour sweeps */
      int out = a->row_ptr[i], in = offsets[i];
      while (out < a->row_ptr[i + 1] || in < offsets[i + 1]) {
        int oc = out < a->row_ptr[i + 1] ? a->col[out] : n;
        int ic = in < offsets[i + 1] ? sources[in] : n;
        int column = oc < ic ? oc : ic;
        double w = 0;
        if (oc == column) w = fabs(a->val[out++]);
        if (ic == column) {
          double t = fabs(a->val[find_entry(a, column, i)]);
          w = w > t ? w : t;
          ++in;
        }
        if (column != i && w != 0) {
          if (visit == 0) strongest = strongest > w ? strongest : w;
          else if (map[column] == -1 && w > weight_best && w >= threshold * strongest) {
            partner = column;
            weight_best = w;
          }
        }
      }
      if (visit == 0 && exclude_isolated && strongest == 0) break;
    }
    if (exclude_isolated && strongest == 0) continue;
    map[i] = next;
    if (partner != -1) map[partner] = next;
    ++next;
  }
  if (absorb) {
    /* Mixed-precision hierarchy (kutta_b200's own method, no reference
     * counterpart): an unpaired row joins the pair of its strongest strongly
     * connected neighbour (weight >= threshold * the row's strongest weight
     * and >= 0.01 sqrt(|a_ii a_jj|)) that belongs to a pair; rows in order,
     * aggregates renumbered in order. */
    int* size = xcalloc((size_t)(next > 0 ? next : 1), sizeof(int));
    for (int i = 0; i < n; ++i) if (map[i] >= 0) ++size[map[i]];
    for (int i = 0; i < n; ++i) {
      if (map[i] < 0 || size[map[i]] != 1) continue;
      int best = -1;
      double bw = 0, strongest = 0;
      for (int visit = 0; visit < 2; ++visit) {  /* strongest weight, then the choice */
        int out = a->row_ptr[i], in = offsets[i];
        while (out < a->row_ptr[i + 1] || in < offsets[i + 1]) {
          int oc = out < a->row_ptr[i + 1] ? a->col[out] : n;
          int ic = in < offsets[i + 1] ? sources[in] : n;
          int column = oc < ic ? oc : ic;
          double w = 0;
          if (oc == column) w = fabs(a->val[out++]);
          if (ic == column) {
            double t = fabs(a->val[find_entry(a, column, i)]);
            w = w > t ? w : t;
            ++in;
          }
          if (column == i || w == 0) continue;
          if (visit == 0) {
            if (w > strongest) strongest = w;
          } else {
            int g = map[column];
            double coupling = 0.01 * sqrt(fabs(a->val[a->diag[i]]) * fabs(a->val[a->diag[column]]));
            if (g >= 0 && g != map[i] && size[g] >= 2 && w > bw && w >= threshold * strongest &&
                w >= coupling) {
              best = g;
              bw = w;
            }
          }
        }
      }
      if (best < 0) continue;
      size[map[i]] = 0;
      map[i] = best;
      ++size[best];
    }
    int* renumber = xmalloc(sizeof(int) * (size_t)(next > 0 ? next : 1));
    int kept = 0;
    for (int g = 0; g < next; ++g) renumber[g] = size[g] > 0 ? kept++ : -1;
    for (int i = 0; i < n; ++i) if (map[i] >= 0) map[i] = renumber[map[i]];
    free(size); free(renumber);
  }
  free(offsets); free(sources);
  return map;
}

typedef struct { int col, canonical, source; } tup;
static int tup_cmp(const void* pa, const void* pb) {
  const tup* a = pa; const tup* b = pb;
  if (a->col != b->col) return a->col < b->col ? -1 : 1;
  if (a->canonical != b->canonical) return a->canonical < b->canonical ? -1 : 1;
  return a->source < b->source ? -1 : (a->source > b->source);
}

/* coarsen(), amg.cpp:77-158. Takes ownership of `aggregate`. */
static void coarsen(const hcsr* fine, int* aggregate, int entry_map, int m_matrix, hcsr* cm,
                    transfer* t) {
  memset(cm, 0, sizeof *cm);
  memset(t, 0, sizeof *t);
  t->aggregate = aggregate;
  int nc = 0;
  for (int i = 0; i < fine->n; ++i) if (aggregate[i] + 1 > nc) nc = aggregate[i] + 1;
  cm->n = nc;
  cm->row_ptr = xcalloc((size_t)nc + 1, sizeof(int));
  cm->diag = xcalloc((size_t)nc + 1, sizeof(int));
  t->member_offsets = xcalloc((size_t)nc + 1, sizeof(int));
  for (int i = 0; i < fine->n; ++i) if (aggregate[i] >= 0) ++t->member_offsets[aggregate[i] + 1];
  for (int g = 0; g < nc; ++g) t->member_offsets[g + 1] += t->member_offsets[g];
  t->n_members = t->member_offsets[nc];
  t->members = xmalloc(sizeof(int) * (size_t)t->n_members);
  int* cursor = xmalloc(sizeof(int) * (size_t)(nc + 1));
  memcpy(cursor, t->member_offsets, sizeof(int) * (size_t)(nc + 1));
  for (int i = 0; i < fine->n; ++i) if (aggregate[i] >= 0) t->members[cursor[aggregate[i]]++] = i;
  free(cursor);
  size_t cap = (size_t)fine->nnz + 1;
  cm->col = xmalloc(sizeof(int) * cap);
  cm->val = xmalloc(sizeof(double) * cap);
  if (entry_map) {
    t->entries = xmalloc(sizeof(int) * cap);
    t->entry_offsets = xmalloc(sizeof(int) * (cap + 1));
    t->entry_offsets[0] = 0;
  }
  int n_offsets = 1, ncol = 0;
  size_t row_cap = 64;
  tup* row = xmalloc(sizeof(tup) * row_cap);
  for (int g = 0; g < nc; ++g) {
    size_t count = 0;
    for (int m = t->member_offsets[g]; m < t->member_offsets[g + 1]; ++m) {
      int i = t->members[m];
      for (int j = fine->row_ptr[i]; j < fine->row_ptr[i + 1]; ++j) {
        int target = aggregate[fine->col[j]];
        if (target < 0) continue;
        int canonical = j;
        if (m_matrix) {
          int opposite = find_entry(fine, fine->col[j], i);
          canonical = j < opposite ? j : opposite;
        }
        if (count == row_cap) { row_cap *= 2; row = realloc(row, sizeof(tup) * row_cap); if (!row) fail(-1, "oom"); }
        row[count].col = target; row[count].canonical = canonical; row[count].source = j;
        ++count;
      }
    }
    qsort(row, count, sizeof(tup), tup_cmp);
    int previous = -1;
    float sum = 0, error = 0;
    for (size_t k = 0; k < count; ++k) {
      if (row[k].col != previous) {
        if (previous != -1) cm->val[ncol - 1] = sum + error;
        sum = error = 0;
        if (entry_map && previous != -1) t->entry_offsets[n_offsets++] = t->n_entries;
        if (row[k].col == g) cm->diag[g] = ncol;
        cm->col[ncol] = row[k].col;
        cm->val[ncol] = 0;
        ++ncol;
        previous = row[k].col;
      }
      if (entry_map) t->entries[t->n_entries++] = row[k].source;
      float term = (float)fine->val[row[k].source];
      float next = sum + term;
      error += fabsf(sum) >= fabsf(term) ? (sum - next) + term : (term - next) + sum;
      sum = next;
    }
    if (previous != -1) cm->val[ncol - 1] = sum + error;
    if (entry_map) t->entry_offsets[n_offsets++] = t->n_entries;
    cm->row_ptr[g + 1] = ncol;
    if (m_matrix) {
      upper d = {0, 0};
      for (int m = t->member_offsets[g]; m < t->member_offsets[g + 1]; ++m) {
        int i = t->members[m];
        upper surplus = {(float)fine->val[fine->diag[i]], 0};
        for (int j = fine->row_ptr[i]; j < fine->row_ptr[i + 1]; ++j)
          if (j != fine->diag[i]) surplus = upper_add(surplus, (float)fine->val[j]);
        d = upper_add(d, upper_value(surplus));
      }
      for (int j = cm->row_ptr[g]; j < cm->row_ptr[g + 1]; ++j)
        if (j != cm->diag[g]) d = upper_add(d, -(float)cm->val[j]);
      cm->val[cm->diag[g]] = upper_value(d);
    }
  }
  free(row);
  cm->nnz = ncol;
}

/* aggregate(), amg.cpp:160-174. */
static void aggregate_level(const hcsr* a, const ko_options* o, hcsr* cm, transfer* t) {
  int* map = pairs(a, o->threshold, 1, o->absorb);
  for (int pass = 1; pass < o->passes; ++pass) {
    hcsr im; transfer it;
    coarsen(a, map, 0, o->m_matrix, &im, &it);
    int* next = pairs(&im, o->threshold, 0, o->absorb);
    map = it.aggregate;
    it.aggregate = NULL;
    for (int i = 0; i < a->n; ++i) if (map[i] >= 0) map[i] = next[map[i]];
    free(next);
    hcsr_free(&im);
    transfer_free(&it);
  }
  coarsen(a, map, 1, o->m_matrix, cm, t);
}

/* diagonal_values(), src/kutta/linalg/solver.cpp:37-53. */
static float* diagonal_values(const hcsr* a, int l1, int nullspace) {
  float* inverse = xmalloc(sizeof(float) * (size_t)a->n);
  for (int i = 0; i < a->n; ++i) {
    float d = (float)a->val[a->diag[i]];
    REQUIRE(!l1 || d >= 0, "AMG: requires positive diagonals");
    REQUIRE(d != 0 || (nullspace && a->n == 1), "solver: invalid values or zero diagonal");
    float off = 0;
    if (l1)
      for (int j = a->row_ptr[i]; j < a->row_ptr[i + 1]; ++j)
        if (j != a->diag[i]) off += fabsf((float)a->val[j]);
    float h = 0.5f * (fabsf(d) + off);
    float scale = l1 ? (fabsf(d) < h ? h : fabsf(d)) : d;
    inverse[i] = scale != 0 ? 1.0f / scale : 0;
    REQUIRE(isfinite(scale) && isfinite(inverse[i]), "solver: invalid values or diagonal inverse");
  }
  return inverse;
}

/* csr.cpp:11-31,58-64. */
static void validate_host(const hcsr* a) {
  REQUIRE(a->n >= 0, "CSR: negative row count");
  REQUIRE(a->row_ptr[0] == 0 && a->row_ptr[a->n] == a->nnz, "CSR: invalid row offsets");
  for (int i = 0; i < a->n; ++i) {
    REQUIRE(a->row_ptr[i] >= 0 && a->row_ptr[i] <= a->row_ptr[i + 1] && a->row_ptr[i + 1] <= a->nnz,
            "CSR: invalid row range");
    int previous = -1;
    for (int j = a->row_ptr[i]; j < a->row_ptr[i + 1]; ++j) {
      REQUIRE(a->col[j] > previous && a->col[j] < a->n, "CSR: columns must be in range, unique and sorted");
      previous = a->col[j];
    }
    REQUIRE(a->diag[i] >= a->row_ptr[i] && a->diag[i] < a->row_ptr[i + 1] && a->col[a->diag[i]] == i,
            "CSR: missing or incorrect diagonal");
  }
  for (int j = 0; j < a->nnz; ++j)
    REQUIRE(isfinite(a->val[j]) && fabs(a->val[j]) <= 3.4028234663852886e38,
            "CSR: nonfinite or out-of-range value");
}

/* ------------------------------------------------------------ solver ---- */
typedef struct {
  int n, nnz;
  int *row_ptr, *col, *diag;
  float* val;  /* coarse operators (level 0 uses the caller's values) */
  float *l1, *xa, *ra, *b, *projection;
  float *x, *r;  /* current roles of the ping-pong pair */
  transfer t;
} level;

struct ko_solver {
  ko_options o;
  int n, nnz, nlevels, amg, bicg, nullspace;
  level* levels;
  double complexity;
  float* jacobi_inverse;
  float *r, *z, *p, *q, *shadow, *s, *t, *zs, *best;
  float scalars[24], projection[2];
  int status[3];
  int speculate, has_spec;
  double speculated, best_residual;
  int previous_iterations, verified_current;
  const float* val;
};

static float* fvec(int n) { return xcalloc((size_t)(n > 0 ? n : 1), sizeof(float)); }

ko_solver* ko_create(int n, int nnz, const int* row_ptr, const int* col, const int* diag,
                     const double* val, const ko_options* o, char* err, int errlen) {
  jmp_buf jump;
  jmp_buf* saved = g_jump;
  g_jump = &jump;
  ko_solver* s = NULL;
  if (setjmp(jump)) {
    g_jump = saved;
    if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", g_msg);
    return NULL;  /* leaks partial state on error; test infrastructure only */
  }
  hcsr a = {n, nnz, (int*)row_ptr, (int*)col, (int*)diag, (double*)val};
  s = xcalloc(1, sizeof(ko_solver));
  s->o = *o;
  s->n = n; s->nnz = nnz;
  s->amg = o->kind == 3 || o->kind == 4;
  s->bicg = o->kind == 2 || o->kind == 4;
  s->nullspace = o->nullspace;
  REQUIRE(o->kind >= 0 && o->kind <= 4, "unknown SolverKind");
  if (s->amg) { /* make_amg_solver checks, amg.cpp:347-379 */
    REQUIRE(o->cycle == 0 && o->pre_sweeps > 0 && o->post_sweeps > 0 && o->coarse_sweeps > 0 &&
            o->coarse_rows >= 1 && o->max_levels >= 1 && o->passes >= 1 && o->passes <= 8 &&
            isfinite(o->threshold) && o->threshold >= 0 && o->threshold <= 1, "AMG: invalid options");
    REQUIRE(o->kind != 3 || o->pre_sweeps == o->post_sweeps, "AMG-PCG requires equal pre/post sweeps");
  }
  validate_host(&a);
  if (s->amg && o->m_matrix) {
    for (int i = 0; i < n; ++i) {
      long double sum = 0;
      for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j) {
        float value = (float)val[j];
        sum += value;
        int c = col[j], opp = find_entry(&a, c, i);
        REQUIRE(opp < row_ptr[c + 1] && col[opp] == i && value == (float)val[opp] && (c == i || value <= 0),
                "AMG M-matrix: expected symmetric nonpositive edges");
      }
      REQUIRE(sum >= 0, "AMG M-matrix: expected diagonally dominant rows");
    }
  }
  int cap = s->amg ? (o->max_levels > 0 ? o->max_levels : 1) : 1;
  s->levels = xcalloc((size_t)cap, sizeof(level));
  level* l0 = &s->levels[0];
  l0->n = n; l0->nnz = nnz;
  l0->row_ptr = xmalloc(sizeof(int) * (size_t)(n + 1)); memcpy(l0->row_ptr, row_ptr, sizeof(int) * (size_t)(n + 1));
  l0->col = xmalloc(sizeof(int) * (size_t)nnz); memcpy(l0->col, col, sizeof(int) * (size_t)nnz);
  l0->diag = xmalloc(sizeof(int) * (size_t)n); memcpy(l0->diag, diag, sizeof(int) * (size_t)n);
  s->nlevels = 1;
  if (s->amg) { /* Aggregation ctor, amg.cpp:200-226 */
    l0->l1 = diagonal_values(&a, 1, o->nullspace);
    l0->ra = fvec(n); l0->r = l0->ra;
    if (o->nullspace) l0->projection = fvec(2);
    hcsr fine = a, owned = {0};
    size_t total = (size_t)nnz;
    while (fine.n > o->coarse_rows && s->nlevels < o->max_levels) {
      hcsr cm; transfer t;
      aggregate_level(&fine, o, &cm, &t);
      int active = t.n_members;
      if (active == 0 || (double)cm.n >= 0.85 * (double)active) { hcsr_free(&cm); transfer_free(&t); break; }
      s->levels[s->nlevels - 1].t = t;
      total += (size_t)cm.nnz;
      level* l = &s->levels[s->nlevels++];
      l->n = cm.n; l->nnz = cm.nnz;
      l->row_ptr = xmalloc(sizeof(int) * (size_t)(cm.n + 1)); memcpy(l->row_ptr, cm.row_ptr, sizeof(int) * (size_t)(cm.n + 1));
      l->col = xmalloc(sizeof(int) * (size_t)(cm.nnz ? cm.nnz : 1)); memcpy(l->col, cm.col, sizeof(int) * (size_t)cm.nnz);
      l->diag = xmalloc(sizeof(int) * (size_t)(cm.n ? cm.n : 1)); memcpy(l->diag, cm.diag, sizeof(int) * (size_t)cm.n);
      l->val = fvec(cm.nnz);
      for (int j = 0; j < cm.nnz; ++j) l->val[j] = (float)cm.val[j];
      l->l1 = diagonal_values(&cm, 1, o->nullspace);
      l->xa = fvec(cm.n); l->x = l->xa;
      l->ra = fvec(cm.n); l->r = l->ra;
      l->b = fvec(cm.n);
      if (o->nullspace) l->projection = fvec(2);
      if (owned.row_ptr) hcsr_free(&owned);
      owned = cm;
      fine = owned;
    }
    if (owned.row_ptr) hcsr_free(&owned);
    s->complexity = nnz ? (double)total / nnz : 0;
  } else {
    s->jacobi_inverse = diagonal_values(&a, 0, 0);
  }
  s->r = fvec(n); s->z = fvec(n); s->p = fvec(n); s->q = fvec(n); s->best = fvec(n);
  if (s->bicg) { s->shadow = fvec(n); s->s = fvec(n); s->t = fvec(n); s->zs = fvec(n); }
  s->speculate = o->kind != 0 && n <= (1 << 17);
  g_jump = saved;
  return s;
}

int ko_levels(const ko_solver* s) { return s->nlevels; }
void ko_level_shape(const ko_solver* s, int level, int* n, int* nnz) {
  *n = s->levels[level].n; *nnz = s->levels[level].nnz;
}
void ko_level_copy(const ko_solver* s, int lv, int* row_ptr, int* col, float* val, float* l1,
                   int* aggregate) {
  const level* l = &s->levels[lv];
  if (row_ptr) memcpy(row_ptr, l->row_ptr, sizeof(int) * (size_t)(l->n + 1));
  if (col) memcpy(col, l->col, sizeof(int) * (size_t)l->nnz);
  if (val && l->val) memcpy(val, l->val, sizeof(float) * (size_t)l->nnz);
  if (l1 && l->l1) memcpy(l1, l->l1, sizeof(float) * (size_t)l->n);
  if (aggregate && l->t.aggregate) memcpy(aggregate, l->t.aggregate, sizeof(int) * (size_t)l->n);
}

void ko_destroy(ko_solver* s) {
  if (!s) return;
  for (int i = 0; i < s->nlevels; ++i) {
    level* l = &s->levels[i];
    free(l->row_ptr); free(l->col); free(l->diag); free(l->val); free(l->l1);
    free(l->xa); free(l->ra); free(l->b); free(l->projection);
    transfer_free(&l->t);
  }
  free(s->levels); free(s->jacobi_inverse);
  free(s->r); free(s->z); free(s->p); free(s->q); free(s->best);
  free(s->shadow); free(s->s); free(s->t); free(s->zs);
  free(s);
}

int ko_describe(const ko_solver* s, char* out, int len) {
  const char* name = s->o.kind == 0 ? "damped Jacobi" : (s->o.kind == 1 || s->o.kind == 3 ? "PCG" : "BiCGStab");
  if (s->amg)
    return snprintf(out, (size_t)len, "%s, aggregation AMG V-cycle, %d levels, op complexity %.3f%s", name,
                    s->nlevels, s->complexity, s->nullspace ? ", constant-nullspace projection" : "");
  return snprintf(out, (size_t)len, "%s, Jacobi%s", name, s->nullspace ? ", constant-nullspace projection" : "");
}

/* Aggregation::refresh, amg.cpp:228-256; Jacobi::refresh, solver.cpp:61-64. */
int ko_refresh(ko_solver* s, const float* val, char* err, int errlen) {
  jmp_buf jump;
  jmp_buf* saved = g_jump;
  g_jump = &jump;
  if (setjmp(jump)) {
    g_jump = saved;
    if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", g_msg);
    return -1;
  }
  float* invalid = fvec(s->n);
  if (!s->amg) {
    ko_diagonal(s->n, s->levels[0].row_ptr, s->levels[0].diag, val, s->jacobi_inverse, invalid, 0);
    double bad = dmax_abs(invalid, s->n);
    free(invalid);
    REQUIRE(bad == 0, "Jacobi: invalid values or zero diagonal");
    g_jump = saved;
    return 0;
  }
  const float* matrix = val;
  double checks[64];
  double allowed[64];
  for (int i = 0; i < s->nlevels; ++i) {
    level* l = &s->levels[i];
    ko_diagonal(l->n, l->row_ptr, l->diag, matrix, l->l1, invalid, 1);
    allowed[i] = s->nullspace && l->n == 1 ? 1 : 0;
    checks[i] = dmax_abs(invalid, l->n);
    if (i + 1 < s->nlevels) {
      level* c = &s->levels[i + 1];
      ko_galerkin(c->nnz, l->t.entry_offsets, l->t.entries, matrix, c->val);
      if (s->o.m_matrix)
        m_matrix_diagonal(c->n, l->t.member_offsets, l->t.members, l->row_ptr, l->diag, matrix,
                          c->row_ptr, c->diag, c->val);
      matrix = c->val;
    }
  }
  free(invalid);
  for (int i = 0; i < s->nlevels; ++i) {
    REQUIRE(checks[i] != 3, "AMG: requires positive diagonals");
    REQUIRE(checks[i] <= allowed[i], "AMG: invalid values or zero diagonal");
  }
  g_jump = saved;
  return 0;
}

/* project(), src/kutta/linalg/detail.hpp:13-19 + solver_project scalars.kern.h:150-152. */
static void project(float* x, int n, float* scalar) {
  if (n == 0) return;
  store_pair(scalar, dsum(x, n));
  float count = (float)n;
  float mean = kp_float(kp_div(kp_load(scalar, 0), kp(count, (float)((double)n - (double)count))));
  for (int i = 0; i < n; ++i) x[i] -= mean;
}

static void smooth(ko_solver* s, level* l, const float* vals, const float* b, float** x, int sweeps,
                   int zero_start) {
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    ko_smooth(l->n, l->row_ptr, l->col, vals, *x, b, l->l1, l->r, s->status, zero_start && sweep == 0);
    float* t = *x; *x = l->r; l->r = t;
  }
}

/* Aggregation::cycle, amg.cpp:283-310. */
static void cycle(ko_solver* s, int index, const float* b, float** x) {
  level* l = &s->levels[index];
  const float* vals = index == 0 ? s->val : l->val;
  memset(*x, 0, sizeof(float) * (size_t)l->n);  /* dev.fill(x, 0) */
  if (index + 1 == s->nlevels) {
    if (l->n <= 24) ko_coarse_solve(l->row_ptr, l->col, vals, *x, b, l->l1, s->status, l->n, s->o.coarse_sweeps);
    else smooth(s, l, vals, b, x, s->o.coarse_sweeps, 1);
  } else {
    smooth(s, l, vals, b, x, s->o.pre_sweeps, 1);
    if (s->status[0] == 0) ko_residual(l->n, l->row_ptr, l->col, vals, *x, b, l->r);
    level* c = &s->levels[index + 1];
    if (s->status[0] == 0) ko_restrict(c->n, l->t.member_offsets, l->t.members, l->r, c->b);
    if (s->nullspace) project(c->b, c->n, c->projection);
    cycle(s, index + 1, c->b, &c->x);
    if (s->status[0] == 0) ko_prolong(l->n, l->t.aggregate, c->x, *x);
    smooth(s, l, vals, b, x, s->o.post_sweeps, 0);
  }
  if (s->nullspace && index != 0) project(*x, l->n, l->projection);
}

/* Krylov::apply, solver.cpp:197-200. */
static void apply(ko_solver* s, const float* r, float** z) {
  if (s->amg) cycle(s, 0, r, z);
  else if (s->status[0] == 0) for (int i = 0; i < s->n; ++i) (*z)[i] = r[i] * s->jacobi_inverse[i];
  if (s->nullspace) project(*z, s->n, s->projection);
}

static void residual(ko_solver* s, const float* x, const float* b, float* r) {
  ko_residual(s->n, s->levels[0].row_ptr, s->levels[0].col, s->val, x, b, r);
}
static double norm(const float* x, int n) { return sqrt(ddot(x, x, n)); }
static void copyv(float* dst, const float* src, int n) { if (dst != src) memcpy(dst, src, sizeof(float) * (size_t)n); }

/* Krylov::verified, solver.cpp:201-222. */
static int verified(ko_solver* s, float* x, const float* b, double target, ko_stats* st) {
  float* spec_r = s->bicg ? s->t : s->q;
  float* spec_x = s->bicg ? s->s : s->z;
  if (s->has_spec) {
    if (s->nullspace) copyv(x, spec_x, s->n);
    copyv(s->r, spec_r, s->n);
    st->final_residual = s->speculated;
    s->has_spec = 0;
  } else {
    if (s->nullspace) project(x, s->n, s->projection);
    residual(s, x, b, s->r);
    st->final_residual = norm(s->r, s->n);
  }
  s->verified_current = 1;
  st->converged = isfinite(st->final_residual) && st->final_residual <= target;
  if (st->final_residual < s->best_residual) { s->best_residual = st->final_residual; copyv(s->best, x, s->n); }
  if (s->nullspace) project(s->r, s->n, s->projection);
  return st->converged;
}
static int diverged(const ko_stats* st) {
  return !isfinite(st->final_residual) || st->final_residual > 1e3 * st->initial_residual;
}
/* Krylov::poll, solver.cpp:230-244 (the speculative residual for small n). */
static void poll(ko_solver* s, const float* x, const float* b) {
  if (s->speculate) {
    float* spec_r = s->bicg ? s->t : s->q;
    float* spec_x = s->bicg ? s->s : s->z;
    const float* source = x;
    if (s->nullspace) { copyv(spec_x, x, s->n); project(spec_x, s->n, s->projection); source = spec_x; }
    residual(s, source, b, spec_r);
    s->speculated = sqrt(ddot(spec_r, spec_r, s->n));
    s->has_spec = 1;
  }
}
static int replacement(ko_solver* s, float* x, const float* b, double target, ko_stats* st,
                       int* restarts, double* last) {
  if (verified(s, x, b, target, st) || diverged(st)) return 0;
  *restarts = st->final_residual >= 0.9 * *last ? *restarts + 1 : 0;
  *last = st->final_residual;
  return *restarts < 12;
}
static int batch_interval(const ko_solver* s, const ko_control* c) {
  return s->previous_iterations > 0 && s->previous_iterations < c->interval ? s->previous_iterations + 1 : c->interval;
}

static void dot_into(const float* x, const float* y, int n, float* sc, int off) { store_pair(sc + off, ddot(x, y, n)); }

/* Krylov::pcg, solver.cpp:271-313. */
static void pcg(ko_solver* s, float* x, const float* b, const ko_control* c, double target, ko_stats* st) {
  int n = s->n;
  const level* l0 = &s->levels[0];
#define RESTART() do { ko_scalar(9, s->scalars, s->status, st->iterations); apply(s, s->r, &s->z); \
    copyv(s->p, s->z, n); dot_into(s->r, s->z, n, s->scalars, 0); } while (0)
  RESTART();
  int restarts = 0;
  double last = st->initial_residual;
  int interval = batch_interval(s, c);
  while (st->iterations < c->max_iter) {
    int batch = interval < c->max_iter - st->iterations ? interval : c->max_iter - st->iterations;
    s->verified_current = 0;
    s->has_spec = 0;
    for (int j = 0; j < batch; ++j) {
      if (s->status[0] == 0) ko_spmv(n, l0->row_ptr, l0->col, s->val, s->p, s->q);
      dot_into(s->p, s->q, n, s->scalars, 2);
      ko_scalar(0, s->scalars, s->status, 0);
      ko_solver_step(n, x, s->r, s->p, s->q, s->scalars, s->status);
      dot_into(s->r, s->r, n, s->scalars, 18);
      ko_scalar(7, s->scalars, s->status, 0);
      if (st->iterations + j + 1 == c->max_iter) continue;
      apply(s, s->r, &s->z);
      dot_into(s->r, s->z, n, s->scalars, 4);
      ko_scalar(1, s->scalars, s->status, 0);
      if (s->status[0] == 0) {
        float beta = kp_float(kp_load(s->scalars, 10));
        for (int i = 0; i < n; ++i) s->p[i] = s->z[i] + beta * s->p[i];
      }
    }
    poll(s, x, b);
    st->iterations = s->status[1];
    if (s->status[0] == 2) break;
    if (s->status[0] == 1) {
      if (!replacement(s, x, b, target, st, &restarts, &last) || st->iterations == c->max_iter) break;
      if (st->final_residual <= 10 * target) interval = 1;
      RESTART();
    }
  }
#undef RESTART
}

/* Krylov::bicgstab, solver.cpp:314-361. */
static void bicgstab(ko_solver* s, float* x, const float* b, const ko_control* c, double target, ko_stats* st) {
  int n = s->n;
  const level* l0 = &s->levels[0];
  float* sc = s->scalars;
#define RESTART() do { ko_scalar(9, sc, s->status, st->iterations); copyv(s->shadow, s->r, n); \
    memset(s->p, 0, sizeof(float) * (size_t)n); memset(s->q, 0, sizeof(float) * (size_t)n); } while (0)
  RESTART();
  int restarts = 0;
  double last = st->initial_residual;
  int interval = batch_interval(s, c);
  while (st->iterations < c->max_iter) {
    int batch = interval < c->max_iter - st->iterations ? interval : c->max_iter - st->iterations;
    s->verified_current = 0;
    s->has_spec = 0;
    for (int j = 0; j < batch; ++j) {
      dot_into(s->shadow, s->r, n, sc, 0);
      ko_scalar(3, sc, s->status, 0);
      if (s->status[0] == 0) {
        float beta = kp_float(kp_load(sc, 10)), omega = kp_float(kp_load(sc, 12));
        for (int i = 0; i < n; ++i) s->p[i] = s->r[i] + beta * (s->p[i] - omega * s->q[i]);
      }
      apply(s, s->p, &s->z);
      if (s->status[0] == 0) ko_spmv(n, l0->row_ptr, l0->col, s->val, s->z, s->q);
      dot_into(s->shadow, s->q, n, sc, 2);
      ko_scalar(4, sc, s->status, 0);
      if (s->status[0] == 0) {
        float alpha = kp_float(kp_load(sc, 8));
        for (int i = 0; i < n; ++i) s->s[i] = s->r[i] - alpha * s->q[i];
      }
      dot_into(s->s, s->s, n, sc, 16);
      ko_scalar(5, sc, s->status, 0);
      apply(s, s->s, &s->zs);
      if (s->status[0] == 0) ko_spmv(n, l0->row_ptr, l0->col, s->val, s->zs, s->t);
      store_pair(sc + 2, ddot(s->t, s->t, n));
      store_pair(sc + 4, ddot(s->t, s->s, n));
      ko_scalar(6, sc, s->status, 0);
      if (s->status[0] == 0) {
        float alpha = kp_float(kp_load(sc, 8)), omega = kp_float(kp_load(sc, 12));
        for (int i = 0; i < n; ++i) {
          if (s->status[2] != 0) { x[i] += alpha * s->z[i]; s->r[i] = s->s[i]; }
          else { x[i] += alpha * s->z[i] + omega * s->zs[i]; s->r[i] = s->s[i] - omega * s->t[i]; }
        }
      }
      dot_into(s->r, s->r, n, sc, 18);
      ko_scalar(8, sc, s->status, 0);
    }
    poll(s, x, b);
    st->iterations = s->status[1];
    if (s->status[0] == 2) break;
    if (s->status[0] == 1) {
      if (!replacement(s, x, b, target, st, &restarts, &last) || st->iterations == c->max_iter) break;
      if (st->final_residual <= 10 * target) interval = 1;
      RESTART();
    }
  }
#undef RESTART
}

/* Krylov::solve, solver.cpp:97-176. */
int ko_solve(ko_solver* s, const float* val, float* x, const float* b, const ko_control* c,
             ko_stats* st, char* err, int errlen) {
  jmp_buf jump;
  jmp_buf* saved = g_jump;
  g_jump = &jump;
  if (setjmp(jump)) {
    g_jump = saved;
    if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", g_msg);
    return g_code;
  }
  int n = s->n;
  s->val = val;
  REQUIRE(x != b || n == 0, "solve: vector size or alias mismatch");
  REQUIRE(c->max_iter >= 0 && isfinite(c->rel_tol) && c->rel_tol >= 0 && isfinite(c->abs_tol) &&
          c->abs_tol >= 0 && c->interval > 0, "solve: invalid control");
  s->has_spec = 0;
  memset(st, 0, sizeof *st);
  if (!s->nullspace) residual(s, x, b, s->r);
  double e0 = ddot(b, b, n), e1 = ddot(x, x, n);
  double e2 = s->nullspace ? dsum(b, n) : ddot(s->r, s->r, n);
  double bnorm = sqrt(e0);
  if (!(isfinite(bnorm) && isfinite(sqrt(e1)))) fail(-2, "solve: nonfinite input vector");
  if (s->nullspace) {
    if (n != 0) {
      REQUIRE(fabs(e2) <= 1e-6 * sqrt((double)n) * bnorm, "solve: incompatible RHS for constant Neumann nullspace");
      project(x, n, s->projection);
    }
    residual(s, x, b, s->r);
    st->initial_residual = norm(s->r, n);
  } else st->initial_residual = sqrt(e2);
  st->final_residual = st->initial_residual;
  s->verified_current = 1;
  double target = c->abs_tol > c->rel_tol * st->initial_residual ? c->abs_tol : c->rel_tol * st->initial_residual;
  if (!isfinite(st->initial_residual)) { g_jump = saved; return 0; }
  if (st->final_residual <= target) { st->converged = 1; g_jump = saved; return 0; }
  if (s->nullspace) project(s->r, n, s->projection);
  s->best_residual = st->initial_residual;
  copyv(s->best, x, n);
  if (s->o.kind != 0) {
    memset(s->scalars, 0, sizeof s->scalars);  /* solver_limits writes all 24 slots */
    store_pair(s->scalars + 20, target * target);
    store_pair(s->scalars + 22, 1e6 * st->initial_residual * st->initial_residual);
  }
  ko_scalar(9, s->scalars, s->status, 0);
  if (s->o.kind == 0) {
    for (int i = 0; i < c->max_iter; ++i) {
      apply(s, s->r, &s->z);
      for (int k = 0; k < n; ++k) x[k] = x[k] + (2.0f / 3.0f) * s->z[k];
      s->verified_current = 0;
      ++st->iterations;
      if (st->iterations % c->interval == 0 || st->iterations == c->max_iter) {
        if (verified(s, x, b, target, st) || diverged(st)) break;
      } else residual(s, x, b, s->r);
    }
  } else if (s->o.kind == 1 || s->o.kind == 3) pcg(s, x, b, c, target, st);
  else bicgstab(s, x, b, c, target, st);
  if (!s->verified_current || s->nullspace) verified(s, x, b, target, st);
  if (!isfinite(st->final_residual) || st->final_residual > s->best_residual) {
    copyv(x, s->best, n);
    verified(s, x, b, target, st);
  }
  s->previous_iterations = st->converged ? st->iterations : 0;
  g_jump = saved;
  return 0;
}

/* ----------------------------------------------------- FP64 oracle ---- */
/* Conjugate gradients in double on the double-valued matrix (the independent
 * double reference of tests/linalg/matrices.hpp:89-105, with Jacobi scaling),
 * parallel over rows with OpenMP; stops at ||r|| <= rel_tol ||b||. */
int ko_cg64(int n, const int* row_ptr, const int* col, const double* val, const double* b,
            double* x, double rel_tol, int max_iter, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  double *r = malloc(sizeof(double) * (size_t)(n ? n : 1)), *z = malloc(sizeof(double) * (size_t)(n ? n : 1));
  double *p = malloc(sizeof(double) * (size_t)(n ? n : 1)), *q = malloc(sizeof(double) * (size_t)(n ? n : 1));
  double* dinv = malloc(sizeof(double) * (size_t)(n ? n : 1));
  if (!r || !z || !p || !q || !dinv) { free(r); free(z); free(p); free(q); free(dinv); return -1; }
  double bb = 0;
#pragma omp parallel for reduction(+ : bb)
  for (int i = 0; i < n; ++i) {
    x[i] = 0; r[i] = b[i]; bb += b[i] * b[i];
    double d = 0;
    for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j) if (col[j] == i) d = val[j];
    dinv[i] = d != 0 ? 1.0 / d : 1.0;
    z[i] = dinv[i] * r[i]; p[i] = z[i];
  }
  double rz = 0;
#pragma omp parallel for reduction(+ : rz)
  for (int i = 0; i < n; ++i) rz += r[i] * z[i];
  double limit = rel_tol * rel_tol * bb;
  int it = 0;
  for (; it < max_iter; ++it) {
    double pq = 0;
#pragma omp parallel for reduction(+ : pq)
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j) s += val[j] * p[col[j]];
      q[i] = s; pq += p[i] * s;
    }
    double alpha = rz / pq, rr = 0, rz2 = 0;
#pragma omp parallel for reduction(+ : rr, rz2)
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i]; r[i] -= alpha * q[i]; z[i] = dinv[i] * r[i];
      rr += r[i] * r[i]; rz2 += r[i] * z[i];
    }
    if (rr <= limit) { ++it; break; }
    double beta = rz2 / rz;
    rz = rz2;
#pragma omp parallel for
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  free(r); free(z); free(p); free(q); free(dinv);
  return it;
}

double ko_true_residual(int n, const int* row_ptr, const int* col, const double* val,
                        const double* b, const float* x) {
  double total = 0;
#pragma omp parallel for reduction(+ : total)
  for (int i = 0; i < n; ++i) {
    double s = b[i];
    for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j) s -= val[j] * (double)x[col[j]];
    total += s * s;
  }
  return sqrt(total);
}
