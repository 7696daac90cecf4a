// extern "C" boundary (include/kutta_b200.h): status codes, thread-local error
// text, and the mapping of the reference's linalg entry points onto kb2::Solver.
#include "kutta_b200.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "cuda/kernels.hpp"
#include "host/coupled.hpp"
#include "host/coupled_setup.hpp"
#include "host/mixed.hpp"
#include "host/setup.hpp"

static_assert(B2_LEARNED_CYCLE == kb2::Solver::kLearnedCycle &&
                  B2_LEARNED_WARM_START == kb2::Solver::kLearnedWarmStart,
              "learned-stage mode bits");
#include "host/solver.hpp"

struct b2_workspace {
  std::shared_ptr<kb2::Workspace> w;
};
struct b2_solver {
  std::unique_ptr<kb2::Solver> s;
};
struct b2_hierarchy {
  kb2::Hierarchy h;
  kb2::HostCsr fine;
};
struct b2_mixed {
  std::unique_ptr<kb2::MixedSolver> s;
};
struct b2_coupled {
  std::unique_ptr<kb2::CoupledSolver> s;
};
struct b2_coupled_setup {
  kb2::CoupledSetup s;
};
struct b2_gnn {
  std::unique_ptr<kb2::Gnn> g;
};

namespace {
thread_local std::string g_error;

int fail(int code, const char* message) {
  g_error = message;
  return code;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return B2_OK;
  } catch (const kb2::NonfiniteError& e) {
    return fail(B2_NONFINITE, e.what());
  } catch (const kb2::TimeoutError& e) {
    return fail(B2_TIMEOUT, e.what());
  } catch (const kb2::DeviceError& e) {
    const bool oom = std::strstr(e.what(), "out of device memory") != nullptr;
    return fail(oom ? B2_OUT_OF_MEMORY : B2_DEVICE_ERROR, e.what());
  } catch (const kb2::Error& e) {
    return fail(B2_INVALID_ARGUMENT, e.what());
  } catch (const std::bad_alloc&) {
    return fail(B2_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(B2_INTERNAL, e.what());
  }
}

kb2::Options to_options(const b2_options* o) {
  kb2::Options r;
  if (!o) return r;
  r.cycle = o->cycle == B2_CYCLE_K ? kb2::Cycle::K : kb2::Cycle::V;
  KB2_REQUIRE(o->cycle == B2_CYCLE_V || o->cycle == B2_CYCLE_K, "AMG: invalid options");
  r.pre_sweeps = o->pre_sweeps;
  r.post_sweeps = o->post_sweeps;
  r.coarse_sweeps = o->coarse_sweeps;
  r.coarse_rows = o->coarse_rows;
  r.max_levels = o->max_levels;
  r.aggregation_passes = o->aggregation_passes;
  r.strength_threshold = o->strength_threshold;
  KB2_REQUIRE(o->nullspace == B2_NULLSPACE_NONE || o->nullspace == B2_NULLSPACE_CONSTANT,
              "solver: invalid nullspace option");
  r.nullspace = o->nullspace == B2_NULLSPACE_CONSTANT;
  KB2_REQUIRE(o->structure == B2_STRUCTURE_GENERAL || o->structure == B2_STRUCTURE_SYMMETRIC_M_MATRIX,
              "AMG: invalid operator structure");
  r.m_matrix = o->structure == B2_STRUCTURE_SYMMETRIC_M_MATRIX;
  KB2_REQUIRE(o->setup == B2_SETUP_HOST || o->setup == B2_SETUP_DEVICE, "AMG: invalid setup option");
  r.device_setup = o->setup == B2_SETUP_DEVICE;
  return r;
}

kb2::Options mixed_options(const b2_mixed_options& m) {
  auto o = to_options(&m.amg);
  o.absorb_singletons = m.absorb_singletons != 0;
  KB2_REQUIRE(m.dense_rows >= 1 && m.dense_rows <= 4096, "mixed: dense_rows must be in [1, 4096]");
  o.coarse_rows = m.dense_rows;
  return o;
}

kb2::CsrView view(int n, int nnz, const int32_t* row_ptr, const int32_t* col, const int32_t* diag,
                  const double* val) {
  KB2_REQUIRE(n >= 0 && nnz >= 0 && row_ptr != nullptr, "CSR: invalid array sizes");
  return kb2::CsrView{n, nnz, row_ptr, col, diag, val};
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }
}  // namespace

namespace kb2 {
// Sets the text b2_last_error() returns, for entry points defined in other
// translation units.
int report_error(int code, const char* message) { return fail(code, message); }
}  // namespace kb2

// Coupled-solve argument conversion (used by the b2_coupled_* entry points).
namespace {
kb2::CoupledMeshHost coupled_mesh(const b2_coupled_mesh* m) {
  KB2_REQUIRE(m != nullptr, "coupled: null mesh");
  kb2::CoupledMeshHost h;
  h.n_cells = m->n_cells;
  h.n_faces = m->n_faces;
  h.n_internal = m->n_internal;
  h.owner = m->owner;
  h.neighbour = m->neighbour;
  h.cell_face_offsets = m->cell_face_offsets;
  h.cell_faces = m->cell_faces;
  h.cell_face_sign = m->cell_face_sign;
  h.adjacent = m->adjacent;
  h.area_x = m->area_x;
  h.area_y = m->area_y;
  h.area_z = m->area_z;
  h.face_area = m->face_area;
  h.cell_centroid = m->cell_centroid;
  h.owner_to_face_x = m->owner_to_face_x;
  h.owner_to_face_y = m->owner_to_face_y;
  h.owner_to_face_z = m->owner_to_face_z;
  h.neighbour_to_face_x = m->neighbour_to_face_x;
  h.neighbour_to_face_y = m->neighbour_to_face_y;
  h.neighbour_to_face_z = m->neighbour_to_face_z;
  h.lsq_x = m->lsq_x;
  h.lsq_y = m->lsq_y;
  h.lsq_z = m->lsq_z;
  h.boundary_delta_x = m->boundary_delta_x;
  h.boundary_delta_y = m->boundary_delta_y;
  h.boundary_delta_z = m->boundary_delta_z;
  h.lsq_inverse = m->lsq_inverse;
  h.diffusion = m->diffusion;
  h.volume = m->volume;
  h.boundary_kind = m->boundary_kind;
  h.pattern_row_ptr = m->pattern_row_ptr;
  h.pattern_col = m->pattern_col;
  h.pattern_diag = m->pattern_diag;
  h.low_order = m->low_order;
  return h;
}
kb2::CoupledOptions coupled_options(const b2_coupled_options* o) {
  b2_coupled_options defaults;
  b2_coupled_options_default(&defaults);
  const b2_coupled_options& c = o ? *o : defaults;
  kb2::CoupledOptions r;
  r.pre_sweeps = c.pre_sweeps;
  r.post_sweeps = c.post_sweeps;
  r.coarsest_sweeps = c.coarsest_sweeps;
  r.smoother_damping = c.smoother_damping;
  r.courant = c.courant;
  r.coarsest_rows = c.coarsest_rows;
  r.aggregation_passes = c.aggregation_passes;
  r.recompute = c.recompute;
  return r;
}
kb2::CoupledSolver& coupled(b2_coupled* s) {
  KB2_REQUIRE(s && s->s, "coupled: null solver");
  return *s->s;
}
const kb2::CoupledSolver& coupled_view(const b2_coupled* s) {
  KB2_REQUIRE(s && s->s, "coupled: null solver");
  return *s->s;
}
template <class T>
void read_back(T* out, const T* d, std::size_t n, cudaStream_t s) {
  if (!out || n == 0) return;
  kb2::cuda_check(cudaMemcpyAsync(out, d, n * sizeof(T), cudaMemcpyDeviceToHost, s), "read back");
}
}  // namespace

extern "C" {

void b2_options_default(b2_options* o) {
  if (!o) return;
  o->cycle = B2_CYCLE_V;
  o->pre_sweeps = 5;
  o->post_sweeps = 5;
  o->coarse_sweeps = 32;
  o->coarse_rows = 24;
  o->max_levels = 24;
  o->aggregation_passes = 3;
  o->strength_threshold = 0.25;
  o->nullspace = B2_NULLSPACE_NONE;
  o->structure = B2_STRUCTURE_GENERAL;
  o->workspace = nullptr;
  o->setup = B2_SETUP_DEVICE;
}

void b2_control_default(b2_control* c) {
  if (!c) return;
  c->rel_tol = 1e-2;
  c->abs_tol = 1e-12;
  c->max_iter = 200;
  c->residual_check_interval = 8;
}

size_t b2_last_error(char* buffer, size_t length) {
  if (buffer && length) std::snprintf(buffer, length, "%s", g_error.c_str());
  return g_error.size();
}

int b2_workspace_create(int rows, b2_workspace** out) {
  return guarded([&] {
    KB2_REQUIRE(out != nullptr && rows >= 0, "workspace: invalid arguments");
    *out = new b2_workspace{std::make_shared<kb2::Workspace>(rows)};
  });
}
void b2_workspace_destroy(b2_workspace* w) { delete w; }

int b2_solver_create(int kind, int n, int nnz, const int32_t* row_ptr, const int32_t* col,
                     const int32_t* diag, const double* val, const b2_options* options,
                     int use_amg_options, b2_solver** out) {
  return guarded([&] {
    KB2_REQUIRE(out != nullptr, "solver: null output handle");
    *out = nullptr;
    KB2_REQUIRE(kind >= B2_JACOBI && kind <= B2_AMG_BICGSTAB, "unknown SolverKind");
    const auto k = static_cast<kb2::Kind>(kind);
    const bool amg_factory = options && use_amg_options;
    const bool amg_kind = k == kb2::Kind::AmgPcg || k == kb2::Kind::AmgBicgstab;
    // make_amg_solver checks the kind first (amg.cpp:347-348).
    KB2_REQUIRE(amg_kind || !amg_factory, "AMG: expected an AMG solver kind");
    const auto a = view(n, nnz, row_ptr, col, diag, val);
    kb2::Options o;
    if (amg_factory) {
      o = to_options(options);
    } else if (options) {
      // make_solver: AMG defaults with only nullspace and structure taken over
      // (amg.cpp:388-396), and where the hierarchy is built.
      const auto given = to_options(options);
      o.nullspace = given.nullspace;
      o.m_matrix = given.m_matrix;
      o.device_setup = given.device_setup;
    }
    std::shared_ptr<kb2::Workspace> ws = options && options->workspace ? options->workspace->w : nullptr;
    if (amg_kind) {
      kb2::check_amg(k, a, o);
    } else {
      kb2::validate_host(a);
      o.m_matrix = false;
    }
    // The reference's last host checks before device work (krylov_solver,
    // solver.cpp:396-406): the workspace size, then the Jacobi kinds' diagonal
    // (Jacobi ctor, solver.cpp:56-60 -> diagonal_values :37-53).
    KB2_REQUIRE(!ws || ws->rows() == n, "Krylov workspace size mismatch");
    if (!amg_kind) (void)kb2::diagonal_values(a, false, false);
    auto solver = std::make_unique<kb2::Solver>(k, a, o, ws);
    *out = new b2_solver{std::move(solver)};
  });
}

int b2_solver_refresh(b2_solver* s, const float* d_val, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    KB2_REQUIRE(d_val != nullptr || s->s->entries() == 0, "solver: device or matrix mismatch");
    s->s->refresh(d_val, as_stream(stream));
  });
}

int b2_solver_solve(b2_solver* s, const float* d_val, float* d_x, const float* d_b,
                    const b2_control* control, b2_stats* stats, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    KB2_REQUIRE(d_val != nullptr || s->s->entries() == 0, "solver: device or matrix mismatch");
    kb2::Control c;
    if (control) {
      c.rel_tol = control->rel_tol;
      c.abs_tol = control->abs_tol;
      c.max_iter = control->max_iter;
      c.residual_check_interval = control->residual_check_interval;
    }
    const auto r = s->s->solve(d_val, d_x, d_b, c, as_stream(stream));
    if (stats) {
      stats->iterations = r.iterations;
      stats->converged = r.converged ? 1 : 0;
      stats->initial_residual = r.initial_residual;
      stats->final_residual = r.final_residual;
    }
  });
}

size_t b2_solver_describe(const b2_solver* s, char* buffer, size_t length) {
  if (!s || !s->s) return 0;
  const auto d = s->s->describe();
  if (buffer && length) std::snprintf(buffer, length, "%s", d.c_str());
  return d.size();
}

void b2_solver_destroy(b2_solver* s) { delete s; }

int b2_csr_spmv(int n, int nnz, const int32_t* d_row_ptr, const int32_t* d_col,
                const float* d_val, const float* d_x, float* d_y, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(n >= 0 && nnz >= 0, "CSR: invalid array sizes");
    if (n == 0) return;  // nothing to compute, nothing queued
    KB2_REQUIRE(d_row_ptr && d_x && d_y && (nnz == 0 || (d_col && d_val)), "CSR: null argument");
    KB2_REQUIRE(d_x != d_y, "CSR: input/output aliasing is unsupported");
    kb2::launch::spmv(n, d_row_ptr, d_col, d_val, d_x, d_y, nullptr, as_stream(stream));
    kb2::cuda_check(cudaGetLastError(), "csr_spmv");
  });
}

int b2_csr_residual(int n, int nnz, const int32_t* d_row_ptr, const int32_t* d_col,
                    const float* d_val, const float* d_x, const float* d_b, float* d_r,
                    void* stream) {
  return guarded([&] {
    KB2_REQUIRE(n >= 0 && nnz >= 0, "CSR: invalid array sizes");
    if (n == 0) return;
    KB2_REQUIRE(d_row_ptr && d_x && d_b && d_r && (nnz == 0 || (d_col && d_val)),
                "CSR: null argument");
    KB2_REQUIRE(d_x != d_r && d_b != d_r, "CSR: residual RHS size or alias mismatch");
    kb2::launch::residual(n, d_row_ptr, d_col, d_val, d_x, d_b, d_r, nullptr, as_stream(stream));
    kb2::cuda_check(cudaGetLastError(), "csr_residual");
  });
}

int b2_solver_profile(b2_solver* s, int enable) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    s->s->set_profile(enable != 0);
  });
}

int b2_solver_profile_read(b2_solver* s, b2_profile* out) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s && out, "solver: null handle");
    const auto p = s->s->profile();
    out->launches = p.launches;
    out->fine_sweeps = p.fine_sweeps;
    out->fine_sweep_ms = p.fine_sweep_ms;
    out->fine_sweep_bytes = p.fine_sweep_bytes;
    out->algorithmic_bytes = p.algorithmic_bytes;
    out->solves = p.solves;
  });
}

long long b2_kernel_launches(void) { return kb2::launch::counter.load(); }

int b2_amg_smooth(int n, const int32_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                  const float* d_x, const float* d_b, const float* d_inverse, float* d_next,
                  int zero_start, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(n >= 0, "CSR: invalid array sizes");
    if (n == 0) return;
    // Every row holds its diagonal, so col and val are never empty; a zero
    // start does not read x.
    KB2_REQUIRE(d_row_ptr && d_col && d_val && d_b && d_inverse && d_next &&
                    (zero_start || d_x),
                "smooth: null argument");
    KB2_REQUIRE(d_next != d_x && d_next != d_b, "smooth: output aliases an input");
    kb2::launch::smooth(n, d_row_ptr, d_col, d_val, d_x, d_b, d_inverse, d_next, nullptr,
                        zero_start != 0, as_stream(stream));
    kb2::cuda_check(cudaGetLastError(), "amg_smooth");
  });
}

int b2_solver_levels(const b2_solver* s) { return s && s->s ? s->s->levels() : 0; }

int b2_solver_level_shape(const b2_solver* s, int level, int* n, int* nnz) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s && level >= 0 && level < s->s->levels(), "level out of range");
    const auto& l = s->s->level(level);
    if (n) *n = l.n;
    if (nnz) *nnz = l.nnz;
  });
}

int b2_solver_level_copy(const b2_solver* s, int level, int32_t* row_ptr, int32_t* col,
                         float* val, float* inverse_l1, int32_t* aggregate, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s && level >= 0 && level < s->s->levels(), "level out of range");
    const auto& l = s->s->level(level);
    const auto st = as_stream(stream);
    auto get = [&](void* dst, const void* src, std::size_t bytes) {
      if (dst && src && bytes)
        kb2::cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), "level copy");
    };
    get(row_ptr, l.row_ptr.get(), sizeof(int) * (static_cast<std::size_t>(l.n) + 1));
    get(col, l.col.get(), sizeof(int) * static_cast<std::size_t>(l.nnz));
    const float* values = level == 0 ? s->s->current_values() : l.val.get();
    get(val, values, sizeof(float) * static_cast<std::size_t>(l.nnz));
    if (l.l1.allocated()) get(inverse_l1, l.l1.get(), sizeof(float) * static_cast<std::size_t>(l.n));
    if (l.aggregate.allocated())
      get(aggregate, l.aggregate.get(), sizeof(int) * static_cast<std::size_t>(l.n));
    kb2::wait(st);
  });
}

int b2_fv_pressure_assemble(int n, const int32_t* offsets, const int32_t* faces, const float* sign,
                            const int32_t* adjacent, const int32_t* entry, const int32_t* rows,
                            const int32_t* diag, const float* coefficient, const float* flux,
                            float* values, float* rhs, int reference, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(n >= 0, "assemble: negative cell count");
    KB2_REQUIRE(n == 0 || (offsets && faces && sign && adjacent && entry && rows && diag &&
                           coefficient && flux && values && rhs),
                "assemble: null argument");
    KB2_REQUIRE(reference >= -1 && reference < n, "assemble: reference cell out of range");
    if (n == 0) return;
    kb2::launch::fv_pressure_assemble(n, offsets, faces, sign, adjacent, entry, rows, diag,
                                      coefficient, flux, values, rhs, reference,
                                      as_stream(stream));
    kb2::cuda_check(cudaGetLastError(), "fv_pressure_assemble");
  });
}

int b2_fv_correct_flux(int n_faces, const int32_t* owner, const int32_t* neighbour,
                       const float* correction, const float* coefficient, float* flux,
                       int internal, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(n_faces >= 0 && internal >= 0 && internal <= n_faces,
                "correct_flux: invalid face counts");
    KB2_REQUIRE(n_faces == 0 || (owner && (neighbour || internal == 0) && correction &&
                                 coefficient && flux),
                "correct_flux: null argument");
    if (n_faces == 0) return;
    kb2::launch::fv_correct_flux(n_faces, owner, neighbour, correction, coefficient, flux,
                                 internal, as_stream(stream));
    kb2::cuda_check(cudaGetLastError(), "fv_correct_flux");
  });
}

int b2_fv_correct_velocity(int n, const float* volume, const float* inverse, const float* diagonal,
                           const float* gx, const float* gy, const float* gz,
                           const float* correction, float* u, float* v, float* w, float* p,
                           float alpha, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(n >= 0, "correct_velocity: negative cell count");
    KB2_REQUIRE(n == 0 || (volume && inverse && diagonal && gx && gy && gz && correction && u &&
                           v && w && p),
                "correct_velocity: null argument");
    if (n == 0) return;
    kb2::launch::fv_correct_velocity(n, volume, inverse, diagonal, gx, gy, gz, correction, u, v, w,
                                     p, alpha, as_stream(stream));
    kb2::cuda_check(cudaGetLastError(), "fv_correct_velocity");
  });
}

namespace {
kb2::FvPressure fv_pressure(const int32_t* offsets, const int32_t* faces, const float* sign,
                            const int32_t* adjacent, const int32_t* entry,
                            const float* coefficient, const float* flux, int reference) {
  kb2::FvPressure fv;
  fv.offsets = offsets;
  fv.faces = faces;
  fv.sign = sign;
  fv.adjacent = adjacent;
  fv.entry = entry;
  fv.coefficient = coefficient;
  fv.flux = flux;
  fv.reference = reference;
  return fv;
}
}  // namespace

int b2_solver_assemble_refresh(b2_solver* s, const int32_t* offsets, const int32_t* faces,
                               const float* sign, const int32_t* adjacent, const int32_t* entry,
                               const float* coefficient, const float* flux, float* values,
                               float* rhs, int reference, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    s->s->assemble_refresh(
        fv_pressure(offsets, faces, sign, adjacent, entry, coefficient, flux, reference), values,
        rhs, as_stream(stream));
  });
}

int b2_mixed_assemble_refresh(b2_mixed* s, const int32_t* offsets, const int32_t* faces,
                              const float* sign, const int32_t* adjacent, const int32_t* entry,
                              const float* coefficient, const float* flux, float* values,
                              float* rhs, int reference, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    s->s->assemble_refresh(
        fv_pressure(offsets, faces, sign, adjacent, entry, coefficient, flux, reference), values,
        rhs, as_stream(stream));
  });
}

int b2_solver_level_transfer(const b2_solver* s, int level, int32_t* diag, int32_t* member_offsets,
                             int32_t* members, int32_t* entry_offsets, int32_t* entries,
                             void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s && level >= 0 && level < s->s->levels(), "level out of range");
    const auto& l = s->s->level(level);
    const auto st = as_stream(stream);
    auto get = [&](void* dst, const kb2::DArray<int>& src, std::size_t count) {
      if (dst && src.allocated() && count)
        kb2::cuda_check(cudaMemcpyAsync(dst, src.get(), sizeof(int) * count,
                                        cudaMemcpyDeviceToHost, st),
                        "level copy");
    };
    get(diag, l.diag, static_cast<std::size_t>(l.n));
    if (level + 1 < s->s->levels()) {
      const auto& c = s->s->level(level + 1);
      get(member_offsets, l.member_offsets, static_cast<std::size_t>(c.n) + 1);
      get(members, l.members, l.members.size());
      get(entry_offsets, l.entry_offsets, static_cast<std::size_t>(c.nnz) + 1);
      get(entries, l.entries, l.entries.size());
    }
    kb2::wait(st);
  });
}

int b2_hierarchy_build(int n, int nnz, const int32_t* row_ptr, const int32_t* col,
                       const int32_t* diag, const double* val, const b2_options* options,
                       int spd, b2_hierarchy** out) {
  return guarded([&] {
    KB2_REQUIRE(out != nullptr, "hierarchy: null output handle");
    *out = nullptr;
    const auto a = view(n, nnz, row_ptr, col, diag, val);
    const auto o = to_options(options);
    kb2::check_amg(spd ? kb2::Kind::AmgPcg : kb2::Kind::AmgBicgstab, a, o);
    auto h = std::make_unique<b2_hierarchy>();
    h->h = kb2::build_hierarchy(a, o);
    h->fine.n = n;
    h->fine.row_ptr.assign(row_ptr, row_ptr + n + 1);
    h->fine.col.assign(col, col + nnz);
    h->fine.diag.assign(diag, diag + n);
    h->fine.val.assign(val, val + nnz);
    *out = h.release();
  });
}

int b2_hierarchy_levels(const b2_hierarchy* h) { return h ? static_cast<int>(h->h.levels.size()) : 0; }

int b2_hierarchy_level_shape(const b2_hierarchy* h, int level, int* n, int* nnz) {
  return guarded([&] {
    KB2_REQUIRE(h && level >= 0 && level < b2_hierarchy_levels(h), "level out of range");
    const auto& m = level == 0 ? h->fine : h->h.levels[level].matrix;
    if (n) *n = m.n;
    if (nnz) *nnz = m.nnz();
  });
}

int b2_hierarchy_level_copy(const b2_hierarchy* h, int level, int32_t* row_ptr, int32_t* col,
                            float* val, float* inverse_l1, int32_t* aggregate) {
  return guarded([&] {
    KB2_REQUIRE(h && level >= 0 && level < b2_hierarchy_levels(h), "level out of range");
    const auto& l = h->h.levels[level];
    const auto& m = level == 0 ? h->fine : l.matrix;
    if (row_ptr) std::memcpy(row_ptr, m.row_ptr.data(), sizeof(int) * m.row_ptr.size());
    if (col) std::memcpy(col, m.col.data(), sizeof(int) * m.col.size());
    if (val)
      for (std::size_t j = 0; j < m.val.size(); ++j) val[j] = static_cast<float>(m.val[j]);
    if (inverse_l1) std::memcpy(inverse_l1, l.l1.data(), sizeof(float) * l.l1.size());
    if (aggregate && !l.transfer.aggregate.empty())
      std::memcpy(aggregate, l.transfer.aggregate.data(), sizeof(int) * l.transfer.aggregate.size());
  });
}

void b2_hierarchy_free(b2_hierarchy* h) { delete h; }

void b2_mixed_options_default(b2_mixed_options* o) {
  if (!o) return;
  b2_options_default(&o->amg);
  o->amg.structure = B2_STRUCTURE_SYMMETRIC_M_MATRIX;
  o->amg.cycle = B2_CYCLE_K;
  o->amg.pre_sweeps = o->amg.post_sweeps = 1;
  o->absorb_singletons = 1;
  o->dense_rows = 112;  // the largest coarsest level inverted on chip
  o->coarse_bf16 = 1;
  o->inner_rel_tol = 1e-3;
  o->inner_max_iter = 300;
  o->max_refinements = 30;
  o->fused_coarse = 0;
  o->k_cycle_levels = 1;
  o->cuda_graphs = 1;
  o->packed_rows = 1;
}

int b2_mixed_create(int n, int nnz, const int32_t* row_ptr, const int32_t* col,
                    const int32_t* diag, const double* val, const b2_mixed_options* options,
                    b2_mixed** out) {
  return guarded([&] {
    KB2_REQUIRE(out != nullptr, "solver: null output handle");
    *out = nullptr;
    b2_mixed_options defaults;
    b2_mixed_options_default(&defaults);
    const b2_mixed_options& m = options ? *options : defaults;
    const auto a = view(n, nnz, row_ptr, col, diag, val);
    kb2::MixedOptions o;
    o.amg = mixed_options(m);
    o.amg.coarse_bf16 = m.coarse_bf16 != 0;
    o.amg.dense_coarsest = true;
    o.amg.fused_tail = m.fused_coarse != 0;
    o.amg.graphs = m.cuda_graphs != 0;
    o.amg.packed_fine = m.packed_rows != 0;
    KB2_REQUIRE(m.k_cycle_levels >= 0, "mixed: k_cycle_levels must be >= 0");
    o.amg.k_levels = m.k_cycle_levels;
    KB2_REQUIRE(std::isfinite(m.inner_rel_tol) && m.inner_rel_tol > 0 && m.inner_rel_tol < 1 &&
                    m.inner_max_iter > 0 && m.max_refinements > 0,
                "mixed: invalid refinement options");
    o.inner_rel_tol = m.inner_rel_tol;
    o.inner_max_iter = m.inner_max_iter;
    o.max_refinements = m.max_refinements;
    kb2::check_amg(kb2::Kind::AmgPcg, a, o.amg);
    *out = new b2_mixed{std::make_unique<kb2::MixedSolver>(a, o)};
  });
}

int b2_mixed_refresh(b2_mixed* s, const float* d_val, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    s->s->refresh(d_val, as_stream(stream));
  });
}

namespace {
kb2::Control control_of(const b2_control* control) {
  kb2::Control c;
  if (control) {
    c.rel_tol = control->rel_tol;
    c.abs_tol = control->abs_tol;
    c.max_iter = control->max_iter;
    c.residual_check_interval = control->residual_check_interval;
  }
  return c;
}

void put_stats(const kb2::MixedStats& r, b2_mixed_stats* stats) {
  if (!stats) return;
  stats->refinements = r.refinements;
  stats->learned_fallback = r.learned_fallback ? 1 : 0;
  stats->iterations = r.iterations;
  stats->converged = r.converged ? 1 : 0;
  stats->initial_residual = r.initial_residual;
  stats->final_residual = r.final_residual;
}
}  // namespace

int b2_mixed_solve(b2_mixed* s, const float* d_val, double* d_x, const float* d_b,
                   const b2_control* control, b2_mixed_stats* stats, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    put_stats(s->s->solve(d_val, d_x, d_b, control_of(control), as_stream(stream)), stats);
  });
}

int b2_mixed_solve_f32(b2_mixed* s, const float* d_val, float* d_x, const float* d_b,
                       const b2_control* control, b2_mixed_stats* stats, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    put_stats(s->s->solve32(d_val, d_x, d_b, control_of(control), as_stream(stream)), stats);
  });
}

size_t b2_mixed_describe(const b2_mixed* s, char* buffer, size_t length) {
  if (!s || !s->s) return 0;
  const auto d = s->s->describe();
  if (buffer && length) std::snprintf(buffer, length, "%s", d.c_str());
  return d.size();
}

void b2_mixed_destroy(b2_mixed* s) { delete s; }

int b2_dense_inverse(int n, const int32_t* d_row_ptr, const int32_t* d_col, const float* d_val,
                     double* d_inverse, double* d_not_spd, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(n >= 1 && n <= 1024, "dense inverse: n must be in [1, 1024]");
    KB2_REQUIRE(d_row_ptr && d_col && d_val && d_inverse && d_not_spd,
                "dense inverse: null argument");
    const auto st = as_stream(stream);
    double* lower = nullptr;
    kb2::cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&lower),
                                    sizeof(double) * static_cast<std::size_t>(n) * n, st),
                    "cudaMallocAsync");
    kb2::launch::dense_inverse(n, d_row_ptr, d_col, d_val, lower, d_inverse, d_not_spd, st);
    const cudaError_t launched = cudaGetLastError();
    kb2::cuda_check(cudaFreeAsync(lower, st), "cudaFreeAsync");
    kb2::cuda_check(launched, "dense_inverse");
  });
}

int b2_mixed_profile(b2_mixed* s, int enable) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    s->s->inner().set_profile(enable != 0);
  });
}

int b2_gnn_create(uint64_t seed, b2_gnn** out) {
  return guarded([&] {
    KB2_REQUIRE(out != nullptr, "learned stage: null output handle");
    *out = nullptr;
    *out = new b2_gnn{std::make_unique<kb2::Gnn>(seed)};
  });
}

void b2_gnn_destroy(b2_gnn* g) { delete g; }

int b2_gnn_parameter_count(void) { return kb2::Gnn::parameter_count(); }

int b2_gnn_bind(b2_gnn* g, int n, const int32_t* d_row_ptr, const int32_t* d_col,
                const int32_t* d_diag, const float* d_val, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(g && g->g, "learned stage: null handle");
    g->g->bind(n, d_row_ptr, d_col, d_diag, d_val, as_stream(stream));
  });
}

int b2_gnn_apply(b2_gnn* g, const float* d_r, float* d_z, float beta, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(g && g->g && d_r && d_z, "learned stage: null argument");
    KB2_REQUIRE(beta == 0.0f || beta == 1.0f, "learned stage: beta must be 0 or 1");
    g->g->forward(d_r, d_z, beta, as_stream(stream));
    g->g->check(as_stream(stream));
  });
}

int b2_gnn_set_wait_limit(b2_gnn* g, long long polls) {
  return guarded([&] {
    KB2_REQUIRE(g && g->g, "learned stage: null argument");
    g->g->set_wait_polls(polls);
  });
}

int b2_gnn_train_step(b2_gnn* g, const float* d_t, const float* d_e, float learning_rate,
                      float* loss, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(g && g->g && d_t && d_e, "learned stage: null argument");
    KB2_REQUIRE(learning_rate > 0 && std::isfinite(learning_rate),
                "learned stage: invalid learning rate");
    const float l = g->g->train_step(d_t, d_e, learning_rate, as_stream(stream));
    if (loss) *loss = l;
  });
}

int b2_gnn_gradient(b2_gnn* g, const float* d_t, const float* d_e, int tensor_cores,
                    float* host_gradient, size_t count, float* loss, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(g && g->g && d_t && d_e && host_gradient, "learned stage: null argument");
    KB2_REQUIRE(count == static_cast<size_t>(kb2::Gnn::parameter_count()),
                "learned stage: wrong number of weights");
    const auto grad = g->g->gradient(d_t, d_e, tensor_cores != 0, loss, as_stream(stream));
    std::memcpy(host_gradient, grad.data(), sizeof(float) * grad.size());
  });
}

int b2_gnn_set_geometry(b2_gnn* g, const float* d_geometry) {
  return guarded([&] {
    KB2_REQUIRE(g && g->g, "learned stage: null argument");
    g->g->set_geometry(d_geometry);
  });
}

int b2_gnn_get_weights(const b2_gnn* g, float* host, size_t count) {
  return guarded([&] {
    KB2_REQUIRE(g && g->g && host, "learned stage: null argument");
    const auto w = g->g->weights();
    KB2_REQUIRE(count == w.size(), "learned stage: wrong number of weights");
    std::memcpy(host, w.data(), sizeof(float) * w.size());
  });
}

int b2_gnn_set_weights(b2_gnn* g, const float* host, size_t count) {
  return guarded([&] {
    KB2_REQUIRE(g && g->g && host, "learned stage: null argument");
    g->g->set_weights(std::vector<float>(host, host + count));
  });
}

int b2_mixed_set_learned(b2_mixed* s, b2_gnn* g, int mode) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s, "solver: null handle");
    s->s->inner().set_learned(g ? g->g.get() : nullptr, mode);
  });
}

int b2_mixed_precondition(b2_mixed* s, const float* d_val, const float* d_r, float* d_z,
                          void* stream) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s && d_val, "solver: null argument");
    s->s->inner().precondition_into(d_val, d_r, d_z, as_stream(stream));
  });
}

int b2_mixed_profile_read(b2_mixed* s, b2_profile* out) {
  return guarded([&] {
    KB2_REQUIRE(s && s->s && out, "solver: null handle");
    const auto p = s->s->inner().profile();
    out->launches = p.launches;
    out->fine_sweeps = p.fine_sweeps;
    out->fine_sweep_ms = p.fine_sweep_ms;
    out->fine_sweep_bytes = p.fine_sweep_bytes;
    out->algorithmic_bytes = p.algorithmic_bytes;
    out->solves = p.solves;
  });
}

int b2_mixed_hierarchy_build(int n, int nnz, const int32_t* row_ptr, const int32_t* col,
                             const int32_t* diag, const double* val,
                             const b2_mixed_options* options, b2_hierarchy** out) {
  return guarded([&] {
    KB2_REQUIRE(out != nullptr && options != nullptr, "hierarchy: null argument");
    *out = nullptr;
    const auto a = view(n, nnz, row_ptr, col, diag, val);
    auto o = mixed_options(*options);
    kb2::check_amg(kb2::Kind::AmgPcg, a, o);
    auto h = std::make_unique<b2_hierarchy>();
    h->h = kb2::build_hierarchy(a, o);
    h->fine.n = n;
    h->fine.row_ptr.assign(row_ptr, row_ptr + n + 1);
    h->fine.col.assign(col, col + nnz);
    h->fine.diag.assign(diag, diag + n);
    h->fine.val.assign(val, val + nnz);
    *out = h.release();
  });
}

// ---- Coupled (4x4-block) solve ----------------------------------------------


void b2_coupled_options_default(b2_coupled_options* o) {
  if (!o) return;
  const kb2::CoupledOptions d;
  o->pre_sweeps = d.pre_sweeps;
  o->post_sweeps = d.post_sweeps;
  o->coarsest_sweeps = d.coarsest_sweeps;
  o->smoother_damping = d.smoother_damping;
  o->courant = d.courant;
  o->coarsest_rows = d.coarsest_rows;
  o->aggregation_passes = d.aggregation_passes;
  o->recompute = d.recompute;
}

int b2_coupled_create(const b2_coupled_mesh* mesh, int reference,
                      const b2_coupled_options* options, void* stream, b2_coupled** out) {
  return guarded([&] {
    KB2_REQUIRE(out != nullptr, "coupled: null output handle");
    *out = nullptr;
    auto h = std::make_unique<b2_coupled>();
    h->s = std::make_unique<kb2::CoupledSolver>(coupled_mesh(mesh), reference,
                                                coupled_options(options), as_stream(stream));
    kb2::wait(as_stream(stream));
    *out = h.release();
  });
}

int b2_coupled_capture_diagonal(b2_coupled* s, int component, const int32_t* d_row_ptr,
                                const int32_t* d_diag, const float* d_val,
                                const float* d_physical, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(d_row_ptr && d_diag && d_val && d_physical, "coupled: null diagonal input");
    coupled(s).capture_diagonal(component, d_row_ptr, d_diag, d_val, d_physical,
                                as_stream(stream));
  });
}

int b2_coupled_solve(b2_coupled* s, const b2_coupled_residuals* in, const b2_control* control,
                     b2_stats* stats, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(in != nullptr, "coupled: null residuals");
    kb2::CoupledSolveInputs i;
    i.ru = in->d_ru;
    i.rv = in->d_rv;
    i.rw = in->d_rw;
    i.mass = in->d_mass;
    i.viscosity = in->d_viscosity;
    i.physical_diagonal = in->d_physical_diagonal;
    i.face_weights = in->d_face_weights;
    i.net_outflow = in->d_net_outflow;
    b2_control defaults;
    b2_control_default(&defaults);
    const b2_control& c = control ? *control : defaults;
    kb2::Control k;
    k.rel_tol = c.rel_tol;
    k.abs_tol = c.abs_tol;
    k.max_iter = c.max_iter;
    k.residual_check_interval = c.residual_check_interval;
    const auto r = coupled(s).solve(i, in->density, in->velocity_scale, k, as_stream(stream));
    if (stats) {
      stats->iterations = r.iterations;
      stats->converged = r.converged ? 1 : 0;
      stats->initial_residual = r.initial_residual;
      stats->final_residual = r.final_residual;
    }
  });
}

int b2_coupled_update(b2_coupled* s, float* d_u, float* d_v, float* d_w, float* d_p,
                      double alpha_u, double alpha_p, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(d_u && d_v && d_w && d_p, "coupled: null field");
    coupled(s).update(d_u, d_v, d_w, d_p, alpha_u, alpha_p, as_stream(stream));
  });
}

int b2_coupled_paired_update(b2_coupled* s, float* d_u, float* d_v, float* d_w, float* d_p,
                             float* d_u_lo, float* d_v_lo, float* d_w_lo, float* d_p_lo,
                             double alpha_u, double alpha_p, float velocity_slack,
                             float pressure_slack, void* stream) {
  return guarded([&] {
    KB2_REQUIRE(d_u && d_v && d_w && d_p && d_u_lo && d_v_lo && d_w_lo && d_p_lo,
                "coupled: null field");
    coupled(s).paired_update(d_u, d_v, d_w, d_p, d_u_lo, d_v_lo, d_w_lo, d_p_lo, alpha_u,
                             alpha_p, velocity_slack, pressure_slack, as_stream(stream));
  });
}

size_t b2_coupled_bytes(const b2_coupled* s) { return s && s->s ? s->s->bytes() : 0; }

size_t b2_coupled_describe(const b2_coupled* s, char* buffer, size_t length) {
  if (!s || !s->s) return 0;
  const auto d = s->s->describe();
  if (buffer && length) std::snprintf(buffer, length, "%s", d.c_str());
  return d.size();
}

void b2_coupled_destroy(b2_coupled* s) { delete s; }

long long b2_coupled_copy(const b2_coupled* s, int what, float* out, void* stream) {
  long long count = -1;
  const int rc = guarded([&] {
    const auto& c = coupled_view(s);
    const cudaStream_t st = as_stream(stream);
    const std::size_t n = c.cells();
    if (what == 0 || what == 1) {
      count = static_cast<long long>(4 * n);
      if (!out) return;
      std::vector<float> aos(4 * n);
      read_back(aos.data(), what == 0 ? c.solution() : c.rhs(), 4 * n, st);
      kb2::wait(st);
      for (std::size_t i = 0; i < n; ++i)
        for (int k = 0; k < 4; ++k) out[k * n + i] = aos[4 * i + k];
    } else if (what == 2) {
      count = static_cast<long long>(27 * n);
      if (!out) return;
      read_back(out, c.cell_data(), 20 * n, st);
      std::vector<float> inv(4 * n), inv_h(4 * n);
      c.copy_inverse(inv.data(), inv_h.data(), st);
      kb2::wait(st);
      for (std::size_t i = 0; i < n; ++i) {
        out[20 * n + i] = inv[4 * i];
        out[21 * n + i] = inv[4 * i + 1];
        out[22 * n + i] = inv[4 * i + 2];
        out[23 * n + i] = inv_h[4 * i];
        out[24 * n + i] = inv_h[4 * i + 1];
        out[25 * n + i] = inv_h[4 * i + 2];
        out[26 * n + i] = inv[4 * i + 3];
      }
    } else if (what == 3) {
      count = c.faces();
      if (!out) return;
      read_back(out, c.face_coefficients(), static_cast<std::size_t>(c.faces()), st);
      kb2::wait(st);
    } else {
      KB2_REQUIRE(false, "coupled: unknown array");
    }
  });
  return rc == B2_OK ? count : -1;
}

int b2_coupled_levels(const b2_coupled* s) { return s && s->s ? s->s->levels() : 0; }

int b2_coupled_level_shape(const b2_coupled* s, int level, int* n, int* nnz) {
  return guarded([&] {
    const auto& c = coupled_view(s);
    KB2_REQUIRE(level >= 0 && level < c.levels(), "coupled: level out of range");
    if (n) *n = c.level_rows(level);
    if (nnz) *nnz = level == 0 ? 0 : c.level(level).nnz;
  });
}

int b2_coupled_level_copy(const b2_coupled* s, int level, int32_t* rows, int32_t* cols,
                          int32_t* diag, float* a, float* c_out, float* g, float* h, float* d,
                          int32_t* aggregate, void* stream) {
  return guarded([&] {
    const auto& c = coupled_view(s);
    KB2_REQUIRE(level >= 1 && level < c.levels(), "coupled: level out of range");
    const cudaStream_t st = as_stream(stream);
    const auto& l = c.level(level);
    const std::size_t n = l.n, nnz = l.nnz;
    read_back(rows, l.rows, n + 1, st);
    read_back(cols, l.cols, nnz, st);
    read_back(diag, l.diag, n, st);
    read_back(a, static_cast<const float*>(l.a), nnz, st);
    read_back(c_out, static_cast<const float*>(l.c), nnz, st);
    read_back(g, static_cast<const float*>(l.g), 3 * nnz, st);
    read_back(h, static_cast<const float*>(l.h), 3 * nnz, st);
    read_back(d, static_cast<const float*>(l.d), 11 * n, st);
    read_back(aggregate, c.transfer(level - 1).aggregate,
              static_cast<std::size_t>(c.level_rows(level - 1)), st);
    kb2::wait(st);
  });
}

int b2_coupled_apply(b2_coupled* s, int op, const float* d_x, const float* d_b, float* d_y,
                     void* stream) {
  return guarded([&] {
    auto& c = coupled(s);
    KB2_REQUIRE(d_y && (op == 3 || d_x) && (op == 0 || d_b), "coupled: null vector");
    const cudaStream_t st = as_stream(stream);
    if (op == 0)
      c.apply(d_x, d_y, st);
    else if (op == 1)
      c.residual(d_x, d_b, d_y, st);
    else if (op == 2 || op == 3)
      c.smooth(d_x, d_b, d_y, op == 3, st);
    else
      KB2_REQUIRE(false, "coupled: unknown operator");
    kb2::cuda_check(cudaGetLastError(), "coupled apply");
  });
}

int b2_coupled_level_apply(b2_coupled* s, int level, int op, const float* d_x,
                           const float* d_b, float* d_y, void* stream) {
  return guarded([&] {
    const bool needs_b = op == 1 || op == 2 || op == 3;
    KB2_REQUIRE(d_y && (op == 3 || d_x) && (!needs_b || d_b), "coupled: null vector");
    coupled(s).level_apply(level, op, d_x, d_b, d_y, as_stream(stream));
    kb2::cuda_check(cudaGetLastError(), "coupled level apply");
  });
}

int b2_coupled_setup_build(const b2_coupled_mesh* mesh, const b2_coupled_options* options,
                           b2_coupled_setup** out) {
  return guarded([&] {
    KB2_REQUIRE(out != nullptr, "coupled: null output handle");
    *out = nullptr;
    auto h = std::make_unique<b2_coupled_setup>();
    h->s = kb2::coupled_setup(coupled_mesh(mesh), coupled_options(options));
    *out = h.release();
  });
}

int b2_coupled_setup_levels(const b2_coupled_setup* s) {
  return s ? static_cast<int>(s->s.levels.size()) + 1 : 0;
}

int b2_coupled_setup_level_shape(const b2_coupled_setup* s, int level, int* n, int* nnz) {
  return guarded([&] {
    KB2_REQUIRE(s && level >= 0 && level < b2_coupled_setup_levels(s), "level out of range");
    if (n) *n = level == 0 ? s->s.n : s->s.levels[level - 1].n;
    if (nnz) *nnz = level == 0 ? 0 : s->s.levels[level - 1].nnz;
  });
}

int b2_coupled_setup_level_copy(const b2_coupled_setup* s, int level, int32_t* rows,
                                int32_t* cols, int32_t* diag, int32_t* aggregate,
                                int32_t* member_offsets, int32_t* members) {
  return guarded([&] {
    KB2_REQUIRE(s && level >= 0 && level < b2_coupled_setup_levels(s), "level out of range");
    const auto copy = [](int32_t* out, const std::vector<int>& v) {
      if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(int));
    };
    if (level > 0) {
      const auto& l = s->s.levels[level - 1];
      copy(rows, l.rows);
      copy(cols, l.cols);
      copy(diag, l.diag);
    }
    if (level < static_cast<int>(s->s.transfers.size())) {
      const auto& t = s->s.transfers[level];
      copy(aggregate, t.aggregate);
      copy(member_offsets, t.offsets);
      copy(members, t.members);
    }
  });
}

int b2_coupled_setup_cell(const b2_coupled_setup* s, float* out) {
  return guarded([&] {
    KB2_REQUIRE(s && out, "coupled: null argument");
    std::memcpy(out, s->s.cell.data(), s->s.cell.size() * sizeof(float));
  });
}

int b2_coupled_setup_width(const b2_coupled_setup* s) { return s ? s->s.width : 0; }

void b2_coupled_setup_free(b2_coupled_setup* s) { delete s; }

}  // extern "C"
