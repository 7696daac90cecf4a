// Test infrastructure only: a C-ABI shim over the reference library's own CPU
// path (kutta::make_solver / make_amg_solver on the serial CPU Device), built by
// oracle/build_ref.sh from the reference sources into oracle/_ref/. Only the
// tests, the golden-fixture generator and bench.py's reference/CPU-baseline arm
// load it; the product never does.
//
// It exposes three things:
//   kref_solve      set up, refresh and solve one system exactly as the reference
//                   does (src/kutta/linalg/amg.cpp:345-406, solver.cpp:97-176);
//   kref_hierarchy  capture the AMG hierarchy the reference actually solves with
//                   (aggregates, coarse CSR patterns and values, L1 inverse
//                   diagonals) from the kernels its V-cycle launches, the way
//                   tests/linalg/test_solvers.cpp:509-521 reads them back;
//   kref_fv_*       the finite-volume kernels on either side of the pressure
//                   solve (src/kutta/kernels/fv_flow.kern.h:164-201).
#include <chrono>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "kernels.hpp"
#include "kutta/linalg/amg.hpp"
#include "ref_watch.hpp"

using namespace kutta;
using kref::WatchDevice;

// Host array -> CPU-device buffer.
template <class T>
static Buffer<T> put(Device& dev, const T* p, std::size_t n) {
  return dev.upload<T>(std::span<const T>(p, n));
}

extern "C" {

struct kref_options {
  int kind;           // 0 Jacobi, 1 PcgJacobi, 2 BicgstabJacobi, 3 AmgPcg, 4 AmgBicgstab
  int cycle;          // 0 V, 1 K
  int pre_sweeps, post_sweeps, coarse_sweeps, coarse_rows, max_levels, passes;
  double threshold;
  int nullspace;      // 0 None, 1 Constant
  int structure;      // 0 General, 1 SymmetricMMatrix
  int use_make_solver;  // 1: make_solver(kind, dev, a, {nullspace, structure}) defaults
};
struct kref_control { double rel_tol, abs_tol; int max_iter, interval; };
struct kref_stats {
  int iterations, converged, levels, pad;
  double initial_residual, final_residual, setup_s, refresh_s, solve_s;
};

static thread_local std::string g_error;
const char* kref_last_error() { return g_error.c_str(); }

static CsrMatrixHost host_matrix(int n, int nnz, const int* row_ptr, const int* col,
                                 const int* diag, const double* val) {
  CsrMatrixHost a;
  a.pattern.n_rows = n;
  a.pattern.row_ptr.assign(row_ptr, row_ptr + n + 1);
  a.pattern.col.assign(col, col + nnz);
  a.pattern.diag.assign(diag, diag + n);
  a.val.assign(val, val + nnz);
  return a;
}

static std::unique_ptr<LinearSolver> build(Device& dev, const CsrMatrixHost& a,
                                           const kref_options& o) {
  const auto kind = static_cast<SolverKind>(o.kind);
  if (o.use_make_solver || (kind != SolverKind::AmgPcg && kind != SolverKind::AmgBicgstab)) {
    SolverOptions so;
    so.nullspace = static_cast<NullSpace>(o.nullspace);
    so.structure = static_cast<OperatorStructure>(o.structure);
    return make_solver(kind, dev, a, so);
  }
  AmgOptions ao;
  ao.cycle = o.cycle ? AmgCycle::K : AmgCycle::V;
  ao.pre_sweeps = o.pre_sweeps;
  ao.post_sweeps = o.post_sweeps;
  ao.coarse_sweeps = o.coarse_sweeps;
  ao.coarse_rows = o.coarse_rows;
  ao.max_levels = o.max_levels;
  ao.aggregation_passes = o.passes;
  ao.strength_threshold = o.threshold;
  ao.nullspace = static_cast<NullSpace>(o.nullspace);
  ao.structure = static_cast<OperatorStructure>(o.structure);
  return make_amg_solver(kind, dev, a, ao);
}

// Full reference lifecycle: setup from host values, refresh, solve. x holds the
// initial guess on entry and the solution on return. Returns 0, or -1 with the
// reference's exception text in kref_last_error().
int kref_solve(int n, int nnz, const int* row_ptr, const int* col, const int* diag,
               const double* val, const float* b, float* x, const kref_options* o,
               const kref_control* c, kref_stats* s, char* describe, int describe_len) {
  try {
    using Clock = std::chrono::steady_clock;
    auto dev = Device::create(Backend::Cpu);
    const auto a = host_matrix(n, nnz, row_ptr, col, diag, val);
    auto matrix = upload(*dev, a);
    auto t0 = Clock::now();
    auto solver = build(*dev, a, *o);
    auto t1 = Clock::now();
    solver->refresh(*dev, matrix);
    auto t2 = Clock::now();
    auto db = dev->upload<float>(std::span<const float>(b, n));
    auto dx = dev->upload<float>(std::span<const float>(x, n));
    auto t3 = Clock::now();
    const auto st = solver->solve(*dev, matrix, dx, db,
                                  {c->rel_tol, c->abs_tol, c->max_iter, c->interval});
    auto t4 = Clock::now();
    dev->download(dx, std::span<float>(x, n));
    s->iterations = st.iterations;
    s->converged = st.converged ? 1 : 0;
    s->initial_residual = st.initial_residual;
    s->final_residual = st.final_residual;
    s->setup_s = std::chrono::duration<double>(t1 - t0).count();
    s->refresh_s = std::chrono::duration<double>(t2 - t1).count();
    s->solve_s = std::chrono::duration<double>(t4 - t3).count();
    if (describe && describe_len > 0) {
      const auto d = solver->describe();
      std::snprintf(describe, describe_len, "%s", d.c_str());
    }
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

// Captured hierarchy: level 0 is the input matrix, levels 1.. are the coarse
// operators the V-cycle really used; aggregate[l] maps level-l rows to level
// l+1 rows (-1 for rows left out).
struct KrefHierarchy {
  struct Level {
    int n = 0;
    std::vector<int> row_ptr, col, aggregate;
    std::vector<float> val, l1;
  };
  std::vector<Level> levels;
};

void* kref_hierarchy(int n, int nnz, const int* row_ptr, const int* col, const int* diag,
                     const double* val, const kref_options* o) {
  try {
    WatchDevice dev;
    const auto a = host_matrix(n, nnz, row_ptr, col, diag, val);
    auto matrix = upload(dev, a);
    auto solver = build(dev, a, *o);
    solver->refresh(dev, matrix);
    std::map<std::size_t, KrefHierarchy::Level> ops;
    std::map<std::size_t, std::vector<int>> aggregates;
    std::map<std::size_t, std::vector<float>> inverse_l1;
    dev.observer = [&](KernelId id, std::size_t count, std::span<const KernelArg> args) {
      // Argument positions follow the kernel signatures in
      // src/kutta/kernels/linalg.kern.h and amg.kern.h.
      if (id == KernelId::amg_coarse_solve) count = static_cast<std::size_t>(args[7].get<int>());
      const bool smooth = id == KernelId::amg_smooth || id == KernelId::amg_smooth_zero;
      if ((id == KernelId::csr_residual_guarded || smooth || id == KernelId::amg_coarse_solve) &&
          !ops.contains(count)) {
        auto& l = ops[count];
        l.n = static_cast<int>(count);
        l.row_ptr = dev.read<int>(args[0].buffer);
        l.col = dev.read<int>(args[1].buffer);
        l.val = dev.read<float>(args[2].buffer);
      }
      if ((smooth || id == KernelId::amg_coarse_solve) && !inverse_l1.contains(count))
        inverse_l1[count] = dev.read<float>(args[5].buffer);
      if (id == KernelId::amg_prolong_guarded && !aggregates.contains(count))
        aggregates[count] = dev.read<int>(args[0].buffer);
    };
    auto db = dev.upload<float>(std::vector<float>(n, 1.0f));
    auto dx = dev.alloc<float>(n);
    dev.fill(dx, 0.0f);
    solver->solve(dev, matrix, dx, db, {0, 0, 1, 8});
    auto* h = new KrefHierarchy;
    for (auto it = ops.rbegin(); it != ops.rend(); ++it) {
      auto l = std::move(it->second);
      l.row_ptr.resize(l.n + 1);
      l.col.resize(l.row_ptr.back());
      l.val.resize(l.row_ptr.back());
      l.l1 = inverse_l1[it->first];
      l.l1.resize(l.n);
      if (aggregates.contains(it->first)) {
        l.aggregate = aggregates[it->first];
        l.aggregate.resize(l.n);
      }
      h->levels.push_back(std::move(l));
    }
    return h;
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

int kref_hierarchy_levels(void* h) { return static_cast<int>(static_cast<KrefHierarchy*>(h)->levels.size()); }
void kref_hierarchy_shape(void* h, int level, int* n, int* nnz, int* has_aggregate) {
  const auto& l = static_cast<KrefHierarchy*>(h)->levels[level];
  *n = l.n;
  *nnz = l.row_ptr.empty() ? 0 : l.row_ptr.back();
  *has_aggregate = l.aggregate.empty() ? 0 : 1;
}
void kref_hierarchy_copy(void* h, int level, int* row_ptr, int* col, float* val, float* l1,
                         int* aggregate) {
  const auto& l = static_cast<KrefHierarchy*>(h)->levels[level];
  std::memcpy(row_ptr, l.row_ptr.data(), l.row_ptr.size() * sizeof(int));
  std::memcpy(col, l.col.data(), l.col.size() * sizeof(int));
  std::memcpy(val, l.val.data(), l.val.size() * sizeof(float));
  std::memcpy(l1, l.l1.data(), l.l1.size() * sizeof(float));
  if (aggregate && !l.aggregate.empty())
    std::memcpy(aggregate, l.aggregate.data(), l.aggregate.size() * sizeof(int));
}
void kref_hierarchy_free(void* h) { delete static_cast<KrefHierarchy*>(h); }

// The reference's own finite-volume kernels (fv_flow.kern.h:164-201) on the
// serial CPU device, host arrays in and out. nc = cells, nf = faces, ns =
// cell-face slots, nnz = matrix entries.
int kref_fv_pressure_assemble(int nc, int nf, int ns, int nnz, const int* offsets, const int* faces,
                              const float* sign, const int* adjacent, const int* entry,
                              const int* rows, const int* diag, const float* coefficient,
                              const float* flux, float* values, float* rhs, int reference) {
  try {
    auto dev = Device::create(Backend::Cpu);
    auto d_values = put(*dev, values, nnz);
    auto d_rhs = put(*dev, rhs, nc);
    kern::fv_pressure_assemble(*dev, nc, put(*dev, offsets, nc + 1), put(*dev, faces, ns),
                               put(*dev, sign, ns), put(*dev, adjacent, ns), put(*dev, entry, ns),
                               put(*dev, rows, nc + 1), put(*dev, diag, nc),
                               put(*dev, coefficient, nf), put(*dev, flux, nf), d_values, d_rhs,
                               reference);
    dev->download(d_values, std::span<float>(values, nnz));
    dev->download(d_rhs, std::span<float>(rhs, nc));
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

int kref_fv_correct_flux(int nf, int nc, const int* owner, const int* neighbour,
                         const float* correction, const float* coefficient, float* flux,
                         int internal) {
  try {
    auto dev = Device::create(Backend::Cpu);
    auto d_flux = put(*dev, flux, nf);
    kern::fv_correct_flux(*dev, nf, put(*dev, owner, nf), put(*dev, neighbour, internal),
                          put(*dev, correction, nc), put(*dev, coefficient, nf), d_flux, internal);
    dev->download(d_flux, std::span<float>(flux, nf));
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

int kref_fv_correct_velocity(int nc, const float* volume, const float* inverse,
                             const float* diagonal, const float* gx, const float* gy,
                             const float* gz, const float* correction, float* u, float* v,
                             float* w, float* p, float alpha) {
  try {
    auto dev = Device::create(Backend::Cpu);
    auto du = put(*dev, u, nc), dv = put(*dev, v, nc), dw = put(*dev, w, nc), dp = put(*dev, p, nc);
    kern::fv_correct_velocity(*dev, nc, put(*dev, volume, nc), put(*dev, inverse, nc),
                              put(*dev, diagonal, nc), put(*dev, gx, nc), put(*dev, gy, nc),
                              put(*dev, gz, nc), put(*dev, correction, nc), du, dv, dw, dp, alpha);
    dev->download(du, std::span<float>(u, nc));
    dev->download(dv, std::span<float>(v, nc));
    dev->download(dw, std::span<float>(w, nc));
    dev->download(dp, std::span<float>(p, nc));
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

}  // extern "C"
