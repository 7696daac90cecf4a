// The reference-side adapter: kutta::LinearSolver (src/kutta/linalg/solver.hpp:74-81)
// implemented over the kutta_b200 C ABI, for the reference's CUDA backend.
// It is compiled with the reference's sources, not with this library:
//
//   src/kutta/linalg/b200_solver.cpp   this file
//   include path                       kutta_b200's include/ and the CUDA toolkit's
//   link                               libkutta_b200.so, -lcudart
//
// Two things come from the reference's CUDA backend:
//   - the device pointer behind a buffer: cuda_ptr(BufferHandle*)
//     (runtime/cuda/cuda_kernel_table.hpp:16);
//   - the device's stream. CudaDevice keeps it private (stream_,
//     runtime/cuda/cuda_device.cu:122); cuda_stream(Device&) below is the
//     one-line accessor a maintainer adds next to cuda_ptr, so that the
//     library's kernels queue in order with the backend's own.
//
// The factories dispatch here when dev.backend() == Backend::Cuda:
//
//   make_solver(kind, dev, a, options)        solver.cpp  -> make_b200_solver
//   make_amg_solver(kind, dev, a, options)    amg.cpp:345 -> make_b200_amg_solver
//
// and a steady solver that opts into the mixed-precision pressure solve builds
// it with make_b200_mixed_solver(a, options) in place of make_solver(AmgPcg, ...).
//
// The option checks (kinds, sweeps, M-matrix structure) run inside
// b2_solver_create with the reference's messages; its status codes map back to
// kutta::Error and kutta::NonfiniteError (core/types.hpp:24-33).
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "kutta/linalg/amg.hpp"
#include "kutta/runtime/cuda/cuda_kernel_table.hpp"
#include "kutta_b200.h"

namespace kutta {
cudaStream_t cuda_stream(Device& dev);  // added to runtime/cuda/cuda_device.cu

namespace {

void check(int status) {
  if (status == B2_OK) return;
  char message[1024];
  b2_last_error(message, sizeof message);
  if (status == B2_NONFINITE) throw NonfiniteError(message);
  throw Error(message);
}

float* ptr(const Buffer<float>& b) { return static_cast<float*>(cuda_ptr(b.handle())); }

// The enums cross the C ABI as their values.
static_assert(static_cast<int>(SolverKind::Jacobi) == B2_JACOBI &&
              static_cast<int>(SolverKind::PcgJacobi) == B2_PCG_JACOBI &&
              static_cast<int>(SolverKind::BicgstabJacobi) == B2_BICGSTAB_JACOBI &&
              static_cast<int>(SolverKind::AmgPcg) == B2_AMG_PCG &&
              static_cast<int>(SolverKind::AmgBicgstab) == B2_AMG_BICGSTAB);
static_assert(static_cast<int>(AmgCycle::V) == B2_CYCLE_V &&
              static_cast<int>(AmgCycle::K) == B2_CYCLE_K);
static_assert(static_cast<int>(NullSpace::None) == B2_NULLSPACE_NONE &&
              static_cast<int>(NullSpace::Constant) == B2_NULLSPACE_CONSTANT);
static_assert(static_cast<int>(OperatorStructure::General) == B2_STRUCTURE_GENERAL &&
              static_cast<int>(OperatorStructure::SymmetricMMatrix) ==
                  B2_STRUCTURE_SYMMETRIC_M_MATRIX);

// The C ABI takes bare pointers, so the vector sizes it cannot see are checked
// here, with the reference's messages (csr.cpp:12-16, 55). The value count
// comes before the row checks: the library reads nnz values.
void check_sizes(const CsrMatrixHost& a) {
  const CsrPattern& p = a.pattern;
  if (p.n_rows < 0) throw Error("CSR: negative row count");
  if (p.col.size() > static_cast<std::size_t>(std::numeric_limits<Index>::max()))
    throw Error("CSR: exceeds 32-bit entry limit");
  if (p.row_ptr.size() != static_cast<std::size_t>(p.n_rows) + 1 ||
      p.diag.size() != static_cast<std::size_t>(p.n_rows))
    throw Error("CSR: invalid array sizes");
  if (a.val.size() != p.col.size()) throw Error("CSR: value count mismatch");
}

// A KrylovWorkspace shared by several solvers maps to one b2_workspace. The
// library's solvers hold their own share of it, so the handle kept here only
// decides which solvers share; it is replaced once its KrylovWorkspace is gone.
b2_workspace* shared_workspace(const std::shared_ptr<KrylovWorkspace>& w) {
  if (!w) return nullptr;
  struct Entry {
    std::weak_ptr<KrylovWorkspace> owner;
    std::unique_ptr<b2_workspace, void (*)(b2_workspace*)> handle{nullptr, b2_workspace_destroy};
  };
  static std::mutex lock;
  static std::map<const KrylovWorkspace*, Entry> table;
  std::lock_guard<std::mutex> guard(lock);
  for (auto it = table.begin(); it != table.end();)
    it = it->second.owner.expired() ? table.erase(it) : std::next(it);
  Entry& e = table[w.get()];
  if (!e.handle) {
    b2_workspace* h = nullptr;
    check(b2_workspace_create(w->rows(), &h));
    e.owner = w;
    e.handle.reset(h);
  }
  return e.handle.get();
}

class B200Solver final : public LinearSolver {
 public:
  B200Solver(SolverKind kind, const CsrMatrixHost& a, const b2_options& options,
             bool amg_options) {
    check_sizes(a);
    check(b2_solver_create(static_cast<int>(kind), a.pattern.n_rows, a.pattern.nnz(),
                           a.pattern.row_ptr.data(), a.pattern.col.data(), a.pattern.diag.data(),
                           a.val.data(), &options, amg_options ? 1 : 0, &s_));
  }
  ~B200Solver() override { b2_solver_destroy(s_); }
  B200Solver(const B200Solver&) = delete;
  B200Solver& operator=(const B200Solver&) = delete;

  void refresh(Device& dev, const CsrMatrix& a) override {
    check(b2_solver_refresh(s_, ptr(a.val), cuda_stream(dev)));
  }

  SolveStats solve(Device& dev, const CsrMatrix& a, Buffer<float>& x, const Buffer<float>& b,
                   const SolveControl& c) override {
    const b2_control control{c.rel_tol, c.abs_tol, c.max_iter, c.residual_check_interval};
    b2_stats st{};
    check(b2_solver_solve(s_, ptr(a.val), ptr(x), ptr(b), &control, &st, cuda_stream(dev)));
    return {st.iterations, st.initial_residual, st.final_residual, st.converged != 0};
  }

  std::string describe() const override {
    char text[512];
    b2_solver_describe(s_, text, sizeof text);
    return text;
  }

 private:
  b2_solver* s_ = nullptr;
};

// The mixed-precision pressure solve (no reference counterpart) behind the
// same interface. x stays FP32 as LinearSolver::solve has it: the library
// widens it into an FP64 copy, refines, and rounds the solution back. The
// reported final residual is the FP64 solution's; targets below the FP32
// floor (about 1e-7 relative) need b2_mixed_solve and an FP64 x instead.
class B200MixedSolver final : public LinearSolver {
 public:
  B200MixedSolver(const CsrMatrixHost& a, const b2_mixed_options& options) {
    check_sizes(a);
    check(b2_mixed_create(a.pattern.n_rows, a.pattern.nnz(), a.pattern.row_ptr.data(),
                          a.pattern.col.data(), a.pattern.diag.data(), a.val.data(), &options,
                          &s_));
  }
  ~B200MixedSolver() override { b2_mixed_destroy(s_); }
  B200MixedSolver(const B200MixedSolver&) = delete;
  B200MixedSolver& operator=(const B200MixedSolver&) = delete;

  void refresh(Device& dev, const CsrMatrix& a) override {
    check(b2_mixed_refresh(s_, ptr(a.val), cuda_stream(dev)));
  }

  SolveStats solve(Device& dev, const CsrMatrix& a, Buffer<float>& x, const Buffer<float>& b,
                   const SolveControl& c) override {
    const b2_control control{c.rel_tol, c.abs_tol, c.max_iter, c.residual_check_interval};
    b2_mixed_stats st{};
    check(b2_mixed_solve_f32(s_, ptr(a.val), ptr(x), ptr(b), &control, &st, cuda_stream(dev)));
    return {st.iterations, st.initial_residual, st.final_residual, st.converged != 0};
  }

  std::string describe() const override {
    char text[512];
    b2_mixed_describe(s_, text, sizeof text);
    return text;
  }

 private:
  b2_mixed* s_ = nullptr;
};

}  // namespace

// The pressure solver of steady_solver.cpp:578-580 in its mixed-precision
// form: the library's tuned defaults, with the caller's structure and null
// space. Only the SPD pressure equation takes it (flexible CG inside). It
// keeps its own Krylov vectors, so a shared KrylovWorkspace is not used.
std::unique_ptr<LinearSolver> make_b200_mixed_solver(const CsrMatrixHost& a,
                                                     const SolverOptions& o) {
  b2_mixed_options options;
  b2_mixed_options_default(&options);
  options.amg.nullspace = static_cast<int>(o.nullspace);
  options.amg.structure = static_cast<int>(o.structure);
  return std::make_unique<B200MixedSolver>(a, options);
}

std::unique_ptr<LinearSolver> make_b200_solver(SolverKind kind, const CsrMatrixHost& a,
                                               const SolverOptions& o) {
  b2_options options;
  b2_options_default(&options);  // the library's defaults, the device setup among them
  options.nullspace = static_cast<int>(o.nullspace);
  options.structure = static_cast<int>(o.structure);
  options.workspace = shared_workspace(o.workspace);
  return std::make_unique<B200Solver>(kind, a, options, false);
}

std::unique_ptr<LinearSolver> make_b200_amg_solver(SolverKind kind, const CsrMatrixHost& a,
                                                   const AmgOptions& o) {
  b2_options options;
  b2_options_default(&options);
  options.cycle = static_cast<int>(o.cycle);  // an invalid value is rejected by the library
  options.pre_sweeps = o.pre_sweeps;
  options.post_sweeps = o.post_sweeps;
  options.coarse_sweeps = o.coarse_sweeps;
  options.coarse_rows = static_cast<int>(o.coarse_rows);
  options.max_levels = o.max_levels;
  options.aggregation_passes = o.aggregation_passes;
  options.strength_threshold = o.strength_threshold;
  options.nullspace = static_cast<int>(o.nullspace);
  options.structure = static_cast<int>(o.structure);
  options.workspace = shared_workspace(o.workspace);
  return std::make_unique<B200Solver>(kind, a, options, true);
}

}  // namespace kutta
