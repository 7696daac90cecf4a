// FP64 iterative refinement: x (FP64) += e, where e solves A e = r with the
// FP32 AMG-PCG to a fixed relative reduction, and r = b - A x is recomputed in
// FP64 each step. The FP32 solve cannot return an iterate better than its
// rounding floor (||A|| ||x|| eps_f / ||b||, 2.8e-6 on a 5.3M-cell tet pressure
// matrix); the refinement carries the solution past it.
#include "mixed.hpp"

#include <cmath>
#include <sstream>

namespace kb2 {

MixedSolver::MixedSolver(const CsrView& a, const MixedOptions& o)
    : o_(o), inner_(Kind::AmgPcg, a, o.amg, nullptr), n_(a.n) {
  rf_.reset(static_cast<std::size_t>(n_));
  e_.reset(static_cast<std::size_t>(n_));
  partials_.reset(kReducePartials);
  norm_.reset(2);
  ticket_.reset(1);
  cuda_check(cudaMemset(ticket_.get(), 0, sizeof(unsigned)), "memset");
}

double MixedSolver::residual(const float* val, const double* x, const float* b, cudaStream_t s) {
  const auto& l = inner_.level(0);
  launch::residual64(n_, l.row_ptr.get(), l.col.get(), val, x, b, rf_.get(),
                     DeviceReducer{partials_.get(), ticket_.get()}, norm_.get(), 0, s);
  inner_.add_bytes(8.0 * l.nnz + 4.0 * (n_ + 1) + 16.0 * n_);  // A, x (FP64), b, rf
  cuda_check(cudaMemcpyAsync(host_.get(), norm_.get(), sizeof(double), cudaMemcpyDeviceToHost, s),
             "residual readback");
  wait(s);
  cuda_check(cudaGetLastError(), "refinement residual");
  return std::sqrt(host_[0]);
}

MixedStats MixedSolver::solve32(const float* val, float* x, const float* b, const Control& c,
                                cudaStream_t s) {
  inner_.check_device();
  KB2_REQUIRE(n_ == 0 || (x != nullptr && b != nullptr && x != b),
              "solve: vector size or alias mismatch");
  if (n_ > 0 && !x64_.allocated()) x64_.reset(static_cast<std::size_t>(n_));
  launch::widen(n_, x, x64_.get(), s);
  const MixedStats st = solve(val, x64_.get(), b, c, s);
  launch::narrow(n_, x64_.get(), x, s);
  return st;
}

MixedStats MixedSolver::solve(const float* val, double* x, const float* b, const Control& c,
                              cudaStream_t s) {
  inner_.check_device();
  KB2_REQUIRE(n_ == 0 || (x != nullptr && b != nullptr), "solve: vector size or alias mismatch");
  KB2_REQUIRE(c.max_iter >= 0 && std::isfinite(c.rel_tol) && c.rel_tol >= 0 &&
                  std::isfinite(c.abs_tol) && c.abs_tol >= 0 && c.residual_check_interval > 0,
              "solve: invalid control");
  MixedStats st;
  if (n_ == 0) {
    st.converged = true;
    return st;
  }
  double r = residual(val, x, b, s);
  if (!std::isfinite(r)) throw NonfiniteError("solve: nonfinite input vector");
  st.initial_residual = st.final_residual = r;
  const double target = std::max(c.abs_tol, c.rel_tol * r);
  if (r > target && (inner_.learned_mode() & Solver::kLearnedWarmStart)) {
    // The learned warm start: one safeguarded step along G(b - A x0); the
    // tolerance stays relative to the residual of the caller's x0.
    inner_.learned_warm_start(val, rf_.get(), x, s);
    r = residual(val, x, b, s);
  }
  int stalled = 0;
  Gnn* const stage = inner_.learned();
  const int mode = inner_.learned_mode();
  while (r > target && st.refinements < o_.max_refinements && st.iterations < c.max_iter) {
    cuda_check(cudaMemsetAsync(e_.get(), 0, sizeof(float) * static_cast<std::size_t>(n_), s),
               "memset");
    Control inner;
    // Ask the inner solve for the reduction still needed, but at least the
    // per-step reduction it is configured for.
    inner.rel_tol = std::max(o_.inner_rel_tol, 0.5 * target / r);
    inner.abs_tol = 0;
    inner.max_iter = std::min(o_.inner_max_iter, c.max_iter - st.iterations);
    inner.residual_check_interval = c.residual_check_interval;
    const Stats is = inner_.solve(val, e_.get(), rf_.get(), inner, s);
    st.iterations += is.iterations;
    launch::update64(n_, x, e_.get(), s);
    inner_.add_bytes(20.0 * n_);
    const double next = residual(val, x, b, s);
    ++st.refinements;
    stalled = next < 0.9 * r ? 0 : stalled + 1;
    r = next;
    if (stalled > 0 && (mode & Solver::kLearnedCycle) && !st.learned_fallback) {
      // The plain AMG cycle is the learned stage's fallback: a refinement
      // that stalls with the stage attached is retried without it.
      const int rest = mode & ~Solver::kLearnedCycle;
      inner_.set_learned(rest != 0 ? stage : nullptr, rest);
      st.learned_fallback = true;
      stalled = 0;
      continue;
    }
    if (!std::isfinite(r) || stalled >= 2) break;
  }
  if (st.learned_fallback) inner_.set_learned(stage, mode);
  inner_.check_learned(s);
  st.final_residual = r;
  st.converged = std::isfinite(r) && r <= target;
  return st;
}

std::string MixedSolver::describe() const {
  std::ostringstream out;
  out << "FP64 iterative refinement over " << inner_.describe();
  return out.str();
}

}  // namespace kb2
