// Mixed-precision pressure solve (no reference counterpart): FP64 iterative
// refinement around the FP32 AMG-PCG of solver.hpp in its mixed mode.
#pragma once

#include <string>

#include "solver.hpp"

namespace kb2 {

struct MixedOptions {
  Options amg;                // pairing, sweeps, structure; coarse_bf16 / dense_coarsest / absorb
  double inner_rel_tol = 1e-3;
  int inner_max_iter = 300;
  int max_refinements = 30;
};

struct MixedStats {
  int refinements = 0, iterations = 0;
  bool converged = false;
  // The learned cycle stage was detached after a stalled refinement and the
  // solve finished with the AMG cycle alone (the stage is re-attached after).
  bool learned_fallback = false;
  double initial_residual = 0, final_residual = 0;
};

class MixedSolver {
 public:
  MixedSolver(const CsrView& a, const MixedOptions& o);
  void refresh(const float* val, cudaStream_t s) { inner_.refresh(val, s); }
  void assemble_refresh(const FvPressure& fv, float* values, float* rhs, cudaStream_t s) {
    inner_.assemble_refresh(fv, values, rhs, s);
  }
  // x: FP64 solution (initial guess in); b: FP32 right-hand side.
  MixedStats solve(const float* val, double* x, const float* b, const Control& c, cudaStream_t s);
  // The same solve for a caller that holds x in FP32 (the reference's
  // LinearSolver::solve): x is widened into an FP64 copy the solver keeps,
  // solved, and rounded back to nearest. A rounded x carries the FP32 floor
  // again, so targets below it need the FP64 form.
  MixedStats solve32(const float* val, float* x, const float* b, const Control& c,
                     cudaStream_t s);
  std::string describe() const;
  Solver& inner() { return inner_; }

 private:
  double residual(const float* val, const double* x, const float* b, cudaStream_t s);

  MixedOptions o_;
  Solver inner_;
  int n_;
  DArray<float> rf_, e_;
  DArray<double> partials_, norm_, x64_;
  DArray<unsigned> ticket_;
  Pinned<double> host_{2};
};

}  // namespace kb2
