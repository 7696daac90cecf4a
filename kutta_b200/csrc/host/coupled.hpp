// The Coupled (4x4-block) pressure-velocity solve on one B200
// (src/kutta/fv/coupled_solver.hpp:61-101): block BiCGStab preconditioned by
// a block aggregation-AMG V-cycle with damped block-Jacobi smoothing, on the
// block Jacobian of momentum and continuity that fv_coupled.kern.h defines.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../cuda/coupled_kernels.hpp"
#include "coupled_setup.hpp"
#include "device.hpp"
#include "solver.hpp"

namespace kb2 {

class CoupledSolver {
 public:
  // Host setup (sensitivities, aggregation, coarse patterns), then the
  // device arrays. reference >= 0 anchors a closed domain's pressure there.
  CoupledSolver(const CoupledMeshHost& mesh, int reference, const CoupledOptions& options,
                cudaStream_t s);
  CoupledSolver(const CoupledSolver&) = delete;
  CoupledSolver& operator=(const CoupledSolver&) = delete;
  ~CoupledSolver();

  // One momentum component's assembled diagonal (device CSR over the stencil
  // pattern and its physical diagonal), floored and relaxed by the Courant
  // number (coupled_solver.cpp:472-477).
  void capture_diagonal(int component, const int* rows, const int* diag, const float* values,
                        const float* physical, cudaStream_t s);
  // Assembles the Jacobian and right-hand side, then solves for the update
  // (coupled_solver.cpp:479-512).
  Stats solve(const CoupledSolveInputs& in, double density, double velocity_scale,
              const Control& control, cudaStream_t s);
  // u += alpha_u du, p += alpha_p wc dp, then the closed-domain gauge.
  void update(float* u, float* v, float* w, float* p, double alpha_u, double alpha_p,
              cudaStream_t s);
  // The same on the float pairs hi + lo with kpair_add's slacks.
  void paired_update(float* u, float* v, float* w, float* p, float* u_lo, float* v_lo,
                     float* w_lo, float* p_lo, double alpha_u, double alpha_p,
                     float velocity_slack, float pressure_slack, cudaStream_t s);

  std::size_t bytes() const { return bytes_; }
  std::string describe() const;
  int cells() const { return n_; }
  int faces() const { return mesh_.n_faces; }
  // The fine block inverse as two float4 per cell: (iu, iv, iw, schur) and
  // (Hx iu, Hy iv, Hz iw, 0); asynchronous copies to host memory on `s`.
  void copy_inverse(float* inverse, float* inverse_h, cudaStream_t s) const;
  int levels() const { return static_cast<int>(levels_.size()) + 1; }
  int level_rows(int k) const { return k == 0 ? n_ : levels_[k - 1].op.n; }
  // The last solution (float4 per cell, (du, dv, dw, dp~)), the right-hand
  // side and the 27-plane cell data, on the device.
  const float* solution() const { return reinterpret_cast<const float*>(x_); }
  const float* rhs() const { return reinterpret_cast<const float*>(b_.get()); }
  const float* cell_data() const { return cell_.get(); }
  const float* face_coefficients() const { return coefficient_.get(); }
  // A coarse level's operator arrays and transfer (1 <= k < levels()).
  const CoupledLevel& level(int k) const { return levels_[k - 1].op; }
  const CoupledTransfer& transfer(int k) const { return transfers_[k].view; }
  // y = J x, r = b - J x and one smoothing sweep of the fine level on float4
  // vectors (device pointers), after a solve assembled the Jacobian.
  void apply(const float* x, float* y, cudaStream_t s);
  void residual(const float* x, const float* b, float* r, cudaStream_t s);
  void smooth(const float* x, const float* b, float* next, bool first, cudaStream_t s);
  // On coarse level k >= 1: op 1 r = b - J x, 2 / 3 one sweep from x / from
  // zero; op 4 restricts level k - 1's x into y (level k), op 5 adds level
  // k's x into y (level k - 1).
  void level_apply(int k, int op, const float* x, const float* b, float* y, cudaStream_t s);

 private:
  struct Level {
    CoupledLevel op;
    DArray<int> rows, cols, diag;
    DArray<float> a, c, g, h, d;
    DArray<float4> b, store[2];
    float4 *x = nullptr, *tmp = nullptr;  // the smoother's ping-pong roles over store
  };
  // One BiCGStab iteration as a CUDA graph, for the buffer roles it starts
  // from; `after` are the roles it leaves.
  struct IterationGraph {
    std::vector<float4*> before, after;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
  };
  struct Transfer {
    CoupledTransfer view;
    DArray<int> aggregate, offsets, members;
  };
  template <class T>
  void own(DArray<T>& a, std::size_t n) {
    a.reset(n);
    bytes_ += n * sizeof(T);
  }
  template <class T>
  void own(DArray<T>& a, const std::vector<T>& v, cudaStream_t s) {
    own(a, v.size());
    a.upload(v.data(), v.size(), s);
  }
  CoupledFine fine() const;
  void fine_smooth(float4*& out, const float4* rhs, int sweeps, bool first);
  void coarse_smooth(Level& l, int sweeps, bool first);
  void cycle(std::size_t k);
  void precondition(const float4* rhs, float4*& out);
  void galerkin(const CoupledSolveInputs& in);
  double norm(const float4* v);
  std::vector<float4*> roles() const;
  void set_roles(const std::vector<float4*>& r);
  // Runs `body` (kernel launches only) directly, or as a cached graph.
  template <class Body>
  void iteration(Body body);
  Stats bicgstab(const Control& c);
  Stats bounded(Stats stats, double target);

  cudaStream_t stream_ = nullptr;
  CoupledOptions options_;
  int n_ = 0, reference_ = -1, width_ = 0;
  float wc_ = 1;
  std::size_t bytes_ = 0;
  CoupledMeshDevice mesh_;
  DArray<int> owner_, neighbour_, offsets_, faces_, adjacent_, kind_;
  DArray<float> sign_, sx_, sy_, sz_, dx_, dy_, dz_, diffusion_, volume_;
  DArray<float> cell_, coefficient_, scratch_;
  DArray<float4> diag_, coupling_, inverse_, inverse_h_, edge_, face_;
  DArray<float2> coupling_yz_;
  DArray<float> edge_h_;
  DArray<int2> link_;
  std::vector<Level> levels_;
  std::vector<Transfer> transfers_;
  DArray<float4> b_, r_, shadow_, p_, q_, sv_, t_;
  // The smoother double-buffers through tmp_, so the solution, the two
  // preconditioned directions and the scratch trade storage: four arrays,
  // four roles.
  DArray<float4> store_[4];
  float4 *x_ = nullptr, *z_ = nullptr, *zs_ = nullptr, *tmp_ = nullptr;
  DArray<float> scalars_, gauge_;
  DArray<int> status_;
  DArray<double> partials_, values_;
  DArray<unsigned> ticket_;
  CoupledSolveInputs inputs_;
  // Pinned host words for the per-iteration status and the norms (a pinned
  // allocation per solve costs milliseconds and its release synchronises).
  Pinned<int> host_status_{3};
  Pinned<double> host_value_{1};
  bool graphs_enabled_ = true;
  // The first coarse level (index into levels_) from which the V-cycle runs
  // as one launch (levels_.size(): none).
  std::size_t tail_ = 0;
  cudaStream_t capture_ = nullptr;
  std::vector<IterationGraph> graphs_;
};

}  // namespace kb2
