// The LinearSolver of the reference's linalg boundary (src/kutta/linalg/solver.hpp),
// re-implemented over sm_100a kernels: Krylov drivers (Jacobi, PCG, BiCGStab) with
// device-resident float-pair scalars, and the aggregation-AMG preconditioner.
#pragma once

#include <cmath>
#include <functional>
#include <initializer_list>
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "../cuda/kernels.hpp"
#include "device.hpp"
#include "learned.hpp"
#include "setup.hpp"

namespace kb2 {

// Face data of the pressure assembly (fv_pressure_assemble's inputs,
// src/kutta/kernels/fv_flow.kern.h:164-167), device pointers.
struct FvPressure {
  const int* offsets = nullptr;   // cell-face slot offsets [n + 1]
  const int* faces = nullptr;     // face of each slot
  const float* sign = nullptr;    // +1 on the owner side, -1 on the neighbour side
  const int* adjacent = nullptr;  // cell across the face, -1 on the boundary
  const int* entry = nullptr;     // CSR position of (cell, adjacent)
  const float* coefficient = nullptr;  // per face
  const float* flux = nullptr;         // per face
  int reference = -1;                  // eliminated reference cell, or -1
};

struct Control {  // SolveControl, solver.hpp:18-23
  double rel_tol = 1e-2, abs_tol = 1e-12;
  int max_iter = 200, residual_check_interval = 8;
};
struct Stats {  // SolveStats, solver.hpp:25-30
  int iterations = 0;
  double initial_residual = 0, final_residual = 0;
  bool converged = false;
};

// KrylovWorkspace, solver.hpp:47-64: vectors allocated on first use and shared by
// solvers of one size whose calls never run concurrently.
class Workspace {
 public:
  enum Slot { R, Z, P, Q, Shadow, S, T, Zs, Best, Scratch, Count };
  explicit Workspace(int rows) : rows_(rows) {}
  int rows() const { return rows_; }
  float* vector(Slot slot) {
    int device = 0;
    cuda_check(cudaGetDevice(&device), "cudaGetDevice");
    KB2_REQUIRE(device_ < 0 || device_ == device, "Krylov workspace shared across devices");
    device_ = device;
    auto& v = v_[slot];
    if (!v.allocated()) v.reset(static_cast<std::size_t>(rows_));
    return v.get();
  }

 private:
  int rows_;
  int device_ = -1;
  DArray<float> v_[Count];
};

struct DevLevel {
  int n = 0, nnz = 0;
  DArray<int> row_ptr, col, diag;
  DArray<float> val;            // coarse levels (level 0 uses the caller's values)
  DArray<float> l1;             // inverse L1 diagonal
  DArray<float> xa, ra, b;      // storage; x/r below name the current roles
  float* x = nullptr;
  float* r = nullptr;
  DArray<float> projection;     // constant-nullspace sum pair
  // K-cycle inner corrections (coarse levels): z ping-pongs with r, x is the
  // correction handed to the prolongation.
  DArray<float> za, p, q, t, scalars;
  DArray<int> status;
  float* z = nullptr;
  // Mixed precision: BF16 operator with row scales; dense FP64 inverse.
  DArray<unsigned short> v16;
  DArray<float> scale;
  DArray<double> dense_lower, dense_inverse;
  // transfer to level + 1
  DArray<int> aggregate, member_offsets, members, entry_offsets, entries;
};

// Solve-time measurement: device time of every fine-level smoother sweep (CUDA
// events on the solve stream) and the algorithmic bytes of every launch.
struct Profile {
  long long launches = 0, fine_sweeps = 0, solves = 0;
  double fine_sweep_ms = 0, fine_sweep_bytes = 0, algorithmic_bytes = 0;
};

class Solver {
 public:
  Solver(Kind kind, const CsrView& a, const Options& options, std::shared_ptr<Workspace> workspace);
  ~Solver();
  void set_profile(bool on);
  Profile profile() const {
    Profile p = prof_;
    p.launches = launch::counter.load() - launch_mark_;
    return p;
  }
  // Bytes of kernels a wrapping driver launched (the FP64 refinement).
  void add_bytes(double bytes) { tally(bytes); }
  void refresh(const float* val, cudaStream_t s);
  // Assembles the pressure matrix into `values` and rhs, then refreshes.
  void assemble_refresh(const FvPressure& fv, float* values, float* rhs, cudaStream_t s);
  Stats solve(const float* val, float* x, const float* b, const Control& c, cudaStream_t s);
  std::string describe() const;

  int levels() const { return static_cast<int>(levels_.size()); }
  const DevLevel& level(int i) const { return levels_[static_cast<std::size_t>(i)]; }
  int rows() const { return n_; }
  int entries() const { return nnz_; }
  // Throws unless the current device is the one the solver was built on: its
  // arrays live there (the reference's Device check, solver.cpp:194-195).
  void check_device() const;
  const float* current_values() const { return val_; }

 private:
  bool amg() const { return kind_ == Kind::AmgPcg || kind_ == Kind::AmgBicgstab; }
  bool bicg() const { return kind_ == Kind::BicgstabJacobi || kind_ == Kind::AmgBicgstab; }
  // A variable preconditioner needs the flexible beta (solver.cpp:296-298): the
  // K-cycle, and the mixed V-cycle (BF16 rounding breaks exact symmetry).
  bool variable() const { return amg() && (options_.cycle == Cycle::K || options_.coarse_bf16); }
  bool dense(const DevLevel& l) const { return l.dense_inverse.allocated(); }
  // Whether coarse level `index` takes the K-cycle's inner Krylov step (given
  // a K-cycle and a level above the coarsest two).
  bool inner_level(std::size_t index) const {
    return options_.k_levels <= 0 || index <= static_cast<std::size_t>(options_.k_levels);
  }
  // The hierarchy built on the device (device_setup.cpp) when the options ask
  // for it and the pattern is structurally symmetric; the host setup else.
  bool device_pattern_symmetric(cudaStream_t s);
  void build_device_levels(const CsrView& a, cudaStream_t s);
  bool device_setup_ = false;
  // Refresh from the level-0 values; fine_done: level 0's L1 diagonal and
  // check slot are already written (by the fused assembly).
  void refresh_levels(const float* val, bool fine_done, cudaStream_t s);
  void prepare_mixed(cudaStream_t s, int error_slot);
  void choose_coarsest(double smallest_pivot);
  bool dense_ok_ = false;  // the dense coarsest inverse is used (well conditioned)
  // Cluster-fused tail of the mixed V-cycle: levels >= tail_start_ in one launch.
  void plan_tail();
  bool tail_on_ = false;
  std::size_t tail_start_ = 0;
  double tail_bytes_ = 0;
  launch::TailPlan tail_{};
  bool mixed() const { return options_.coarse_bf16 || options_.dense_coarsest; }
  // The mixed solve's packed copy of the fine operator (width 0: CSR kernels).
  struct Packed {
    int width = 0;
    DArray<float> vals, diag;
    DArray<short> offsets;
  } packed_;
  void plan_packed(const CsrView& a, cudaStream_t s);
  launch::PackedRows packed() const {
    return launch::PackedRows{packed_.width, packed_.vals.get(), packed_.offsets.get(),
                              packed_.diag.get()};
  }
  // Algorithmic bytes of one pass over the fine operator: CSR, or the packed
  // rows' stored entries (padding slots are not counted).
  double fine_operator_bytes() const {
    return packed_.width > 0 ? 6.0 * (nnz_ - n_) + 4.0 * n_ : 8.0 * nnz_ + 4.0 * (n_ + 1);
  }
  const int* rows0() const { return levels_[0].row_ptr.get(); }
  const int* cols0() const { return levels_[0].col.get(); }

  // Device primitives on stream_.
  void residual(const float* x, const float* b, float* r);
  struct Request {
    ReduceMode mode;
    const float* x;
    const float* y;
    int n;
  };
  // Device::reduce_many: several FP64 reductions behind one host wait.
  std::vector<double> host_reduce(std::initializer_list<Request> requests);
  double norm(const float* x);
  void copy(float* dst, const float* src, int n);
  void project(float* x, int n, float* projection);
  void reset(int iterations);

  // Preconditioner.
  void apply(const float* r, float*& z);
  // Whether the flexible PCG's reductions after the preconditioner can ride
  // on the fine post-sweep (nothing touches z after that sweep), and the
  // request flag set around apply() when they do.
  bool can_fuse_dots() const {
    return amg() && variable() && !nullspace_ && levels_.size() > 1 && options_.post_sweeps >= 1 &&
           !levels_[0].v16.allocated() &&
           !(learned_ != nullptr && (learned_mode_ & kLearnedCycle));
  }
  bool fuse_dots_ = false;
  void precondition(const float* r, float*& z);
  // c = G(t), q = A c and the dots {c.t, c.Ac} for the safeguarded step.
  void learned_direction(const float* t);
  Gnn* learned_ = nullptr;  // optional learned stage (not owned)
  int learned_mode_ = 0;    // kLearnedCycle | kLearnedWarmStart
  DArray<float> learned_residual_, learned_correction_, learned_product_;
  DArray<double> learned_dots_;

 public:
  static constexpr int kLearnedCycle = 1, kLearnedWarmStart = 2;
  // Attaches (or, with null, detaches) a learned stage: after each AMG cycle
  // (kLearnedCycle) and/or as a warm-start step (kLearnedWarmStart). The
  // network must outlive its attachment.
  void set_learned(Gnn* g, int mode);
  int learned_mode() const { return learned_ != nullptr ? learned_mode_ : 0; }
  Gnn* learned() const { return learned_; }
  // x += alpha G(r) in FP64 for the residual r = b - A x, alpha =
  // max(0, c.t / c.Ac): the learned warm start (a no-op unless attached in
  // kLearnedWarmStart mode).
  void learned_warm_start(const float* val, const float* r, double* x, cudaStream_t s);
  // One application of the preconditioner (the cycle, and the learned stage in
  // kLearnedCycle mode) to r, into z.
  void precondition_into(const float* val, const float* r, float* z, cudaStream_t s);
  // Throws TimeoutError if the attached stage recorded a device fault.
  void check_learned(cudaStream_t s) {
    if (learned_ != nullptr) learned_->check(s);
  }

 private:
  struct Graph {
    const void* k1;
    const void* k2;
    int k3;
    cudaGraphExec_t exec;
    long long launches;  // kernels in the graph
    double bytes;        // their algorithmic bytes
  };
  // Whether device work may go through captured graphs now (not while
  // profiling, whose events sample individual sweeps, nor inside a capture).
  bool graphing() const {
    return options_.graphs && graphs_usable_ && !profiling_ && !capturing_;
  }
  void graphed(const void* k1, const void* k2, int k3, float* const& tracked,
               const std::function<void()>& work);
  std::vector<const float*> roles(const float* z) const;
  std::vector<Graph> graphs_;
  bool graphs_usable_ = true;
  bool capturing_ = false;
  cudaStream_t capture_ = nullptr;
  // Work queued by cycle/smooth/inner is skipped on the device while
  // status[0] != 0 (the outer solve's status, or a K-cycle level's own).
  void cycle(std::size_t index, const float* b, float*& x, const int* status);
  void inner(std::size_t index, const int* parent);
  void smooth(DevLevel& l, const int* rows, const int* cols, const float* vals, const float* b,
              float*& x, int sweeps, bool zero_start, const int* status);
  void reduce_into(ReduceMode mode, int n, const float* x, const float* y, const float* u,
                   const float* v, float* scalars, int offset, const int* guard);

  // Krylov driver (solver.cpp:97-393).
  bool verified(float* x, const float* b, double target, Stats& stats);
  bool diverged(const Stats& stats) const {
    return !std::isfinite(stats.final_residual) ||
           stats.final_residual > 1e3 * stats.initial_residual;
  }
  std::vector<int> poll(const float* x, const float* b);
  bool replacement(float* x, const float* b, double target, Stats& stats, int& restarts,
                   double& last_verified);
  void pcg(float* x, const float* b, const Control& c, double target, Stats& stats);
  void bicgstab(float* x, const float* b, const Control& c, double target, Stats& stats);
  int batch_interval(const Control& c) const {
    return previous_iterations_ > 0 && previous_iterations_ < c.residual_check_interval
               ? previous_iterations_ + 1
               : c.residual_check_interval;
  }
  float* speculative_r() { return bicg() ? t_ : q_; }
  float*& speculative_x() { return bicg() ? s_ : z_; }
  DeviceReducer reducer() const { return DeviceReducer{partials_.get(), ticket_.get()}; }

  Kind kind_;
  Options options_;
  int n_, nnz_;
  bool nullspace_;
  int device_ = 0;
  std::shared_ptr<Workspace> workspace_;
  std::vector<DevLevel> levels_;
  double complexity_ = 0;
  DArray<float> jacobi_inverse_;  // Jacobi preconditioner
  DArray<float> surplus_;         // M-matrix diagonal scratch (fine rows)
  float *r_ = nullptr, *z_ = nullptr, *p_ = nullptr, *q_ = nullptr, *shadow_ = nullptr,
        *s_ = nullptr, *t_ = nullptr, *zs_ = nullptr, *best_ = nullptr, *scratch_ = nullptr;
  DArray<float> scalars_, projection_;
  DArray<int> status_;
  DArray<double> partials_, values_;
  DArray<unsigned> ticket_;
  Pinned<double> host_values_{64};
  Pinned<int> host_status_{4};
  bool speculate_ = false;
  std::optional<double> speculated_;
  double best_residual_ = 0;
  int previous_iterations_ = 0;
  bool verified_current_ = false;
  // Per-call state.
  cudaStream_t stream_ = nullptr;
  const float* val_ = nullptr;
  // Measurement.
  void tally(double bytes) {
    if (profiling_) prof_.algorithmic_bytes += bytes;
  }
  void collect_events();
  bool profiling_ = false;
  Profile prof_;
  long long launch_mark_ = 0;
  std::vector<cudaEvent_t> events_;
  std::vector<double> event_bytes_;  // algorithmic bytes of each timed sweep
  double timed_bytes_ = 0;
  std::size_t events_used_ = 0;
  long long sampled_ = 0;
};

}  // namespace kb2
