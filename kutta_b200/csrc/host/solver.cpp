// Krylov drivers and the aggregation-AMG preconditioner on sm_100a kernels.
//
// The host-side control flow follows the reference's Krylov class exactly
// (src/kutta/linalg/solver.cpp:75-393: batched status polls, reliable residual
// replacement, best-iterate restore, small-system speculation) and its
// Aggregation preconditioner (amg.cpp:198-342: refresh with one host wait,
// V-cycle with ping-pong smoothing), so iteration counts and returned iterates
// follow the reference's. All vector and scalar work runs on the device.
#include "solver.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <numeric>
#include <sstream>

namespace kb2 {

namespace {
constexpr int kSpeculativeRows = 1 << 17;  // solver.cpp:387
}


Solver::Solver(Kind kind, const CsrView& a, const Options& options,
               std::shared_ptr<Workspace> workspace)
    : kind_(kind), options_(options), n_(a.n), nnz_(a.nnz), nullspace_(options.nullspace),
      workspace_(std::move(workspace)) {
  cuda_check(cudaGetDevice(&device_), "cudaGetDevice");
  if (!workspace_) workspace_ = std::make_shared<Workspace>(a.n);
  KB2_REQUIRE(workspace_->rows() == a.n, "Krylov workspace size mismatch");
  cudaStream_t s = nullptr;
  // Level 0 pattern: the solver's own device copy of the caller's pattern.
  levels_.reserve(static_cast<std::size_t>(std::max(1, options.max_levels)));
  levels_.emplace_back();
  {
    auto& l = levels_.back();
    l.n = a.n;
    l.nnz = a.nnz;
    l.row_ptr.reset(static_cast<std::size_t>(a.n) + 1);
    l.row_ptr.upload(a.row_ptr, static_cast<std::size_t>(a.n) + 1, s);
    l.col.reset(static_cast<std::size_t>(a.nnz));
    l.col.upload(a.col, static_cast<std::size_t>(a.nnz), s);
    l.diag.reset(static_cast<std::size_t>(a.n));
    l.diag.upload(a.diag, static_cast<std::size_t>(a.n), s);
  }
  if (amg() && options_.device_setup && device_pattern_symmetric(s)) {
    // Aggregation ctor (amg.cpp:200-226) on the device.
    build_device_levels(a, s);
  } else if (amg()) {
    // Aggregation ctor (amg.cpp:200-226): host hierarchy, then uploads.
    const Hierarchy h = build_hierarchy(a, options_);
    complexity_ = h.complexity;
    for (std::size_t i = 0; i < h.levels.size(); ++i) {
      if (i > 0) {
        levels_.emplace_back();
        auto& l = levels_.back();
        const auto& m = h.levels[i].matrix;
        l.n = m.n;
        l.nnz = m.nnz();
        l.row_ptr.upload(m.row_ptr, s);
        l.col.upload(m.col, s);
        l.diag.upload(m.diag, s);
        std::vector<float> v(m.val.begin(), m.val.end());
        l.val.upload(v, s);
        l.xa.reset(static_cast<std::size_t>(m.n));
        l.b.reset(static_cast<std::size_t>(m.n));
        l.x = l.xa.get();
      }
      auto& l = levels_.back();
      l.l1.upload(h.levels[i].l1, s);
      const auto& t = h.levels[i].transfer;
      if (i + 1 < h.levels.size()) {
        l.aggregate.upload(t.aggregate, s);
        l.member_offsets.upload(t.member_offsets, s);
        l.members.upload(t.members, s);
        l.entry_offsets.upload(t.entry_offsets, s);
        l.entries.upload(t.entries, s);
      }
    }
  }
  if (amg()) {
    for (auto& l : levels_) {
      l.ra.reset(static_cast<std::size_t>(l.n));
      l.r = l.ra.get();
      if (nullspace_) l.projection.reset(2);
    }
    // K-cycle work vectors on the levels reached through inner() (Level ctor,
    // amg.cpp:179-195): every coarse level but the coarsest.
    if (options_.cycle == Cycle::K) {
      for (std::size_t i = 1; i + 1 < levels_.size() && inner_level(i); ++i) {
        auto& l = levels_[i];
        const auto rows = static_cast<std::size_t>(l.n);
        l.za.reset(rows);
        l.p.reset(rows);
        l.q.reset(rows);
        l.t.reset(rows);
        l.scalars.reset(12);
        l.status.reset(1);
        l.z = l.za.get();
        cuda_check(cudaMemsetAsync(l.scalars.get(), 0, 12 * sizeof(float), s), "memset");
        cuda_check(cudaMemsetAsync(l.status.get(), 0, sizeof(int), s), "memset");
      }
    }
  } else {
    // Jacobi preconditioner (solver.cpp:56-73).
    jacobi_inverse_.upload(diagonal_values(a, false, false), s);
  }
  // Krylov ctor (solver.cpp:77-90).
  r_ = workspace_->vector(Workspace::R);
  z_ = workspace_->vector(Workspace::Z);
  if (kind_ != Kind::Jacobi) {
    p_ = workspace_->vector(Workspace::P);
    q_ = workspace_->vector(Workspace::Q);
  }
  if (bicg()) {
    shadow_ = workspace_->vector(Workspace::Shadow);
    s_ = workspace_->vector(Workspace::S);
    t_ = workspace_->vector(Workspace::T);
    zs_ = workspace_->vector(Workspace::Zs);
  }
  best_ = workspace_->vector(Workspace::Best);
  if (!amg()) scratch_ = workspace_->vector(Workspace::Scratch);
  scalars_.reset(24);
  status_.reset(3);
  projection_.reset(nullspace_ ? 2 : 0);
  partials_.reset(kReducePartials);
  values_.reset(64);
  ticket_.reset(1);
  cuda_check(cudaMemsetAsync(ticket_.get(), 0, sizeof(unsigned), s), "memset");
  cuda_check(cudaMemsetAsync(scalars_.get(), 0, 24 * sizeof(float), s), "memset");
  cuda_check(cudaMemsetAsync(status_.get(), 0, 3 * sizeof(int), s), "memset");
  speculate_ = kind_ != Kind::Jacobi && n_ <= kSpeculativeRows;
  if (amg() && (options_.coarse_bf16 || options_.dense_coarsest)) {
    for (std::size_t i = 1; i < levels_.size(); ++i) {
      auto& l = levels_[i];
      if (options_.coarse_bf16) {
        l.v16.reset(static_cast<std::size_t>(l.nnz));
        l.scale.reset(static_cast<std::size_t>(l.n));
      }
    }
    auto& c = levels_.back();
    if (options_.dense_coarsest && levels_.size() > 1 && c.n <= 1024) {
      c.dense_lower.reset(static_cast<std::size_t>(c.n) * c.n);
      c.dense_inverse.reset(static_cast<std::size_t>(c.n) * c.n);
    }
    // Usable before the first refresh, from the setup values.
    prepare_mixed(s, 0);
    cuda_check(cudaMemcpyAsync(host_values_.get(), values_.get(), 2 * sizeof(double),
                               cudaMemcpyDeviceToHost, s),
               "setup readback");
    wait(s);
    KB2_REQUIRE(host_values_[0] == 0, "mixed: coarsest operator is not SPD");
    choose_coarsest(host_values_[1]);
    if (options_.fused_tail && options_.coarse_bf16 && !nullspace_) plan_tail();
    if (options_.packed_fine) plan_packed(a, s);
  }
  wait(s);
}

// The packed rows' pattern: each row's off-diagonal column offsets in column
// order, padded with 0 to the width (4 or 8). Left empty (the CSR kernels
// serve) when a row has more than 8 off-diagonal entries or an offset does
// not fit 16 bits.
void Solver::plan_packed(const CsrView& a, cudaStream_t s) {
  int longest = 0;
  for (int i = 0; i < a.n; ++i) {
    longest = std::max(longest, a.row_ptr[i + 1] - a.row_ptr[i] - 1);
    for (int j = a.row_ptr[i]; j < a.row_ptr[i + 1]; ++j)
      if (std::abs(a.col[j] - i) > 32767) return;
  }
  const int width = longest <= 4 ? 4 : (longest <= 8 ? 8 : 0);
  if (width == 0 || a.n == 0) return;
  // Values from the setup values, as the coarse levels are, until a refresh
  // packs the device values.
  const std::size_t slots = static_cast<std::size_t>(width) * static_cast<std::size_t>(a.n);
  std::vector<short> offsets(slots, 0);
  std::vector<float> values(slots, 0.0f), diagonal(static_cast<std::size_t>(a.n));
  for (int i = 0; i < a.n; ++i) {
    std::size_t k = static_cast<std::size_t>(width) * static_cast<std::size_t>(i);
    for (int j = a.row_ptr[i]; j < a.row_ptr[i + 1]; ++j) {
      if (j == a.diag[i]) continue;
      offsets[k] = static_cast<short>(a.col[j] - i);
      values[k++] = static_cast<float>(a.val[j]);
    }
    diagonal[static_cast<std::size_t>(i)] = static_cast<float>(a.val[a.diag[i]]);
  }
  packed_.offsets.upload(offsets, s);
  packed_.vals.upload(values, s);
  packed_.diag.upload(diagonal, s);
  wait(s);  // the host arrays are released on return
  packed_.width = width;
}

// The tail starts at the first coarse level with at most 16,384 rows (about a
// row per thread of a 16-CTA cluster: larger levels run faster spread over
// every SM) and needs at least two levels. CTA k owns rows
// [k 2^shift, (k + 1) 2^shift) of each level, 2^shift >= ceil(n / cluster).
// Each CTA's shared memory holds, per tail level, full copies of the iterate
// and of the spare vector and its own chunk of the right-hand side
// (2 n + 2^shift floats): under 160 KB for a 16,384-row first level. A plan
// that does not fit the kernel's shared-memory ceiling runs without the tail.
void Solver::plan_tail() {
  constexpr int kTailRows = 1 << 14;
  const std::size_t count = levels_.size();
  // The tail runs plain V-cycles, so it starts below the K-cycle inner levels.
  std::size_t start = 0;
  for (std::size_t i = 1; i < count; ++i)
    if (levels_[i].n <= kTailRows && !(options_.cycle == Cycle::K && inner_level(i))) {
      start = i;
      break;
    }
  if (start == 0 || count - start < 2 || count - start > launch::kMaxTailLevels) return;
  const DevLevel& coarsest = levels_.back();
  for (int cluster : {16, 8}) {
    launch::TailPlan p{};
    p.levels = static_cast<int>(count - start);
    p.pre = options_.pre_sweeps;
    p.post = options_.post_sweeps;
    p.coarse_sweeps = options_.coarse_sweeps;
    p.cluster = cluster;
    p.dense = dense(coarsest) ? coarsest.dense_inverse.get() : nullptr;
    double bytes = 0;
    int shared_floats = 0;
    for (int k = 0; k < p.levels; ++k) {
      const std::size_t i = start + static_cast<std::size_t>(k);
      const DevLevel& l = levels_[i];
      auto& t = p.level[k];
      const int per_cta = (l.n + cluster - 1) / cluster;
      int shift = 0;
      while ((1 << shift) < per_cta) ++shift;
      KB2_REQUIRE(static_cast<long long>(cluster) << shift >= l.n, "tail: chunking");
      t.n = l.n;
      t.shift = shift;
      t.rows = l.row_ptr.get();
      t.cols = l.col.get();
      t.v16 = l.v16.get();
      t.scale = l.scale.get();
      t.inv = l.l1.get();
      const bool last = k + 1 == p.levels;
      t.aggregate = last ? nullptr : l.aggregate.get();
      t.offsets = last ? nullptr : l.member_offsets.get();
      t.members = last ? nullptr : l.members.get();
      t.xg = l.xa.get();
      t.bg = l.b.get();
      // Shared-memory copies, 16-byte aligned: x and spare (n each), the
      // owned right-hand side chunk.
      const auto aligned = [](int floats) { return (floats + 3) & ~3; };
      t.xs = shared_floats;
      shared_floats += aligned(l.n);
      t.rs = shared_floats;
      shared_floats += aligned(l.n);
      t.bs = shared_floats;
      shared_floats += aligned(1 << shift);
      const double sweep = 6.0 * l.nnz + 4.0 * (l.n + 1) + 16.0 * l.n;
      if (!last) {
        const double nc = levels_[start + static_cast<std::size_t>(k) + 1].n;
        bytes += 12.0 * l.n + (p.pre - 1 + p.post) * sweep + (sweep - 4.0 * l.n) +
                 4.0 * (nc + 1) + 8.0 * l.n + 4.0 * nc + 12.0 * l.n + 4.0 * nc;
      } else if (p.dense) {
        bytes += 8.0 * l.n * l.n + 8.0 * l.n;
      } else {
        bytes += 12.0 * l.n + (p.coarse_sweeps - 1) * sweep;
      }
    }
    p.smem_bytes = shared_floats * static_cast<int>(sizeof(float));
    if (!launch::tail_cluster_fits(cluster, p.smem_bytes)) continue;
    tail_ = p;
    tail_start_ = start;
    tail_bytes_ = bytes;
    tail_on_ = true;
    return;
  }
}

// BF16 copies of the coarse operators and the dense inverse of the coarsest,
// from the current FP32 coarse values; the dense SPD check lands in values_[0].
void Solver::prepare_mixed(cudaStream_t s, int slot) {
  double* error = values_.get() + slot;
  cuda_check(cudaMemsetAsync(error, 0, 2 * sizeof(double), s), "memset");
  for (std::size_t i = 1; i < levels_.size(); ++i) {
    auto& l = levels_[i];
    if (l.v16.allocated())
      launch::bf16_pack(l.n, l.row_ptr.get(), l.val.get(), l.v16.get(), l.scale.get(), s);
    if (dense(l))
      launch::dense_inverse(l.n, l.row_ptr.get(), l.col.get(), l.val.get(), l.dense_lower.get(),
                            l.dense_inverse.get(), error, s, error + 1);
  }
}

// The coarsest level is solved with its dense inverse only when that is
// well conditioned: a nearly singular operator (smallest relative Cholesky
// pivot below 1e-6) would multiply the FP32 rounding of the restricted
// right-hand side by up to the inverse of that pivot along its near-null
// vector. Such a level is smoothed instead (coarse_sweeps damped sweeps, as the
// reference treats every coarsest level), leaving those components to the
// Krylov iteration. Graphs captured under the other choice are dropped.
void Solver::choose_coarsest(double smallest_pivot) {
  constexpr double kConditioned = 1e-6;
  const bool ok = dense(levels_.back()) && smallest_pivot >= kConditioned;
  if (ok != dense_ok_) {
    for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
    graphs_.clear();
  }
  dense_ok_ = ok;
}

// ---------------------------------------------------------------- primitives --
void Solver::residual(const float* x, const float* b, float* r) {
  if (packed_.width > 0)
    launch::packed_residual(n_, packed(), x, b, r, nullptr, stream_);
  else
    launch::residual(n_, rows0(), cols0(), val_, x, b, r, nullptr, stream_);
  tally(fine_operator_bytes() + 12.0 * n_);
}

Solver::~Solver() {
  for (auto e : events_) cudaEventDestroy(e);
  for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
  if (capture_) cudaStreamDestroy(capture_);
}

void Solver::check_device() const {
  int device = 0;
  cuda_check(cudaGetDevice(&device), "cudaGetDevice");
  KB2_REQUIRE(device == device_, "solver: device or matrix mismatch");
}

void Solver::set_profile(bool on) {
  profiling_ = on;
  prof_ = Profile{};
  prof_.fine_sweep_bytes = 8.0 * nnz_ + 4.0 * (n_ + 1) + 16.0 * n_;
  launch_mark_ = launch::counter.load();
  events_used_ = 0;
  event_bytes_.clear();
  timed_bytes_ = 0;
}

void Solver::collect_events() {
  std::vector<float> times;
  for (std::size_t k = 0; k + 1 < events_used_; k += 2) {
    float ms = 0;
    cuda_check(cudaEventElapsedTime(&ms, events_[k], events_[k + 1]), "cudaEventElapsedTime");
    times.push_back(ms);
  }
  events_used_ = 0;
  if (!times.empty()) {
    // Sweeps queued after a convergence candidate return at once (status guard);
    // they are not sweeps of the matrix and are left out of the kernel time.
    std::vector<float> sorted = times;
    std::nth_element(sorted.begin(), sorted.begin() + sorted.size() / 2, sorted.end());
    const float median = sorted[sorted.size() / 2];
    for (std::size_t k = 0; k < times.size(); ++k)
      if (times[k] >= 0.25f * median) {
        prof_.fine_sweep_ms += times[k];
        ++prof_.fine_sweeps;
        timed_bytes_ += k < event_bytes_.size() ? event_bytes_[k] : 0.0;
      }
    // The average algorithmic bytes of the timed sweeps (a post-sweep with
    // the flexible PCG's reductions fused also reads q).
    if (prof_.fine_sweeps > 0) prof_.fine_sweep_bytes = timed_bytes_ / prof_.fine_sweeps;
  }
  event_bytes_.clear();
  prof_.launches = launch::counter.load() - launch_mark_;
}

std::vector<double> Solver::host_reduce(std::initializer_list<Request> requests) {
  int slot = 0;
  for (const auto& q : requests) {
    launch::reduce_value(q.mode, q.n, q.x, q.y, reducer(), values_.get(), slot++, stream_);
    tally((q.mode == ReduceMode::Dot && q.x != q.y ? 8.0 : 4.0) * q.n);
  }
  cuda_check(cudaMemcpyAsync(host_values_.get(), values_.get(), sizeof(double) * slot,
                             cudaMemcpyDeviceToHost, stream_),
             "reduction readback");
  wait(stream_);
  cuda_check(cudaGetLastError(), "reduction");
  return std::vector<double>(host_values_.get(), host_values_.get() + slot);
}

double Solver::norm(const float* x) {
  return std::sqrt(host_reduce({{ReduceMode::Dot, x, x, n_}})[0]);
}

void Solver::copy(float* dst, const float* src, int n) {
  if (n > 0 && dst != src) {
    cuda_check(cudaMemcpyAsync(dst, src, sizeof(float) * static_cast<std::size_t>(n),
                               cudaMemcpyDeviceToDevice, stream_),
               "copy");
    tally(8.0 * n);
  }
}

// linalg_detail::project, detail.hpp:13-19.
void Solver::project(float* x, int n, float* projection) {
  if (n == 0) return;
  launch::reduce_into(ReduceMode::Sum, n, x, x, x, x, reducer(), projection, 0, status_.get(),
                      false, Epilogue::None, stream_);
  const float count = static_cast<float>(n);
  launch::project(n, x, projection, count,
                  static_cast<float>(static_cast<double>(n) - static_cast<double>(count)), stream_);
}

void Solver::reset(int iterations) { launch::solver_reset(scalars_.get(), status_.get(), iterations, stream_); }

// ------------------------------------------------------------ preconditioner --
void Solver::smooth(DevLevel& l, const int* rows, const int* cols, const float* vals,
                    const float* b, float*& x, int sweeps, bool zero_start, const int* status) {
  const bool fine = &l == &levels_[0];
  for (int sweep = 0; sweep < sweeps; ++sweep) {
    const bool zero = zero_start && sweep == 0;
    // Every 8th fine-level sweep is bracketed by events: enough samples for the
    // average launch time, little added host work inside a timed solve.
    const bool timed = profiling_ && fine && !zero && (sampled_++ % 8 == 0);
    if (timed) {
      while (events_.size() < events_used_ + 2) {
        cudaEvent_t e;
        cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        events_.push_back(e);
      }
      cuda_check(cudaEventRecord(events_[events_used_++], stream_), "cudaEventRecord");
    }
    // The last sweep of the fine level's post-smoothing (pre-smoothing always
    // starts from zero) carries the fused reductions.
    const bool with_dots = fine && fuse_dots_ && !zero_start && sweep + 1 == sweeps;
    const bool packed_rows = with_dots && packed_.width > 0;
    const double bytes =
        zero ? 12.0 * l.n
             : (packed_rows ? fine_operator_bytes() : 8.0 * l.nnz + 4.0 * (l.n + 1)) +
                   (with_dots ? 20.0 : 16.0) * l.n;
    if (timed) event_bytes_.push_back(bytes);
    if (l.v16.allocated())
      launch::bf16_smooth(l.n, rows, cols, l.v16.get(), l.scale.get(), x, b, l.l1.get(), l.r,
                          status, zero, stream_);
    else if (packed_rows)
      launch::packed_smooth_dot2(l.n, packed(), x, b, l.l1.get(), l.r, q_, reducer(),
                                 scalars_.get(), 4, status_.get(), Epilogue::PcgBetaFlexible,
                                 stream_);
    else if (with_dots)
      launch::smooth_dot2(l.n, rows, cols, vals, x, b, l.l1.get(), l.r, q_, reducer(),
                          scalars_.get(), 4, status_.get(), Epilogue::PcgBetaFlexible, stream_);
    else
      launch::smooth(l.n, rows, cols, vals, x, b, l.l1.get(), l.r, status, zero, stream_);
    if (timed) cuda_check(cudaEventRecord(events_[events_used_++], stream_), "cudaEventRecord");
    tally(bytes);
    std::swap(x, l.r);  // ping-pong: the two buffers exchange roles (amg.cpp:280)
  }
}

// Aggregation::cycle, amg.cpp:283-310.
void Solver::cycle(std::size_t index, const float* b, float*& x, const int* status) {
  auto& l = levels_[index];
  const int* rows = l.row_ptr.get();
  const int* cols = l.col.get();
  const float* vals = index == 0 ? val_ : l.val.get();
  // x is not cleared: every first step below writes it without reading it.
  // While status[0] != 0 nothing is written and x is never read.
  if (tail_on_ && index == tail_start_) {
    // The tail reads its right-hand side from, and leaves its result in, the
    // level's own b and first buffer, which never change roles.
    KB2_REQUIRE(b == l.b.get() && x == l.xa.get(), "tail: unexpected level buffers");
    if (dense_ok_) {
      launch::tail_cycle(tail_, status, stream_);
    } else {
      launch::TailPlan smoothed = tail_;
      smoothed.dense = nullptr;
      launch::tail_cycle(smoothed, status, stream_);
    }
    tally(tail_bytes_);
    return;
  }
  if (index + 1 == levels_.size()) {
    if (dense(l) && dense_ok_) {
      launch::dense_solve(l.n, l.dense_inverse.get(), b, x, status, stream_);
      tally(8.0 * l.n * l.n + 8.0 * l.n);
    } else if (l.n <= 24) {
      launch::coarse_solve(l.n, rows, cols, vals, x, b, l.l1.get(), status,
                           options_.coarse_sweeps, stream_);
    } else {
      smooth(l, rows, cols, vals, b, x, options_.coarse_sweeps, true, status);
    }
  } else {
    smooth(l, rows, cols, vals, b, x, options_.pre_sweeps, true, status);
    if (l.v16.allocated())
      launch::bf16_residual(l.n, rows, cols, l.v16.get(), l.scale.get(), x, b, l.r, status,
                            stream_);
    else if (index == 0 && packed_.width > 0)
      launch::packed_residual(l.n, packed(), x, b, l.r, status, stream_);
    else
      launch::residual(l.n, rows, cols, vals, x, b, l.r, status, stream_);
    auto& c = levels_[index + 1];
    if (mixed())
      launch::restrict_lanes(c.n, l.member_offsets.get(), l.members.get(), l.r, c.b.get(), status,
                             stream_);
    else
      launch::restrict_(c.n, l.member_offsets.get(), l.members.get(), l.r, c.b.get(), status,
                        stream_);
    tally(8.0 * l.nnz + 4.0 * (l.n + 1) + 12.0 * l.n + 4.0 * (c.n + 1) + 8.0 * l.n + 4.0 * c.n);
    if (nullspace_) project(c.b.get(), c.n, c.projection.get());
    if (options_.cycle == Cycle::K && index + 2 < levels_.size() && inner_level(index + 1))
      inner(index + 1, status);
    else
      cycle(index + 1, c.b.get(), c.x, status);
    launch::prolong(l.n, l.aggregate.get(), c.x, x, status, stream_);
    tally(12.0 * l.n + 4.0 * c.n);
    smooth(l, rows, cols, vals, b, x, options_.post_sweeps, false, status);
  }
  if (nullspace_ && index != 0) project(x, l.n, l.projection.get());
}

void Solver::reduce_into(ReduceMode mode, int n, const float* x, const float* y, const float* u,
                         const float* v, float* scalars, int offset, const int* guard) {
  // Without an epilogue the reduction only reads the guard.
  launch::reduce_into(mode, n, x, y, u, v, reducer(), scalars, offset, const_cast<int*>(guard),
                      true, Epilogue::None, stream_);
  tally((mode == ReduceMode::Dot2 ? 16.0 : 8.0) * n);
}

// Aggregation::inner, amg.cpp:312-338: two preconditioned Krylov steps on the
// coarse equation of level `index` (A-conjugate directions for SPD, GCR
// otherwise), leaving the correction in l.x for the prolongation. The first
// cycle runs under the parent's status, the rest under the level's own; a
// reduction is skipped exactly when every reader of its slots is.
void Solver::inner(std::size_t index, const int* parent) {
  auto& l = levels_[index];
  const int n = l.n;
  const int* rows = l.row_ptr.get();
  const int* cols = l.col.get();
  const float* vals = l.val.get();
  const bool spd = kind_ == Kind::AmgPcg;
  float* sc = l.scalars.get();
  int* st = l.status.get();
  float *p = l.p.get(), *q = l.q.get(), *t = l.t.get();
  const double spmv_bytes = 8.0 * l.nnz + 4.0 * (n + 1) + 8.0 * n;

  // A BF16 level (mixed precision, SPD) uses its BF16 operator, with the
  // reductions fused into the kernels that produce their operands.
  const bool bf16 = l.v16.allocated() && spd;
  const double bf16_bytes = 6.0 * l.nnz + 4.0 * (n + 1) + 16.0 * n;

  cycle(index, l.b.get(), l.z, parent);
  copy(p, l.z, n);
  if (bf16) {
    launch::bf16_spmv_dot2(n, rows, cols, l.v16.get(), l.scale.get(), p, l.b.get(), q, false,
                           reducer(), sc, parent, stream_);
    tally(bf16_bytes);
  } else {
    launch::spmv(n, rows, cols, vals, p, q, parent, stream_);
    tally(spmv_bytes);
    reduce_into(ReduceMode::Dot2, n, spd ? p : q, q, l.b.get(), spd ? p : q, sc, 0, parent);
  }
  launch::inner_alpha(sc, st, parent, 1, stream_);
  if (bf16) {
    launch::inner_first_dot(n, l.b.get(), p, q, l.x, t, sc, st, reducer(), stream_);
    tally(24.0 * n);
  } else {
    launch::inner_first(n, l.b.get(), p, q, l.x, t, sc, st, stream_);
    tally(24.0 * n);
    reduce_into(ReduceMode::Dot2, n, t, t, l.b.get(), l.b.get(), sc, 4, st);
  }
  launch::inner_check(sc, st, stream_);
  cycle(index, t, l.z, st);
  if (!spd) {
    launch::spmv(n, rows, cols, vals, l.z, l.r, st, stream_);
    tally(spmv_bytes);
  }
  reduce_into(ReduceMode::Dot, n, spd ? l.z : l.r, q, nullptr, nullptr, sc, 4, st);
  launch::inner_beta(sc, st, stream_);
  launch::direction(n, l.z, p, sc, st, stream_);
  tally(12.0 * n);
  if (bf16) {
    launch::bf16_spmv_dot2(n, rows, cols, l.v16.get(), l.scale.get(), p, t, q, false, reducer(),
                           sc, st, stream_);
    tally(bf16_bytes);
  } else {
    launch::spmv(n, rows, cols, vals, p, q, st, stream_);
    tally(spmv_bytes);
    reduce_into(ReduceMode::Dot2, n, spd ? p : q, q, t, spd ? p : q, sc, 0, st);
  }
  launch::inner_alpha(sc, st, parent, 0, stream_);
  launch::inner_step(n, l.x, p, sc, st, stream_);
  tally(12.0 * n);
}

// Krylov::apply (solver.cpp:197-200) with the AMG (amg.cpp:258-261) or Jacobi
// (solver.cpp:65-68) preconditioner.
void Solver::apply(const float* r, float*& z) {
  if (amg() && graphing()) {
    graphed(r, z, fuse_dots_ ? 1 : 0, z, [&] { precondition(r, z); });
  } else if (amg()) {
    precondition(r, z);
  } else {
    launch::multiply(n_, r, jacobi_inverse_.get(), z, status_.get(), stream_);
  }
  if (nullspace_) project(z, n_, projection_.get());
}

// The AMG cycle, then, with a learned stage attached, its correction of what
// the cycle left: c = G(t) for t = r - A z, added as z += alpha c with the
// energy-minimising alpha = max(0, c.t / c.A c), so a poor network cannot
// make the error larger in the A-norm. The result is a variable
// preconditioner, so the Krylov driver must be the flexible one, as it is for
// the mixed solve.
void Solver::precondition(const float* r, float*& z) {
  cycle(0, r, z, status_.get());
  if (learned_ != nullptr && (learned_mode_ & kLearnedCycle)) {
    float* t = learned_residual_.get();
    launch::residual(n_, rows0(), cols0(), val_, z, r, t, status_.get(), stream_);
    learned_direction(t);
    launch::gnn_step(n_, z, learned_correction_.get(), learned_dots_.get(), stream_);
    tally(8.0 * nnz_ + 4.0 * (n_ + 1) + 12.0 * n_ + 12.0 * n_);
  }
}

void Solver::learned_direction(const float* t) {
  float* c = learned_correction_.get();
  float* q = learned_product_.get();
  learned_->forward(t, c, 0.0f, stream_);
  launch::spmv(n_, rows0(), cols0(), val_, c, q, status_.get(), stream_);
  launch::reduce_value(ReduceMode::Dot, n_, c, t, reducer(), learned_dots_.get(), 0, stream_);
  launch::reduce_value(ReduceMode::Dot, n_, c, q, reducer(), learned_dots_.get(), 1, stream_);
  tally(8.0 * nnz_ + 4.0 * (n_ + 1) + 8.0 * n_ + 16.0 * n_);
}

// The warm start takes the step along c = G(r) that minimises the residual,
// alpha = max(0, r.Ac / Ac.Ac): the solve stops on the residual, and the
// energy-optimal step of the cycle stage can raise it (1.25x on the white-noise
// right-hand side of the pressure matrices here), which costs the refinement
// loop iterations. This step never raises the residual.
void Solver::learned_warm_start(const float* val, const float* r, double* x, cudaStream_t s) {
  if (learned_ == nullptr || !(learned_mode_ & kLearnedWarmStart)) return;
  stream_ = s;
  val_ = val;
  reset(0);
  learned_direction(r);
  const float* q = learned_product_.get();
  launch::reduce_value(ReduceMode::Dot, n_, q, r, reducer(), learned_dots_.get(), 2, stream_);
  launch::reduce_value(ReduceMode::Dot, n_, q, q, reducer(), learned_dots_.get(), 3, stream_);
  launch::gnn_step64(n_, x, learned_correction_.get(), learned_dots_.get() + 2, stream_);
  tally(16.0 * n_ + 20.0 * n_);
}

void Solver::precondition_into(const float* val, const float* r, float* z, cudaStream_t s) {
  KB2_REQUIRE(amg(), "precondition: needs an AMG solver");
  check_device();
  KB2_REQUIRE(n_ == 0 || (r != nullptr && z != nullptr && r != z),
              "precondition: null or aliased vector");
  if (n_ == 0) return;
  stream_ = s;
  val_ = val;
  reset(0);
  precondition(r, z_);
  if (nullspace_) project(z_, n_, projection_.get());
  copy(z, z_, n_);
  check_learned(s);
}

void Solver::set_learned(Gnn* g, int mode) {
  KB2_REQUIRE(g == nullptr || (amg() && variable()),
              "learned stage: needs an AMG solver with the flexible Krylov driver");
  KB2_REQUIRE(g == nullptr || (mode >= 1 && mode <= (kLearnedCycle | kLearnedWarmStart)),
              "learned stage: mode must be a nonempty set of cycle and warm start");
  KB2_REQUIRE(g == nullptr || g->device() == device_,
              "learned stage: built on another device than the solver");
  for (auto& graph : graphs_) cudaGraphExecDestroy(graph.exec);
  graphs_.clear();
  learned_ = g;
  learned_mode_ = g != nullptr ? mode : 0;
  if (g != nullptr) {
    if (!learned_residual_.allocated()) {
      learned_residual_.reset(static_cast<std::size_t>(n_));
      learned_correction_.reset(static_cast<std::size_t>(n_));
      learned_product_.reset(static_cast<std::size_t>(n_));
      learned_dots_.reset(4);
    }
    if (val_ != nullptr) g->bind(n_, rows0(), cols0(), levels_[0].diag.get(), val_, stream_);
  }
}

// Every level's current buffer roles (the ping-pong smoother swaps them).
std::vector<const float*> Solver::roles(const float* z) const {
  std::vector<const float*> out{z};
  for (const auto& l : levels_) {
    out.push_back(l.x);
    out.push_back(l.r);
    out.push_back(l.z);
  }
  return out;
}

// `work` (kernels only, no host waits) as a CUDA graph: captured the first
// time for this key on an internal stream, then launched on the solve stream.
// The ping-pong smoother swaps each level's buffers an even number of times
// per cycle, so the buffer roles after the work equal those before and one
// capture serves every later call with the same key; if a capture finds
// otherwise, graphs are turned off for this solver after that capture has been
// launched once (it is the right work for this call).
void Solver::graphed(const void* k1, const void* k2, int k3, float* const& tracked,
                     const std::function<void()>& work) {
  for (const auto& g : graphs_)
    if (g.k1 == k1 && g.k2 == k2 && g.k3 == k3) {
      cuda_check(cudaGraphLaunch(g.exec, stream_), "cudaGraphLaunch");
      launch::counter += g.launches;
      tally(g.bytes);
      return;
    }
  if (capture_ == nullptr)
    cuda_check(cudaStreamCreateWithFlags(&capture_, cudaStreamNonBlocking), "cudaStreamCreate");
  const auto before = roles(tracked);
  cudaStream_t solve = stream_;
  stream_ = capture_;
  capturing_ = true;
  const long long launches0 = launch::counter.load();
  const double bytes0 = prof_.algorithmic_bytes;
  cudaGraph_t graph = nullptr;
  cuda_check(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal), "capture");
  try {
    work();
  } catch (...) {
    cudaStreamEndCapture(capture_, &graph);
    if (graph) cudaGraphDestroy(graph);
    stream_ = solve;
    capturing_ = false;
    throw;
  }
  const cudaError_t ended = cudaStreamEndCapture(capture_, &graph);
  stream_ = solve;
  capturing_ = false;
  cuda_check(ended, "capture");
  Graph g{k1, k2, k3, nullptr, launch::counter.load() - launches0,
          prof_.algorithmic_bytes - bytes0};
  launch::counter -= g.launches;  // counted when launched
  const cudaError_t made = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  cuda_check(made, "cudaGraphInstantiate");
  cuda_check(cudaGraphLaunch(g.exec, stream_), "cudaGraphLaunch");
  launch::counter += g.launches;
  if (roles(tracked) == before) {
    graphs_.push_back(g);
  } else {
    // Launched in stream order above; CUDA defers the release until it ends.
    cudaGraphExecDestroy(g.exec);
    graphs_usable_ = false;
  }
}

// Krylov::refresh (solver.cpp:92-95) + Aggregation::refresh (amg.cpp:228-256) or
// Jacobi::refresh (solver.cpp:61-64). One host wait for all validity checks.
void Solver::refresh(const float* val, cudaStream_t s) {
  check_device();
  stream_ = s;
  val_ = val;
  if (!amg()) {
    launch::diagonal(n_, rows0(), levels_[0].diag.get(), val, jacobi_inverse_.get(), 0, reducer(),
                     values_.get(), 0, s);
    cuda_check(cudaMemcpyAsync(host_values_.get(), values_.get(), sizeof(double),
                               cudaMemcpyDeviceToHost, s),
               "refresh readback");
    wait(s);
    cuda_check(cudaGetLastError(), "refresh");
    KB2_REQUIRE(host_values_[0] == 0, "Jacobi: invalid values or zero diagonal");
    return;
  }
  refresh_levels(val, false, s);
}

// The pressure matrix assembled from face data into `values` (the level-0
// values from now on) with its right-hand side, and the refresh, in one pass
// over the cells for level 0: the assembly kernel also writes the L1 inverse
// diagonal and its validity flag; the coarse levels follow as in refresh().
void Solver::assemble_refresh(const FvPressure& fv, float* values, float* rhs, cudaStream_t s) {
  KB2_REQUIRE(amg(), "assemble: needs an AMG solver");
  check_device();
  KB2_REQUIRE(fv.offsets && fv.faces && fv.sign && fv.adjacent && fv.entry && fv.coefficient &&
                  fv.flux && values && rhs,
              "assemble: null argument");
  KB2_REQUIRE(fv.reference >= -1 && fv.reference < n_, "assemble: reference cell out of range");
  stream_ = s;
  val_ = values;
  auto& l = levels_[0];
  launch::fv_pressure_assemble_l1(n_, fv.offsets, fv.faces, fv.sign, fv.adjacent, fv.entry,
                                  l.row_ptr.get(), l.diag.get(), fv.coefficient, fv.flux, values,
                                  rhs, fv.reference, l.l1.get(), reducer(), values_.get(), 0, s);
  refresh_levels(values, true, s);
}

void Solver::refresh_levels(const float* val, bool fine_done, cudaStream_t s) {
  const float* matrix = val;
  std::vector<double> allowed;
  if (options_.m_matrix && !surplus_.allocated() && levels_.size() > 1)
    surplus_.reset(static_cast<std::size_t>(n_));
  for (std::size_t i = 0; i < levels_.size(); ++i) {
    auto& l = levels_[i];
    if (i > 0 || !fine_done)
      launch::diagonal(l.n, l.row_ptr.get(), l.diag.get(), matrix, l.l1.get(), 1, reducer(),
                       values_.get(), static_cast<int>(i), s);
    allowed.push_back(nullspace_ && l.n == 1 ? 1 : 0);
    if (i + 1 < levels_.size()) {
      auto& c = levels_[i + 1];
      launch::galerkin(c.nnz, l.entry_offsets.get(), l.entries.get(), matrix, c.val.get(), s);
      if (options_.m_matrix)
        launch::m_matrix_diagonal(l.n, c.n, l.member_offsets.get(), l.members.get(),
                                  l.row_ptr.get(), l.diag.get(), matrix, c.row_ptr.get(),
                                  c.diag.get(), c.val.get(), surplus_.get(), s);
      matrix = c.val.get();
    }
  }
  const int slots = static_cast<int>(levels_.size());
  if (packed_.width > 0)
    launch::pack_rows(n_, packed_.width, rows0(), cols0(), levels_[0].diag.get(), val,
                      packed_.vals.get(), packed_.diag.get(), s);
  if (mixed()) prepare_mixed(s, slots);
  cuda_check(cudaMemcpyAsync(host_values_.get(), values_.get(),
                             sizeof(double) * (slots + (mixed() ? 2 : 0)), cudaMemcpyDeviceToHost, s),
             "refresh readback");
  wait(s);
  cuda_check(cudaGetLastError(), "refresh");
  for (std::size_t i = 0; i < levels_.size(); ++i) {
    const double invalid = host_values_[i];
    KB2_REQUIRE(invalid != 3, "AMG: requires positive diagonals");
    KB2_REQUIRE(invalid <= allowed[i], "AMG: invalid values or zero diagonal");
  }
  if (mixed()) {
    KB2_REQUIRE(host_values_[slots] == 0, "mixed: coarsest operator is not SPD");
    choose_coarsest(host_values_[slots + 1]);
  }
  // The learned stage's edge weights follow the values.
  if (learned_ != nullptr) learned_->bind(n_, rows0(), cols0(), levels_[0].diag.get(), val, s);
}

// --------------------------------------------------------------------- Krylov --
bool Solver::verified(float* x, const float* b, double target, Stats& stats) {
  if (speculated_) {
    // The same kernels already ran on copies of this exact x; adopt them.
    if (nullspace_) copy(x, speculative_x(), n_);
    copy(r_, speculative_r(), n_);
    stats.final_residual = *speculated_;
    speculated_.reset();
  } else {
    if (nullspace_) project(x, n_, projection_.get());
    residual(x, b, r_);
    stats.final_residual = norm(r_);
  }
  verified_current_ = true;
  stats.converged = std::isfinite(stats.final_residual) && stats.final_residual <= target;
  if (stats.final_residual < best_residual_) {
    best_residual_ = stats.final_residual;
    copy(best_, x, n_);
  }
  if (nullspace_) project(r_, n_, projection_.get());
  return stats.converged;
}

std::vector<int> Solver::poll(const float* x, const float* b) {
  if (speculate_) {
    const float* source = x;
    if (nullspace_) {
      copy(speculative_x(), x, n_);
      project(speculative_x(), n_, projection_.get());
      source = speculative_x();
    }
    float* r = speculative_r();
    residual(source, b, r);
    speculated_ = std::sqrt(host_reduce({{ReduceMode::Dot, r, r, n_}})[0]);
  }
  cuda_check(cudaMemcpyAsync(host_status_.get(), status_.get(), 3 * sizeof(int),
                             cudaMemcpyDeviceToHost, stream_),
             "status readback");
  wait(stream_);
  cuda_check(cudaGetLastError(), "solve");
  return {host_status_[0], host_status_[1], host_status_[2]};
}

bool Solver::replacement(float* x, const float* b, double target, Stats& stats, int& restarts,
                         double& last_verified) {
  if (verified(x, b, target, stats) || diverged(stats)) return false;
  restarts = stats.final_residual >= 0.9 * last_verified ? restarts + 1 : 0;
  last_verified = stats.final_residual;
  return restarts < 12;
}

// Krylov::pcg, solver.cpp:271-313. Per update: SpMV fused with p.q and alpha;
// the x/r update fused with r.r and the convergence check; the preconditioner;
// r.z fused with beta; the direction update.
void Solver::pcg(float* x, const float* b, const Control& c, double target, Stats& stats) {
  auto restart = [&] {
    reset(stats.iterations);
    apply(r_, z_);
    copy(p_, z_, n_);
    launch::reduce_into(ReduceMode::Dot, n_, r_, z_, r_, z_, reducer(), scalars_.get(), 0,
                        status_.get(), true, Epilogue::None, stream_);
  };
  restart();
  int restarts = 0;
  double last_verified = stats.initial_residual;
  int check_interval = batch_interval(c);
  while (stats.iterations < c.max_iter) {
    const int batch = std::min(check_interval, c.max_iter - stats.iterations);
    verified_current_ = false;
    speculated_.reset();
    auto iterate = [&](int j) {
      if (packed_.width > 0)
        launch::packed_spmv_dot(n_, packed(), p_, p_, q_, reducer(), scalars_.get(), 2,
                                status_.get(), Epilogue::PcgAlpha, stream_);
      else
        launch::spmv_dot(n_, rows0(), cols0(), val_, p_, p_, q_, reducer(), scalars_.get(), 2,
                         status_.get(), Epilogue::PcgAlpha, stream_);
      launch::pcg_step_dot(n_, x, r_, p_, q_, reducer(), scalars_.get(), status_.get(), stream_);
      tally(fine_operator_bytes() + 8.0 * n_ + 24.0 * n_);
      if (stats.iterations + j + 1 == c.max_iter) return;
      const bool fused = can_fuse_dots();
      fuse_dots_ = fused;
      apply(r_, z_);
      fuse_dots_ = false;
      tally((variable() ? (fused ? 4.0 : 12.0) : 8.0) * n_ + 12.0 * n_);
      if (variable()) {
        if (!fused)
          launch::reduce_into(ReduceMode::Dot2, n_, r_, z_, z_, q_, reducer(), scalars_.get(), 4,
                              status_.get(), true, Epilogue::PcgBetaFlexible, stream_);
      } else
        launch::reduce_into(ReduceMode::Dot, n_, r_, z_, r_, z_, reducer(), scalars_.get(), 4,
                            status_.get(), true, Epilogue::PcgBeta, stream_);
      launch::direction(n_, z_, p_, scalars_.get(), status_.get(), stream_);
    };
    // A batch of whole iterations between two status polls is one graph.
    if (amg() && graphing() && stats.iterations + batch < c.max_iter)
      graphed(x, r_, -batch, z_, [&] {
        for (int j = 0; j < batch; ++j) iterate(j);
      });
    else
      for (int j = 0; j < batch; ++j) iterate(j);
    const auto state = poll(x, b);
    stats.iterations = state[1];
    if (state[0] == 2) break;
    if (state[0] == 1) {
      if (!replacement(x, b, target, stats, restarts, last_verified) ||
          stats.iterations == c.max_iter)
        break;
      // Within 10x of the target the verified residual is close to what FP32
      // can resolve, so a restarted batch may stop after a single update: poll
      // after every update from here on.
      if (stats.final_residual <= 10 * target) check_interval = 1;
      restart();
    }
  }
}

// Krylov::bicgstab, solver.cpp:314-361.
void Solver::bicgstab(float* x, const float* b, const Control& c, double target, Stats& stats) {
  auto restart = [&] {
    reset(stats.iterations);
    copy(shadow_, r_, n_);
    launch::fill(n_, p_, 0.0f, stream_);
    launch::fill(n_, q_, 0.0f, stream_);
  };
  restart();
  int restarts = 0;
  double last_verified = stats.initial_residual;
  int check_interval = batch_interval(c);
  float* sc = scalars_.get();
  while (stats.iterations < c.max_iter) {
    const int batch = std::min(check_interval, c.max_iter - stats.iterations);
    verified_current_ = false;
    speculated_.reset();
    for (int j = 0; j < batch; ++j) {
      (void)j;
      launch::reduce_into(ReduceMode::Dot, n_, shadow_, r_, shadow_, r_, reducer(), sc, 0,
                          status_.get(), true, Epilogue::BicgBeta, stream_);
      launch::bicg_direction(n_, r_, q_, p_, sc, status_.get(), stream_);
      apply(p_, z_);
      launch::spmv_dot(n_, rows0(), cols0(), val_, z_, shadow_, q_, reducer(), sc, 2,
                       status_.get(), Epilogue::BicgAlpha, stream_);
      launch::bicg_difference(n_, r_, q_, s_, sc, status_.get(), stream_);
      launch::reduce_into(ReduceMode::Dot, n_, s_, s_, s_, s_, reducer(), sc, 16, status_.get(),
                          true, Epilogue::BicgS, stream_);
      apply(s_, zs_);
      launch::spmv(n_, rows0(), cols0(), val_, zs_, t_, status_.get(), stream_);
      launch::reduce_into(ReduceMode::Dot2, n_, t_, t_, t_, s_, reducer(), sc, 2, status_.get(),
                          true, Epilogue::BicgOmega, stream_);
      launch::bicg_step(n_, x, r_, z_, zs_, s_, t_, sc, status_.get(), stream_);
      launch::reduce_into(ReduceMode::Dot, n_, r_, r_, r_, r_, reducer(), sc, 18, status_.get(),
                          true, Epilogue::CheckBicg, stream_);
      tally(2.0 * (8.0 * nnz_ + 4.0 * (n_ + 1)) + 104.0 * n_);
    }
    const auto state = poll(x, b);
    stats.iterations = state[1];
    if (state[0] == 2) break;
    if (state[0] == 1) {
      if (!replacement(x, b, target, stats, restarts, last_verified) ||
          stats.iterations == c.max_iter)
        break;
      if (stats.final_residual <= 10 * target) check_interval = 1;
      restart();
    }
  }
}

// Krylov::solve, solver.cpp:97-176.
Stats Solver::solve(const float* val, float* x, const float* b, const Control& c, cudaStream_t s) {
  check_device();
  stream_ = s;
  val_ = val;
  KB2_REQUIRE((n_ == 0 || (x != nullptr && b != nullptr)) && (x != b || n_ == 0),
              "solve: vector size or alias mismatch");
  KB2_REQUIRE(c.max_iter >= 0 && std::isfinite(c.rel_tol) && c.rel_tol >= 0 &&
                  std::isfinite(c.abs_tol) && c.abs_tol >= 0 && c.residual_check_interval > 0,
              "solve: invalid control");
  speculated_.reset();
  if (!nullspace_) residual(x, b, r_);
  const auto entry = nullspace_
      ? host_reduce({{ReduceMode::Dot, b, b, n_}, {ReduceMode::Dot, x, x, n_},
                     {ReduceMode::Sum, b, b, n_}})
      : host_reduce({{ReduceMode::Dot, b, b, n_}, {ReduceMode::Dot, x, x, n_},
                     {ReduceMode::Dot, r_, r_, n_}});
  const double bnorm = std::sqrt(entry[0]);
  if (!(std::isfinite(bnorm) && std::isfinite(std::sqrt(entry[1]))))
    throw NonfiniteError("solve: nonfinite input vector");
  Stats stats;
  if (nullspace_) {
    if (n_ != 0) {
      KB2_REQUIRE(std::fabs(entry[2]) <= 1e-6 * std::sqrt(static_cast<double>(n_)) * bnorm,
                  "solve: incompatible RHS for constant Neumann nullspace");
      project(x, n_, projection_.get());
    }
    residual(x, b, r_);
    stats.initial_residual = norm(r_);
  } else {
    stats.initial_residual = std::sqrt(entry[2]);
  }
  stats.final_residual = stats.initial_residual;
  verified_current_ = true;
  const double target = std::max(c.abs_tol, c.rel_tol * stats.initial_residual);
  if (!std::isfinite(stats.initial_residual)) return stats;
  if (stats.final_residual <= target) {
    stats.converged = true;
    return stats;
  }
  if (nullspace_) project(r_, n_, projection_.get());
  best_residual_ = stats.initial_residual;
  copy(best_, x, n_);
  if (kind_ != Kind::Jacobi) {
    std::array<float, 4> limits{};
    auto pair = [&](int at, double value) {
      limits[at] = static_cast<float>(value);
      limits[at + 1] = std::isfinite(limits[at])
                           ? static_cast<float>(value - static_cast<double>(limits[at]))
                           : 0.0f;
    };
    pair(0, target * target);
    pair(2, 1e6 * stats.initial_residual * stats.initial_residual);
    launch::solver_limits(scalars_.get(), limits[0], limits[1], limits[2], limits[3], stream_);
  }
  reset(0);
  if (kind_ == Kind::Jacobi) {
    for (int i = 0; i < c.max_iter; ++i) {
      apply(r_, z_);
      launch::axpy(n_, x, z_, 2.0f / 3.0f, stream_);
      verified_current_ = false;
      ++stats.iterations;
      if (stats.iterations % c.residual_check_interval == 0 || stats.iterations == c.max_iter) {
        if (verified(x, b, target, stats) || diverged(stats)) break;
      } else {
        residual(x, b, r_);
      }
    }
  } else if (kind_ == Kind::PcgJacobi || kind_ == Kind::AmgPcg) {
    pcg(x, b, c, target, stats);
  } else {
    bicgstab(x, b, c, target, stats);
  }
  // All exits report the actual residual; restore the best verified iterate.
  if (!verified_current_ || nullspace_) verified(x, b, target, stats);
  if (!std::isfinite(stats.final_residual) || stats.final_residual > best_residual_) {
    copy(x, best_, n_);
    verified(x, b, target, stats);
  }
  previous_iterations_ = stats.converged ? stats.iterations : 0;
  wait(stream_);
  cuda_check(cudaGetLastError(), "solve");
  if (profiling_) {
    collect_events();
    ++prof_.solves;
  }
  return stats;
}

std::string Solver::describe() const {
  const char* name = kind_ == Kind::Jacobi
                         ? "damped Jacobi"
                         : (kind_ == Kind::PcgJacobi || kind_ == Kind::AmgPcg
                                ? (variable() ? "flexible PCG" : "PCG")
                                : "BiCGStab");
  std::ostringstream out;
  out << name << ", ";
  if (amg()) {
    out << "aggregation AMG " << (options_.cycle == Cycle::K ? 'K' : 'V') << "-cycle, "
        << levels_.size() << " levels, op complexity " << std::fixed << std::setprecision(3)
        << complexity_;
    if (mixed())
      out << " (" << (options_.cycle == Cycle::K ? 'K' : 'V') << "(" << options_.pre_sweeps
          << "," << options_.post_sweeps << ")"
          << (options_.cycle == Cycle::K && options_.k_levels > 0
                  ? ", inner Krylov steps on levels 1-" + std::to_string(options_.k_levels)
                  : std::string())
          << (options_.absorb_singletons ? ", singletons absorbed" : "")
          << (options_.coarse_bf16 ? ", BF16 coarse levels" : "")
          << (dense(levels_.back())
                  ? (dense_ok_ ? ", dense FP64 coarsest"
                               : ", nearly singular coarsest smoothed instead of its dense inverse")
                  : "");
    if (packed_.width > 0) out << ", packed fine rows";
    if (tail_on_)
      out << ", levels " << tail_start_ << "-" << levels_.size() - 1 << " in one "
          << tail_.cluster << "-CTA cluster launch";
    if (learned_mode_ & kLearnedCycle) out << ", learned stage";
    if (learned_mode_ & kLearnedWarmStart) out << ", learned warm start";
    if (mixed()) out << ")";
  } else {
    out << "Jacobi";
  }
  if (nullspace_) out << ", constant-nullspace projection";
  return out.str();
}

}  // namespace kb2
