// The AMG hierarchy built on the device (the Aggregation constructor,
// amg.cpp:160-226): pairing passes, their composition, the coarse pattern and
// entry map, and the coarse values through the refresh kernels. The results
// equal the host setup's (setup.cpp) bit for bit; the kernels are in
// cuda/setup_kernels.cu.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "../cuda/kernels.hpp"
#include "solver.hpp"

namespace kb2 {
namespace {

constexpr int kSweepBatch = 8;  // sweeps between convergence readbacks

// Sweeps allowed before giving up. The equations are triangular, so each
// sweep settles at least the next row in dependence order and n + 1 sweeps
// always reach the fixed point; meshes need about 50-90.
int sweep_limit(int n) { return std::max(1 << 14, n + 2); }
constexpr double kAbsorbCoupling = 0.01;

int read_int(const int* d, cudaStream_t s) {
  int v = 0;
  cuda_check(cudaMemcpyAsync(&v, d, sizeof(int), cudaMemcpyDeviceToHost, s), "setup readback");
  wait(s);
  return v;
}

void zero(DArray<int>& a, std::size_t n, cudaStream_t s) {
  if (a.size() < n || !a.allocated()) a.reset(n);
  cuda_check(cudaMemsetAsync(a.get(), 0, sizeof(int) * std::max<std::size_t>(n, 1), s), "memset");
}
// The builder's scratch is stream-ordered (SArray): freeing it neither
// synchronises the device nor pays cudaMalloc's cost again on the next pass.
void zero(SArray<int>& a, std::size_t n, cudaStream_t s) {
  if (a.size() < n || !a.allocated()) a.reset(n, s);
  cuda_check(cudaMemsetAsync(a.get(), 0, sizeof(int) * std::max<std::size_t>(n, 1), s), "memset");
}

// A device CSR operator of the setup (a level, or an intermediate operator).
struct Operator {
  int n = 0, nnz = 0;
  const int* rows = nullptr;
  const int* cols = nullptr;
  const int* diag = nullptr;
  const float* vals = nullptr;
};

// The coarse operator of an aggregation and its transfer.
struct Coarse {
  int n = 0, nnz = 0, active = 0;
  DArray<int> row_ptr, col, diag, member_offsets, members, entry_offsets, entries;
  DArray<float> val;
  Operator view() const { return {n, nnz, row_ptr.get(), col.get(), diag.get(), val.get()}; }
};

class Builder {
 public:
  Builder(const Options& o, cudaStream_t s) : o_(o), s_(s) {}

  // out[0..n] = exclusive scan of in[0..n); returns the total.
  int scan(int n, const int* in, int* out) {
    const auto need = static_cast<std::size_t>(launch::scan_scratch(n));
    if (blocks_.size() < need) blocks_.reset(need, s_);
    launch::exclusive_scan(n, in, out, blocks_.get(), s_);
    return read_int(out + n, s_);
  }

  // pairs(), amg.cpp:25-75, with the singleton absorption of the mixed
  // hierarchy: map[i] = aggregate of row i (-1 left out); returns their count.
  int pair(const Operator& a, bool exclude_isolated, DArray<int>& map) {
    const int n = a.n;
    const auto rows = static_cast<std::size_t>(n);
    SArray<int> count(rows + 1, s_), offsets(rows + 1, s_), state(rows, s_), next(rows, s_),
        owner(rows, s_);
    launch::pair_count(n, a.rows, a.cols, a.vals, o_.strength_threshold, exclude_isolated ? 1 : 0,
                       count.get(), state.get(), s_);
    const int total = scan(n, count.get(), offsets.get());
    SArray<unsigned long long> keys(static_cast<std::size_t>(total), s_);
    SArray<int> pref(static_cast<std::size_t>(total), s_);
    launch::pair_fill(n, a.rows, a.cols, a.vals, o_.strength_threshold, offsets.get(), keys.get(),
                      pref.get(), s_);
    int* cur = state.get();
    int* nxt = next.get();
    SArray<int> changed(kSweepBatch, s_);
    for (int sweeps = 0;; sweeps += kSweepBatch) {
      KB2_REQUIRE(sweeps < sweep_limit(n), "device aggregation: pairing did not settle");
      cuda_check(cudaMemsetAsync(changed.get(), 0, sizeof(int) * kSweepBatch, s_), "memset");
      for (int k = 0; k < kSweepBatch; ++k) {
        launch::pair_sweep(n, offsets.get(), pref.get(), owner.get(), cur, nxt, changed.get() + k, s_);
        std::swap(cur, nxt);
      }
      int flags[kSweepBatch];
      cuda_check(cudaMemcpyAsync(flags, changed.get(), sizeof(flags), cudaMemcpyDeviceToHost, s_),
                 "setup readback");
      wait(s_);
      // A sweep that changed nothing found the fixed point; the later sweeps
      // of the batch left it (and the claims computed from it) as they were.
      if (std::find(flags, flags + kSweepBatch, 0) != flags + kSweepBatch) break;
    }
    SArray<int> leader(rows + 1, s_), id(rows + 1, s_);
    launch::pair_leaders(n, cur, leader.get(), s_);
    const int nc = scan(n, leader.get(), id.get());
    map.reset(rows);
    launch::pair_assign(n, cur, owner.get(), id.get(), map.get(), s_);
    return o_.absorb_singletons ? absorb(a, nc, map) : nc;
  }

  // The absorption pass of setup.cpp's pairs(): singletons join the pair of
  // their strongest strongly coupled neighbour; aggregates renumbered in order.
  int absorb(const Operator& a, int nc, DArray<int>& map) {
    const int n = a.n;
    const auto rows = static_cast<std::size_t>(n);
    SArray<int> size0;
    zero(size0, static_cast<std::size_t>(nc), s_);
    launch::aggregate_sizes(n, map.get(), size0.get(), s_);
    SArray<int> first(rows, s_), second(rows, s_);
    cuda_check(cudaMemcpyAsync(first.get(), map.get(), sizeof(int) * rows, cudaMemcpyDeviceToDevice,
                               s_),
               "copy");
    int* cur = first.get();
    int* nxt = second.get();
    SArray<int> changed(kSweepBatch, s_);
    for (int sweeps = 0;; sweeps += kSweepBatch) {
      KB2_REQUIRE(sweeps < sweep_limit(n), "device aggregation: absorption did not settle");
      cuda_check(cudaMemsetAsync(changed.get(), 0, sizeof(int) * kSweepBatch, s_), "memset");
      for (int k = 0; k < kSweepBatch; ++k) {
        launch::absorb_sweep(n, a.rows, a.cols, a.diag, a.vals, o_.strength_threshold,
                             kAbsorbCoupling, map.get(), size0.get(), cur, nxt,
                             changed.get() + k, s_);
        std::swap(cur, nxt);
      }
      int flags[kSweepBatch];
      cuda_check(cudaMemcpyAsync(flags, changed.get(), sizeof(flags), cudaMemcpyDeviceToHost, s_),
                 "setup readback");
      wait(s_);
      if (std::find(flags, flags + kSweepBatch, 0) != flags + kSweepBatch) break;
    }
    SArray<int> used, renumber(static_cast<std::size_t>(nc) + 1, s_);
    zero(used, static_cast<std::size_t>(nc) + 1, s_);
    launch::mark_used(n, cur, used.get(), s_);
    const int kept = scan(nc, used.get(), renumber.get());
    launch::compose(n, cur, renumber.get(), s_);
    cuda_check(cudaMemcpyAsync(map.get(), cur, sizeof(int) * rows, cudaMemcpyDeviceToDevice, s_),
               "copy");
    return kept;
  }

  // coarsen(), amg.cpp:77-158: pattern, transfer and entry map on the device;
  // values by the refresh kernels over the entry map.
  void coarsen(const Operator& fine, const int* aggregate, int nc, Coarse& c) {
    const auto count = static_cast<std::size_t>(nc);
    c.n = nc;
    SArray<int> size, triples;
    zero(size, count + 1, s_);
    zero(triples, count + 1, s_);
    launch::coarsen_count(fine.n, fine.rows, fine.cols, aggregate, size.get(), triples.get(), s_);
    c.member_offsets.reset(count + 1);
    c.active = scan(nc, size.get(), c.member_offsets.get());
    SArray<int> triple_offsets(count + 1, s_);
    const int total = scan(nc, triples.get(), triple_offsets.get());
    c.members.reset(static_cast<std::size_t>(c.active));
    zero(size, count + 1, s_);  // placement cursors
    launch::place_members(fine.n, aggregate, c.member_offsets.get(), size.get(), c.members.get(),
                          s_);
    launch::sort_members(nc, c.member_offsets.get(), c.members.get(), s_);
    SArray<int4> sorted(static_cast<std::size_t>(total), s_);
    SArray<int> unique(count + 1, s_);
    launch::coarsen_triples(nc, fine.rows, fine.cols, aggregate, c.member_offsets.get(),
                            c.members.get(), triple_offsets.get(), o_.m_matrix ? 1 : 0,
                            sorted.get(), unique.get(), s_);
    c.row_ptr.reset(count + 1);
    c.nnz = scan(nc, unique.get(), c.row_ptr.get());
    const auto nnz = static_cast<std::size_t>(c.nnz);
    c.col.reset(nnz);
    c.diag.reset(count);
    c.entry_offsets.reset(nnz + 1);
    c.entries.reset(static_cast<std::size_t>(total));
    launch::coarsen_fill(nc, triple_offsets.get(), sorted.get(), c.row_ptr.get(), c.col.get(),
                         c.diag.get(), c.entry_offsets.get(), c.entries.get(), s_);
    total_host_ = total;
    cuda_check(cudaMemcpyAsync(c.entry_offsets.get() + nnz, &total_host_, sizeof(int),
                               cudaMemcpyHostToDevice, s_),
               "upload");
    c.val.reset(nnz);
    launch::galerkin(c.nnz, c.entry_offsets.get(), c.entries.get(), fine.vals, c.val.get(), s_);
    if (o_.m_matrix) {
      SArray<float> surplus(static_cast<std::size_t>(fine.n), s_);
      launch::m_matrix_diagonal(fine.n, nc, c.member_offsets.get(), c.members.get(), fine.rows,
                                fine.diag, fine.vals, c.row_ptr.get(), c.diag.get(), c.val.get(),
                                surplus.get(), s_);
    }
    wait(s_);  // total_host_ is read by the copy above
  }

  // aggregate(), amg.cpp:160-174 (setup.cpp's aggregate()).
  void aggregate(const Operator& a, Coarse& out) {
    DArray<int> map;
    int nc = pair(a, true, map);
    for (int pass = 1; pass < o_.aggregation_passes; ++pass) {
      Coarse intermediate;
      coarsen(a, map.get(), nc, intermediate);
      DArray<int> next;
      nc = pair(intermediate.view(), false, next);
      launch::compose(a.n, map.get(), next.get(), s_);
    }
    coarsen(a, map.get(), nc, out);
    out_map_ = std::move(map);
  }

  DArray<int> take_map() { return std::move(out_map_); }

 private:
  const Options& o_;
  cudaStream_t s_;
  SArray<int> blocks_;
  DArray<int> out_map_;
  int total_host_ = 0;
};

}  // namespace

bool Solver::device_pattern_symmetric(cudaStream_t s) {
  DArray<int> flag;
  zero(flag, 1, s);
  launch::pattern_symmetric(n_, levels_[0].row_ptr.get(), levels_[0].col.get(), flag.get(), s);
  return read_int(flag.get(), s) == 0;
}

// The Aggregation constructor's level loop (amg.cpp:200-226) on the device:
// levels until coarse_rows, max_levels or a stalled coarsening
// (n_c >= 0.85 of the aggregated rows).
void Solver::build_device_levels(const CsrView& a, cudaStream_t s) {
  DArray<float> fine_val;
  {
    std::vector<float> v(a.val, a.val + a.nnz);
    fine_val.upload(v, s);
  }
  Builder b(options_, s);
  const auto slots = static_cast<std::size_t>(std::max(1, options_.max_levels));
  DArray<double> checks(slots), partials(kReducePartials);
  DArray<unsigned> ticket(1);
  cuda_check(cudaMemsetAsync(ticket.get(), 0, sizeof(unsigned), s), "memset");
  std::size_t total_nnz = static_cast<std::size_t>(a.nnz);
  Operator fine{a.n, a.nnz, levels_[0].row_ptr.get(), levels_[0].col.get(), levels_[0].diag.get(),
                fine_val.get()};
  while (fine.n > options_.coarse_rows &&
         levels_.size() < static_cast<std::size_t>(options_.max_levels)) {
    Coarse c;
    b.aggregate(fine, c);
    if (c.active == 0 || static_cast<double>(c.n) >= 0.85 * static_cast<double>(c.active)) break;
    auto& f = levels_.back();
    f.aggregate = b.take_map();
    f.member_offsets = std::move(c.member_offsets);
    f.members = std::move(c.members);
    f.entry_offsets = std::move(c.entry_offsets);
    f.entries = std::move(c.entries);
    total_nnz += static_cast<std::size_t>(c.nnz);
    levels_.emplace_back();
    auto& l = levels_.back();
    l.n = c.n;
    l.nnz = c.nnz;
    l.row_ptr = std::move(c.row_ptr);
    l.col = std::move(c.col);
    l.diag = std::move(c.diag);
    l.val = std::move(c.val);
    l.xa.reset(static_cast<std::size_t>(l.n));
    l.b.reset(static_cast<std::size_t>(l.n));
    l.x = l.xa.get();
    fine = {l.n, l.nnz, l.row_ptr.get(), l.col.get(), l.diag.get(), l.val.get()};
  }
  complexity_ = a.nnz ? static_cast<double>(total_nnz) / a.nnz : 0;
  // Inverse L1 diagonals of every level (solver.cpp:37-53) with the validity
  // checks of the host setup's diagonal_values().
  for (std::size_t i = 0; i < levels_.size(); ++i) {
    auto& l = levels_[i];
    l.l1.reset(static_cast<std::size_t>(l.n));
    launch::diagonal(l.n, l.row_ptr.get(), l.diag.get(), i == 0 ? fine_val.get() : l.val.get(),
                     l.l1.get(), 1, DeviceReducer{partials.get(), ticket.get()}, checks.get(),
                     static_cast<int>(i), s);
  }
  std::vector<double> invalid(levels_.size());
  cuda_check(cudaMemcpyAsync(invalid.data(), checks.get(), sizeof(double) * invalid.size(),
                             cudaMemcpyDeviceToHost, s),
             "setup readback");
  wait(s);
  for (std::size_t i = 0; i < levels_.size(); ++i) {
    KB2_REQUIRE(invalid[i] != 3, "AMG: requires positive diagonals");
    KB2_REQUIRE(invalid[i] <= (nullspace_ && levels_[i].n == 1 ? 1 : 0),
                "solver: invalid values or zero diagonal");
  }
  device_setup_ = true;
}

}  // namespace kb2
