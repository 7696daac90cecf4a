// Host-side AMG setup. Follows the reference's aggregation exactly: the same
// greedy matching order, tie-breaking and double-precision threshold test, and
// the same float compensated sums in the same order, so aggregates, coarse
// patterns and coarse values are bit-identical (src/kutta/linalg/amg.cpp).
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <thread>
#include <tuple>
#include <vector>

namespace kb2 {
namespace {

// Upward-rounded float sums (src/kutta/kernels/prelude.h:82-100): TwoSum keeps
// the high-word error; only the low-word accumulation rounds up.
float add_up(float a, float b) {
  const float sum = a + b;
  const float part = sum - a;
  const float error = (a - (sum - part)) + (b - part);
  return error > 0.0f ? std::nextafter(sum, std::numeric_limits<float>::infinity()) : sum;
}
struct UpperSum {
  float sum, error;
};
UpperSum upper_add(UpperSum a, float b) {
  const float sum = a.sum + b;
  const float part = sum - a.sum;
  const float error = (a.sum - (sum - part)) + (b - part);
  return {sum, add_up(a.error, error)};
}
float upper_value(UpperSum a) { return add_up(a.sum, a.error); }

// Index of entry (row, column) in a sorted CSR row (lower_bound).
inline int find_entry(const CsrView& a, int row, int column) {
  const int* first = a.col + a.row_ptr[row];
  const int* last = a.col + a.row_ptr[row + 1];
  return static_cast<int>(std::lower_bound(first, last, column) - a.col);
}

struct Coarsening {
  HostCsr matrix;
  Transfer t;
};

// coarsen(), amg.cpp:77-158. Aggregate row g gathers (coarse column,
// canonical entry, source entry) over its members' entries, sorts them, and
// sums each coarse entry with Neumaier's compensation in that order. For an
// M-matrix the canonical entry is the smaller of an edge's two CSR positions,
// so opposite coarse entries sum the same floats in the same order; the
// diagonal is rebuilt as the upward-rounded sum of fine row surpluses minus the
// coarse off-diagonals.
Coarsening coarsen(const CsrView& fine, std::vector<int> aggregate, bool entry_map,
                   bool m_matrix) {
  Coarsening c;
  c.t.aggregate = std::move(aggregate);
  const auto& agg = c.t.aggregate;
  const int nc = agg.empty() ? 0 : *std::max_element(agg.begin(), agg.end()) + 1;
  auto& cp = c.matrix;
  cp.n = nc;
  cp.row_ptr.assign(static_cast<std::size_t>(nc) + 1, 0);
  cp.diag.assign(static_cast<std::size_t>(nc), 0);
  auto& offsets = c.t.member_offsets;
  offsets.assign(static_cast<std::size_t>(nc) + 1, 0);
  for (int g : agg)
    if (g >= 0) ++offsets[g + 1];
  std::partial_sum(offsets.begin(), offsets.end(), offsets.begin());
  auto& members = c.t.members;
  members.resize(offsets.back());
  {
    std::vector<int> cursor(offsets.begin(), offsets.end() - 1);
    for (int i = 0; i < fine.n; ++i)
      if (agg[i] >= 0) members[cursor[agg[i]]++] = i;
  }
  if (entry_map) {
    c.t.entries.reserve(fine.nnz);
    c.t.entry_offsets.reserve(fine.nnz / 2 + 2);
    c.t.entry_offsets.push_back(0);
  }
  cp.col.reserve(fine.nnz / 2 + 1);
  cp.val.reserve(fine.nnz / 2 + 1);
  std::vector<std::tuple<int, int, int>> row;
  for (int g = 0; g < nc; ++g) {
    row.clear();
    for (int m = offsets[g]; m < offsets[g + 1]; ++m) {
      const int i = members[m];
      for (int j = fine.row_ptr[i]; j < fine.row_ptr[i + 1]; ++j) {
        const int target = agg[fine.col[j]];
        if (target < 0) continue;
        int canonical = j;
        if (m_matrix) canonical = std::min(j, find_entry(fine, fine.col[j], i));
        row.emplace_back(target, canonical, j);
      }
    }
    std::sort(row.begin(), row.end());
    int previous = -1;
    float sum = 0, error = 0;
    for (const auto& [column, canonical, source] : row) {
      (void)canonical;
      if (column != previous) {
        if (previous != -1) cp.val.back() = sum + error;
        sum = error = 0;
        if (entry_map && previous != -1)
          c.t.entry_offsets.push_back(static_cast<int>(c.t.entries.size()));
        if (column == g) cp.diag[g] = static_cast<int>(cp.col.size());
        cp.col.push_back(column);
        cp.val.push_back(0);
        previous = column;
      }
      if (entry_map) c.t.entries.push_back(source);
      const float term = static_cast<float>(fine.val[source]);
      const float next = sum + term;
      error += std::fabs(sum) >= std::fabs(term) ? (sum - next) + term : (term - next) + sum;
      sum = next;
    }
    if (previous != -1) cp.val.back() = sum + error;
    if (entry_map) c.t.entry_offsets.push_back(static_cast<int>(c.t.entries.size()));
    cp.row_ptr[g + 1] = static_cast<int>(cp.col.size());
    if (m_matrix) {
      UpperSum diagonal{0, 0};
      for (int m = offsets[g]; m < offsets[g + 1]; ++m) {
        const int i = members[m];
        UpperSum surplus{static_cast<float>(fine.val[fine.diag[i]]), 0};
        for (int j = fine.row_ptr[i]; j < fine.row_ptr[i + 1]; ++j)
          if (j != fine.diag[i]) surplus = upper_add(surplus, static_cast<float>(fine.val[j]));
        diagonal = upper_add(diagonal, upper_value(surplus));
      }
      for (int j = cp.row_ptr[g]; j < cp.row_ptr[g + 1]; ++j)
        if (j != cp.diag[g]) diagonal = upper_add(diagonal, -static_cast<float>(cp.val[j]));
      cp.val[cp.diag[g]] = upper_value(diagonal);
    }
  }
  return c;
}

// aggregate(), amg.cpp:160-174: one pairing pass on the fine matrix, then
// passes on the intermediate coarse operator (rebuilt from the fine matrix each
// time), composing the maps; the final transfer carries the entry map.
Coarsening aggregate(const CsrView& a, const Options& o) {
  auto map = pairs(a, o.strength_threshold, true, o.absorb_singletons);
  for (int pass = 1; pass < o.aggregation_passes; ++pass) {
    auto intermediate = coarsen(a, std::move(map), false, o.m_matrix);
    const auto next = pairs(CsrView::of(intermediate.matrix), o.strength_threshold, false,
                            o.absorb_singletons);
    map = std::move(intermediate.t.aggregate);
    for (auto& g : map)
      if (g >= 0) g = next[g];
  }
  return coarsen(a, std::move(map), true, o.m_matrix);
}

}  // namespace

// pairs(), amg.cpp:25-75. Strength of (i, j) is max(|a_ij|, |a_ji|) over the
// union of row i and column i (CSR transpose), the diagonal and zero weights
// excluded. Rows are visited in order; an unassigned row takes the strongest
// unassigned neighbour whose weight is >= threshold * its strongest weight
// (strict > keeps the lowest column on ties). With exclude_isolated, rows with
// no nonzero neighbour stay unassigned (-1).
std::vector<int> pairs(const CsrView& a, double threshold, bool exclude_isolated,
                       bool absorb_singletons) {
  const int n = a.n;
  std::vector<int> offsets(static_cast<std::size_t>(n) + 1, 0), sources(a.nnz);
  for (int j = 0; j < a.nnz; ++j) ++offsets[a.col[j] + 1];
  std::partial_sum(offsets.begin(), offsets.end(), offsets.begin());
  {
    std::vector<int> cursor(offsets.begin(), offsets.end() - 1);
    for (int i = 0; i < n; ++i)
      for (int j = a.row_ptr[i]; j < a.row_ptr[i + 1]; ++j) sources[cursor[a.col[j]]++] = i;
  }
  std::vector<int> map(n, -1);
  std::vector<int> cand_col;
  std::vector<double> cand_w;
  // Merges outgoing (row i) and incoming (column i) neighbours in column order;
  // returns the strongest weight.
  auto neighbours = [&](int i) {
    cand_col.clear();
    cand_w.clear();
    int out = a.row_ptr[i], incoming = offsets[i];
    const int out_end = a.row_ptr[i + 1], in_end = offsets[i + 1];
    double strongest = 0;
    while (out < out_end || incoming < in_end) {
      const int oc = out < out_end ? a.col[out] : n;
      const int ic = incoming < in_end ? sources[incoming] : n;
      const int column = std::min(oc, ic);
      double weight = 0;
      if (oc == column) weight = std::fabs(a.val[out++]);
      if (ic == column) {
        weight = std::max(weight, std::fabs(a.val[find_entry(a, column, i)]));
        ++incoming;
      }
      if (column != i && weight != 0) {
        cand_col.push_back(column);
        cand_w.push_back(weight);
        strongest = std::max(strongest, weight);
      }
    }
    return strongest;
  };
  int next = 0;
  for (int i = 0; i < n; ++i) {
    if (map[i] != -1) continue;
    const double strongest = neighbours(i);
    if (exclude_isolated && strongest == 0) continue;
    int partner = -1;
    double weight = 0;
    for (std::size_t k = 0; k < cand_col.size(); ++k) {
      const double w = cand_w[k];
      if (map[cand_col[k]] == -1 && w > weight && w >= threshold * strongest) {
        partner = cand_col[k];
        weight = w;
      }
    }
    map[i] = next;
    if (partner != -1) map[partner] = next;
    ++next;
  }
  if (!absorb_singletons) return map;
  // A row left alone joins the pair of its strongest strongly connected
  // neighbour that belongs to a pair; rows in row order, aggregates then
  // renumbered in their old order. Strongly connected: the pairing criterion
  // (weight >= threshold * the row's strongest weight) and a coupling of at
  // least kAbsorbCoupling relative to the two diagonals, |a_ij| >=
  // 0.01 sqrt(|a_ii a_jj|). The second keeps nearly decoupled cells (a
  // diagonal orders of magnitude below its neighbours', as in real pressure
  // matrices) as coarse rows of their own, where the coarse solve resolves the
  // near-null modes they carry instead of averaging them into a neighbour.
  constexpr double kAbsorbCoupling = 0.01;
  std::vector<int> size(static_cast<std::size_t>(next), 0);
  for (int g : map)
    if (g >= 0) ++size[g];
  for (int i = 0; i < n; ++i) {
    if (map[i] < 0 || size[map[i]] != 1) continue;
    const double strongest = neighbours(i);
    const double di = std::fabs(a.val[a.diag[i]]);
    int best = -1;
    double weight = 0;
    for (std::size_t k = 0; k < cand_col.size(); ++k) {
      const int g = map[cand_col[k]];
      const double dj = std::fabs(a.val[a.diag[cand_col[k]]]);
      if (g >= 0 && g != map[i] && size[g] >= 2 && cand_w[k] > weight &&
          cand_w[k] >= threshold * strongest && cand_w[k] >= kAbsorbCoupling * std::sqrt(di * dj)) {
        best = g;
        weight = cand_w[k];
      }
    }
    if (best < 0) continue;
    size[map[i]] = 0;
    map[i] = best;
    ++size[best];
  }
  std::vector<int> renumber(static_cast<std::size_t>(next), -1);
  int kept = 0;
  for (int g = 0; g < next; ++g)
    if (size[g] > 0) renumber[g] = kept++;
  for (auto& g : map)
    if (g >= 0) g = renumber[g];
  return map;
}

namespace {
// The first failing index of a check over [0, n) and its message; n if none.
struct Failure {
  long long at;
  const char* message;
};

// Scans [0, n) in contiguous chunks on the host's threads; check(begin, end)
// returns its chunk's first failure. The earliest failure over all chunks is
// raised, so a parallel scan reports what a serial one would.
template <class Check>
void first_failure(long long n, Check check) {
  const long long grain = 1 << 16;
  const long long chunks_wanted = (n + grain - 1) / grain;
  const unsigned hardware = std::max(1u, std::thread::hardware_concurrency());
  const long long threads = std::max(1LL, std::min<long long>(hardware, chunks_wanted));
  std::vector<Failure> found(static_cast<std::size_t>(threads), Failure{n, nullptr});
  if (threads == 1) {
    found[0] = check(0, n);
  } else {
    std::vector<std::thread> pool;
    const long long per = (n + threads - 1) / threads;
    for (long long t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        const long long begin = std::min(n, t * per), end = std::min(n, begin + per);
        found[static_cast<std::size_t>(t)] = check(begin, end);
      });
    for (auto& th : pool) th.join();
  }
  for (const auto& f : found)  // chunks in order: the first one that failed
    if (f.message != nullptr) throw Error(f.message);
}
}  // namespace

void validate_host(const CsrView& a) {
  KB2_REQUIRE(a.n >= 0, "CSR: negative row count");
  KB2_REQUIRE(a.nnz >= 0, "CSR: exceeds 32-bit entry limit");
  KB2_REQUIRE(a.row_ptr != nullptr && (a.n == 0 || a.diag != nullptr) &&
                  (a.nnz == 0 || (a.col != nullptr && a.val != nullptr)),
              "CSR: invalid array sizes");
  KB2_REQUIRE(a.row_ptr[0] == 0 && a.row_ptr[a.n] == a.nnz, "CSR: invalid row offsets");
  // Row ranges first (every row's range is then safe to read), then each
  // row's columns and diagonal, then the values: the serial checks' order.
  first_failure(a.n, [&](long long begin, long long end) {
    for (long long r = begin; r < end; ++r) {
      const int i = static_cast<int>(r);
      if (!(a.row_ptr[i] >= 0 && a.row_ptr[i] <= a.row_ptr[i + 1] && a.row_ptr[i + 1] <= a.nnz))
        return Failure{r, "CSR: invalid row range"};
    }
    return Failure{end, nullptr};
  });
  first_failure(a.n, [&](long long begin, long long end) {
    for (long long r = begin; r < end; ++r) {
      const int i = static_cast<int>(r);
      int previous = -1;
      for (int j = a.row_ptr[i]; j < a.row_ptr[i + 1]; ++j) {
        if (!(a.col[j] > previous && a.col[j] < a.n))
          return Failure{r, "CSR: columns must be in range, unique and sorted"};
        previous = a.col[j];
      }
      if (!(a.diag[i] >= a.row_ptr[i] && a.diag[i] < a.row_ptr[i + 1] && a.col[a.diag[i]] == i))
        return Failure{r, "CSR: missing or incorrect diagonal"};
    }
    return Failure{end, nullptr};
  });
  first_failure(a.nnz, [&](long long begin, long long end) {
    for (long long j = begin; j < end; ++j)
      if (!(std::isfinite(a.val[j]) && std::fabs(a.val[j]) <= std::numeric_limits<float>::max()))
        return Failure{j, "CSR: nonfinite or out-of-range value"};
    return Failure{end, nullptr};
  });
}

std::vector<float> diagonal_values(const CsrView& a, bool l1, bool nullspace) {
  std::vector<float> inverse(a.n);
  for (int i = 0; i < a.n; ++i) {
    const float d = static_cast<float>(a.val[a.diag[i]]);
    KB2_REQUIRE(!l1 || d >= 0, "AMG: requires positive diagonals");
    KB2_REQUIRE(d != 0 || (nullspace && a.n == 1), "solver: invalid values or zero diagonal");
    float off = 0;
    if (l1)
      for (int j = a.row_ptr[i]; j < a.row_ptr[i + 1]; ++j)
        if (j != a.diag[i]) off += std::fabs(static_cast<float>(a.val[j]));
    const float scale = l1 ? std::max(std::fabs(d), 0.5f * (std::fabs(d) + off)) : d;
    inverse[i] = scale != 0 ? 1.0f / scale : 0;
    KB2_REQUIRE(std::isfinite(scale) && std::isfinite(inverse[i]),
                "solver: invalid values or diagonal inverse");
  }
  return inverse;
}

void check_amg(Kind kind, const CsrView& a, const Options& o) {
  KB2_REQUIRE(kind == Kind::AmgPcg || kind == Kind::AmgBicgstab, "AMG: expected an AMG solver kind");
  KB2_REQUIRE((o.cycle == Cycle::V || o.cycle == Cycle::K) && o.pre_sweeps > 0 &&
                  o.post_sweeps > 0 && o.coarse_sweeps > 0 && o.coarse_rows >= 1 &&
                  o.max_levels >= 1 && o.aggregation_passes >= 1 && o.aggregation_passes <= 8 &&
                  std::isfinite(o.strength_threshold) && o.strength_threshold >= 0 &&
                  o.strength_threshold <= 1,
              "AMG: invalid options");
  KB2_REQUIRE(kind != Kind::AmgPcg || o.pre_sweeps == o.post_sweeps,
              "AMG-PCG requires equal pre/post sweeps");
  validate_host(a);
  if (o.m_matrix) {
    first_failure(a.n, [&](long long begin, long long end) {
      for (long long r = begin; r < end; ++r) {
        const int i = static_cast<int>(r);
        long double sum = 0;
        for (int j = a.row_ptr[i]; j < a.row_ptr[i + 1]; ++j) {
          const float value = static_cast<float>(a.val[j]);
          sum += value;
          const int column = a.col[j];
          const int* first = a.col + a.row_ptr[column];
          const int* last = a.col + a.row_ptr[column + 1];
          const int* opposite = std::lower_bound(first, last, i);
          if (!(opposite != last && *opposite == i &&
                value == static_cast<float>(a.val[opposite - a.col]) &&
                (column == i || value <= 0)))
            return Failure{r, "AMG M-matrix: expected symmetric nonpositive edges"};
        }
        if (!(sum >= 0)) return Failure{r, "AMG M-matrix: expected diagonally dominant rows"};
      }
      return Failure{end, nullptr};
    });
  }
}

Hierarchy build_hierarchy(const CsrView& a, const Options& o) {
  Hierarchy h;
  h.levels.emplace_back();
  h.levels.back().l1 = diagonal_values(a, true, o.nullspace);
  CsrView fine = a;
  std::size_t total_nnz = static_cast<std::size_t>(a.nnz);
  while (fine.n > o.coarse_rows && h.levels.size() < static_cast<std::size_t>(o.max_levels)) {
    auto c = aggregate(fine, o);
    // Unconnected or diagonal graphs cannot coarsen; smoothing remains valid.
    const auto active = c.t.members.size();
    if (active == 0 || static_cast<double>(c.matrix.n) >= 0.85 * static_cast<double>(active)) break;
    h.levels.back().transfer = std::move(c.t);
    total_nnz += static_cast<std::size_t>(c.matrix.nnz());
    h.levels.emplace_back();
    auto& coarse = h.levels.back();
    coarse.matrix = std::move(c.matrix);
    coarse.l1 = diagonal_values(CsrView::of(coarse.matrix), true, o.nullspace);
    fine = CsrView::of(coarse.matrix);
  }
  h.complexity = a.nnz ? static_cast<double>(total_nnz) / a.nnz : 0;
  return h;
}

}  // namespace kb2
