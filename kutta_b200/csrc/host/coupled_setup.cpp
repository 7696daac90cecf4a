// Host setup of the Coupled (4x4-block) solve. The algorithm steps follow
// src/kutta/fv/coupled_solver.cpp:27-290, whose aggregates, coarse patterns
// and float sensitivities the device solve must reproduce bit for bit; the
// code is this library's own.
#include "coupled_setup.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <utility>

namespace kb2 {

namespace {
struct V3 {
  double x = 0, y = 0, z = 0;
};
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 at3(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

void validate(const CoupledMeshHost& m) {
  KB2_REQUIRE(m.n_cells >= 0 && m.n_faces >= m.n_internal && m.n_internal >= 0,
              "coupled: invalid mesh sizes");
  KB2_REQUIRE(m.owner && (m.n_internal == 0 || m.neighbour) && m.cell_face_offsets &&
                  m.cell_faces && m.cell_face_sign && m.adjacent && m.area_x && m.area_y &&
                  m.area_z && m.face_area && m.cell_centroid && m.owner_to_face_x &&
                  m.owner_to_face_y && m.owner_to_face_z && m.lsq_x && m.lsq_y && m.lsq_z &&
                  m.lsq_inverse && m.diffusion && m.volume && m.pattern_row_ptr &&
                  m.pattern_col && m.pattern_diag,
              "coupled: missing mesh array");
  KB2_REQUIRE(m.n_internal == 0 || (m.neighbour_to_face_x && m.neighbour_to_face_y &&
                                    m.neighbour_to_face_z),
              "coupled: missing neighbour-to-face vectors");
  KB2_REQUIRE(m.n_faces == m.n_internal || (m.boundary_kind && m.boundary_delta_x &&
                                            m.boundary_delta_y && m.boundary_delta_z),
              "coupled: missing boundary arrays");
  KB2_REQUIRE(m.cell_face_offsets[0] == 0 && m.pattern_row_ptr[0] == 0,
              "coupled: offsets must start at zero");
  const int entries = m.entries();
  for (int c = 0; c < m.n_cells; ++c) {
    KB2_REQUIRE(m.cell_face_offsets[c + 1] >= m.cell_face_offsets[c],
                "coupled: cell-face offsets must not decrease");
    KB2_REQUIRE(m.pattern_row_ptr[c + 1] >= m.pattern_row_ptr[c],
                "coupled: pattern row pointers must not decrease");
  }
  for (int j = 0; j < entries; ++j) {
    const int f = m.cell_faces[j];
    KB2_REQUIRE(f >= 0 && f < m.n_faces, "coupled: cell face out of range");
    const int a = m.adjacent[j];
    KB2_REQUIRE(a < m.n_cells && (a >= 0 ? f < m.n_internal : -a - 1 == f - m.n_internal),
                "coupled: adjacent entry does not match its face");
  }
  for (int f = 0; f < m.n_faces; ++f) {
    KB2_REQUIRE(m.owner[f] >= 0 && m.owner[f] < m.n_cells, "coupled: owner out of range");
    if (f < m.n_internal)
      KB2_REQUIRE(m.neighbour[f] >= 0 && m.neighbour[f] < m.n_cells,
                  "coupled: neighbour out of range");
  }
  const int nnz = m.pattern_nnz();
  for (int i = 0; i < m.n_cells; ++i)
    KB2_REQUIRE(m.pattern_diag[i] >= m.pattern_row_ptr[i] &&
                    m.pattern_diag[i] < m.pattern_row_ptr[i + 1] &&
                    m.pattern_col[m.pattern_diag[i]] == i,
                "coupled: pattern diagonal index mismatch");
  for (int j = 0; j < nnz; ++j)
    KB2_REQUIRE(m.pattern_col[j] >= 0 && m.pattern_col[j] < m.n_cells,
                "coupled: pattern column out of range");
}

// Sensitivities of the residual's face pressure force to the cell's own
// pressure (coupled_solver.cpp:132-198): G per cell and Q = T M^-1, with T
// the weighted sum of S (x_f - x_c)^T over faces whose pressure is
// extrapolated (half of each internal face, the whole of an unprescribed
// boundary face). Computed in double, stored as float.
void sensitivities(const CoupledMeshHost& m, std::vector<float>& cell) {
  const int n = m.n_cells, ni = m.n_internal;
  const std::size_t N = n;
  for (int c = 0; c < n; ++c) {
    V3 g, delta;
    double t[9] = {};
    for (int j = m.cell_face_offsets[c]; j < m.cell_face_offsets[c + 1]; ++j) {
      const int f = m.cell_faces[j];
      const V3 area = scale(at3(m.face_area, f), static_cast<double>(m.cell_face_sign[j]));
      const bool internal = f < ni;
      const bool neighbour_side = internal && m.owner[f] != c;
      const int other = internal ? (m.owner[f] == c ? m.neighbour[f] : m.owner[f]) : -1;
      const bool extrapolated =
          !m.low_order || (m.low_order[c] == 0 && (other < 0 || m.low_order[other] == 0));
      V3 r;
      if (extrapolated)
        r = neighbour_side ? V3{m.neighbour_to_face_x[f], m.neighbour_to_face_y[f],
                                m.neighbour_to_face_z[f]}
                           : V3{m.owner_to_face_x[f], m.owner_to_face_y[f], m.owner_to_face_z[f]};
      const int kind = internal ? -1 : m.boundary_kind[f - ni];
      const bool prescribed = !internal && (kind == 2 || kind == 4);
      if (internal)
        delta = add(delta, V3{m.lsq_x[j], m.lsq_y[j], m.lsq_z[j]});
      else if (prescribed)
        delta = add(delta, V3{m.boundary_delta_x[f - ni], m.boundary_delta_y[f - ni],
                              m.boundary_delta_z[f - ni]});
      double weight = 0;
      if (internal) {
        g = add(g, scale(area, .5));
        weight = .5;
      } else if (!prescribed) {
        g = add(g, area);
        weight = 1;
      }
      const double s[3] = {area.x, area.y, area.z}, q[3] = {r.x, r.y, r.z};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) t[3 * a + b] += weight * s[a] * q[b];
    }
    const float* I = m.lsq_inverse;
    const double inv[9] = {I[c],         I[c + N],     I[c + 2 * N], I[c + N],    I[c + 3 * N],
                           I[c + 4 * N], I[c + 2 * N], I[c + 4 * N], I[c + 5 * N]};
    double q[9] = {};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int k = 0; k < 3; ++k) q[3 * a + b] += t[3 * a + k] * inv[3 * k + b];
    g = sub(g, V3{q[0] * delta.x + q[1] * delta.y + q[2] * delta.z,
                  q[3] * delta.x + q[4] * delta.y + q[5] * delta.z,
                  q[6] * delta.x + q[7] * delta.y + q[8] * delta.z});
    cell[4 * N + c] = static_cast<float>(g.x);
    cell[5 * N + c] = static_cast<float>(g.y);
    cell[6 * N + c] = static_cast<float>(g.z);
    for (int k = 0; k < 9; ++k) cell[(10 + k) * N + c] = static_cast<float>(q[k]);
  }
}
}  // namespace

std::vector<int> coupled_pair_rows(const CoupledGraph& g, double threshold, int& count) {
  const int n = g.rows();
  std::vector<int> map(n, -1);
  count = 0;
  for (int i = 0; i < n; ++i) {
    if (map[i] != -1) continue;
    double strongest = 0;
    for (int j = g.row_ptr[i]; j < g.row_ptr[i + 1]; ++j) strongest = std::max(strongest, g.weight[j]);
    int partner = -1;
    double best = 0;
    for (int j = g.row_ptr[i]; j < g.row_ptr[i + 1]; ++j) {
      const int c = g.col[j];
      const double w = g.weight[j];
      if (map[c] == -1 && w > best && w >= threshold * strongest) {
        partner = c;
        best = w;
      }
    }
    map[i] = count;
    if (partner != -1) map[partner] = count;
    ++count;
  }
  return map;
}

void coupled_members(const std::vector<int>& map, int count, std::vector<int>& offsets,
                     std::vector<int>& members) {
  offsets.assign(static_cast<std::size_t>(count) + 1, 0);
  for (const int a : map) ++offsets[a + 1];
  std::partial_sum(offsets.begin(), offsets.end(), offsets.begin());
  members.resize(map.size());
  std::vector<int> next(offsets.begin(), offsets.end() - 1);
  for (int i = 0; i < static_cast<int>(map.size()); ++i) members[next[map[i]]++] = i;
}

CoupledGraph coupled_contract(const CoupledGraph& g, const std::vector<int>& map, int count) {
  std::vector<int> offsets, members;
  coupled_members(map, count, offsets, members);
  CoupledGraph out;
  out.col.reserve(g.col.size());
  out.weight.reserve(g.col.size());
  std::vector<std::pair<int, double>> row;
  for (int c = 0; c < count; ++c) {
    row.clear();
    for (int k = offsets[c]; k < offsets[c + 1]; ++k) {
      const int i = members[k];
      for (int j = g.row_ptr[i]; j < g.row_ptr[i + 1]; ++j) {
        const int target = map[g.col[j]];
        if (target != c) row.emplace_back(target, g.weight[j]);
      }
    }
    // Sorted by target, then weight: equal targets are summed smallest first.
    std::sort(row.begin(), row.end());
    for (std::size_t k = 0; k < row.size();) {
      double sum = 0;
      std::size_t end = k;
      while (end < row.size() && row[end].first == row[k].first) sum += row[end++].second;
      out.col.push_back(row[k].first);
      out.weight.push_back(sum);
      k = end;
    }
    out.row_ptr.push_back(static_cast<int>(out.col.size()));
  }
  return out;
}

CoupledGraph coupled_graph(const CoupledMeshHost& m) {
  const int n = m.n_cells;
  const int nnz = m.pattern_nnz();
  std::vector<double> weight(nnz, 0.0);
  const auto entry = [&](int row, int col) {
    const int* first = m.pattern_col + m.pattern_row_ptr[row];
    const int* last = m.pattern_col + m.pattern_row_ptr[row + 1];
    const int* at = std::lower_bound(first, last, col);
    KB2_REQUIRE(at != last && *at == col, "coupled: face neighbour missing from the pattern");
    return static_cast<int>(at - m.pattern_col);
  };
  for (int f = 0; f < m.n_internal; ++f) {
    const int o = m.owner[f], k = m.neighbour[f];
    const V3 area = at3(m.face_area, f);
    const V3 d = sub(at3(m.cell_centroid, k), at3(m.cell_centroid, o));
    const double w = dot(area, area) / std::max(std::abs(dot(area, d)), 1e-300);
    weight[entry(o, k)] += w;
    weight[entry(k, o)] += w;
  }
  CoupledGraph g;
  g.col.reserve(nnz);
  g.weight.reserve(nnz);
  for (int i = 0; i < n; ++i) {
    for (int j = m.pattern_row_ptr[i]; j < m.pattern_row_ptr[i + 1]; ++j)
      if (j != m.pattern_diag[i]) {
        g.col.push_back(m.pattern_col[j]);
        g.weight.push_back(weight[j]);
      }
    g.row_ptr.push_back(static_cast<int>(g.col.size()));
  }
  return g;
}

CoupledSetup coupled_setup(const CoupledMeshHost& m, const CoupledOptions& o) {
  KB2_REQUIRE(o.pre_sweeps >= 1 && o.post_sweeps >= 0 && o.coarsest_sweeps >= 1 &&
                  o.smoother_damping > 0 && o.smoother_damping <= 1 && o.courant > 0 &&
                  o.coarsest_rows >= 1 && o.aggregation_passes >= 1 &&
                  o.aggregation_passes <= 8,
              "coupled: invalid options");
  validate(m);
  const int n = m.n_cells;
  CoupledSetup s;
  s.n = n;
  KB2_REQUIRE(static_cast<long long>(n) * 27 <= 0x7fffffffLL,
              "coupled: cell data exceeds the 32-bit index range");
  s.cell.assign(27 * static_cast<std::size_t>(n), 0.0f);
  sensitivities(m, s.cell);
  for (int c = 0; c < n; ++c) {
    int internal = 0;
    for (int j = m.cell_face_offsets[c]; j < m.cell_face_offsets[c + 1]; ++j)
      internal += m.adjacent[j] >= 0;
    s.width = std::max(s.width, internal);
  }

  // Aggregation (coupled_solver.cpp:240-289): up to `passes` pairings per
  // level over the contracted graph, until coarsest_rows or a stall.
  CoupledGraph graph = coupled_graph(m);
  int rows_now = n;
  while (rows_now > o.coarsest_rows && s.levels.size() < 24) {
    std::vector<int> map(rows_now);
    std::iota(map.begin(), map.end(), 0);
    CoupledGraph coarse = graph;
    int count = rows_now;
    for (int pass = 0; pass < o.aggregation_passes && count > o.coarsest_rows; ++pass) {
      int next_count = 0;
      const auto next = coupled_pair_rows(coarse, .25, next_count);
      coarse = coupled_contract(coarse, next, next_count);
      for (auto& v : map) v = next[v];
      count = next_count;
    }
    if (count >= .85 * rows_now) break;  // a disconnected or stalled graph
    CoupledSetup::Transfer t;
    coupled_members(map, count, t.offsets, t.members);
    t.aggregate = std::move(map);
    s.transfers.push_back(std::move(t));
    // The coarse pattern: the contracted graph with the diagonal in column order.
    CoupledSetup::Level l;
    l.n = count;
    l.rows.push_back(0);
    l.diag.resize(count);
    for (int i = 0; i < count; ++i) {
      bool placed = false;
      for (int j = coarse.row_ptr[i]; j <= coarse.row_ptr[i + 1]; ++j) {
        const bool end = j == coarse.row_ptr[i + 1];
        if (!placed && (end || coarse.col[j] > i)) {
          l.diag[i] = static_cast<int>(l.cols.size());
          l.cols.push_back(i);
          placed = true;
        }
        if (!end) l.cols.push_back(coarse.col[j]);
      }
      l.rows.push_back(static_cast<int>(l.cols.size()));
    }
    l.nnz = static_cast<int>(l.cols.size());
    s.levels.push_back(std::move(l));
    graph = std::move(coarse);
    rows_now = count;
  }
  return s;
}

}  // namespace kb2
