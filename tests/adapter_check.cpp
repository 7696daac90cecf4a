// Test infrastructure: runs the reference's own factories (make_amg_solver,
// make_solver on the serial CPU Device, from oracle/_ref/libkutta_ref.so) and
// the adapter's (make_b200_amg_solver, make_b200_solver in
// kutta_b200/csrc/adapter/b200_solver.cpp, over libkutta_b200.so) on the same
// inputs, and prints one line per case:
//
//   case|reference type|reference message|adapter type|adapter message
//
// with type one of Error, NonfiniteError, none. Without a GPU the adapter's
// factories stop at their first device call, so a case shows either a host
// check's rejection or every host check passing. The cases follow the checks
// of csr.cpp:11-68, solver.cpp:8-53,396-406 and amg.cpp:345-382.
#include <cmath>
#include <cstdio>
#include <functional>
#include <limits>
#include <memory>
#include <string>

#include "kutta/linalg/amg.hpp"

namespace kutta {
std::unique_ptr<LinearSolver> make_b200_solver(SolverKind kind, const CsrMatrixHost& a,
                                               const SolverOptions& o);
std::unique_ptr<LinearSolver> make_b200_amg_solver(SolverKind kind, const CsrMatrixHost& a,
                                                   const AmgOptions& o);
std::unique_ptr<LinearSolver> make_b200_mixed_solver(const CsrMatrixHost& a,
                                                     const SolverOptions& o);
// The CUDA backend's accessors the adapter calls; no case reaches them.
void* cuda_ptr(BufferHandle*) { return nullptr; }
struct CUstream_st;
CUstream_st* cuda_stream(Device&) { return nullptr; }
}  // namespace kutta

using namespace kutta;

namespace {

// 2D five-point Laplacian on nx*ny cells with a Dirichlet anchor on the
// first row of cells: a symmetric M-matrix with weakly dominant rows.
CsrMatrixHost laplacian(int nx, int ny) {
  CsrMatrixHost a;
  const int n = nx * ny;
  a.pattern.n_rows = n;
  a.pattern.diag.resize(n);
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
      const int i = y * nx + x;
      double diagonal = y == 0 ? 1.0 : 0.0;
      auto off = [&](int j) {
        a.pattern.col.push_back(j);
        a.val.push_back(-1.0);
        diagonal += 1.0;
      };
      if (y > 0) off(i - nx);
      if (x > 0) off(i - 1);
      a.pattern.diag[i] = static_cast<Index>(a.pattern.col.size());
      a.pattern.col.push_back(i);
      a.val.push_back(0.0);
      const std::size_t at = a.val.size() - 1;
      if (x + 1 < nx) off(i + 1);
      if (y + 1 < ny) off(i + nx);
      a.val[at] = diagonal;
      a.pattern.row_ptr.push_back(static_cast<Index>(a.pattern.col.size()));
    }
  return a;
}

std::string kind_of(const std::function<void()>& f, std::string& message) {
  try {
    f();
  } catch (const NonfiniteError& e) {
    message = e.what();
    return "NonfiniteError";
  } catch (const Error& e) {
    message = e.what();
    return "Error";
  } catch (const std::exception& e) {
    message = e.what();
    return "other";
  }
  message.clear();
  return "none";
}

std::string flat(std::string s) {
  for (char& c : s)
    if (c == '|' || c == '\n') c = ' ';
  return s;
}

// With `mixed`, the adapter side is the mixed-precision factory and the
// reference side the pressure solver it stands in for, make_solver(AmgPcg).
void run(const char* name, const CsrMatrixHost& a, SolverKind kind, const AmgOptions* amg,
         const SolverOptions* plain, bool mixed = false) {
  auto dev = Device::create(Backend::Cpu);
  std::string rm, bm;
  const std::string rt = kind_of(
      [&] { (void)(amg ? make_amg_solver(kind, *dev, a, *amg) : make_solver(kind, *dev, a, *plain)); },
      rm);
  const std::string bt = kind_of(
      [&] {
        (void)(mixed ? make_b200_mixed_solver(a, *plain)
                     : amg ? make_b200_amg_solver(kind, a, *amg) : make_b200_solver(kind, a, *plain));
      },
      bm);
  std::printf("%s|%s|%s|%s|%s\n", name, rt.c_str(), flat(rm).c_str(), bt.c_str(),
              flat(bm).c_str());
}

void amg_case(const char* name, const CsrMatrixHost& a, SolverKind kind, const AmgOptions& o) {
  run(name, a, kind, &o, nullptr);
}

void plain_case(const char* name, const CsrMatrixHost& a, SolverKind kind,
                const SolverOptions& o) {
  run(name, a, kind, nullptr, &o);
}

void mixed_case(const char* name, const CsrMatrixHost& a, const SolverOptions& o) {
  run(name, a, SolverKind::AmgPcg, nullptr, &o, true);
}

}  // namespace

int main() {
  const CsrMatrixHost good = laplacian(12, 9);
  const Index n = good.pattern.n_rows;
  AmgOptions m_matrix;
  m_matrix.structure = OperatorStructure::SymmetricMMatrix;

  // Valid inputs: both factories accept them (the adapter's then needs a GPU).
  amg_case("valid_m_matrix", good, SolverKind::AmgPcg, m_matrix);
  amg_case("valid_k_cycle_bicgstab", good, SolverKind::AmgBicgstab, [] {
    AmgOptions o;
    o.cycle = AmgCycle::K;
    o.pre_sweeps = 2;
    o.post_sweeps = 1;
    return o;
  }());
  plain_case("valid_jacobi", good, SolverKind::BicgstabJacobi, SolverOptions{});

  // CSR validation (csr.cpp:11-30, 55-68).
  {
    auto a = good;
    a.pattern.diag[3] = a.pattern.row_ptr[3] == a.pattern.diag[3] ? a.pattern.diag[3] + 1
                                                                    : a.pattern.row_ptr[3];
    amg_case("wrong_diagonal", a, SolverKind::AmgPcg, AmgOptions{});
  }
  {
    auto a = good;
    a.pattern.col[a.pattern.row_ptr[n - 1]] = n;
    amg_case("column_out_of_range", a, SolverKind::AmgPcg, AmgOptions{});
  }
  {
    auto a = good;
    const Index j = a.pattern.row_ptr[20];
    std::swap(a.pattern.col[j], a.pattern.col[j + 1]);
    amg_case("unsorted_columns", a, SolverKind::AmgPcg, AmgOptions{});
  }
  {
    auto a = good;
    a.pattern.row_ptr.back() -= 1;
    amg_case("row_end_mismatch", a, SolverKind::AmgPcg, AmgOptions{});
  }
  {
    auto a = good;
    a.val.pop_back();
    amg_case("value_count", a, SolverKind::AmgPcg, AmgOptions{});
  }
  {
    auto a = good;
    a.val[7] = std::numeric_limits<double>::infinity();
    amg_case("infinite_value", a, SolverKind::AmgPcg, AmgOptions{});
  }
  {
    auto a = good;
    a.val[9] = std::nan("");
    plain_case("nan_value_jacobi", a, SolverKind::PcgJacobi, SolverOptions{});
  }
  {
    auto a = good;
    a.val[5] = 1e39;  // finite in double, not representable in float
    amg_case("value_out_of_float_range", a, SolverKind::AmgBicgstab, AmgOptions{});
  }

  // Factory options (amg.cpp:345-362, solver.cpp:8-12, 396-406).
  amg_case("amg_kind_jacobi", good, SolverKind::PcgJacobi, AmgOptions{});
  {
    AmgOptions o;
    o.pre_sweeps = 2;
    o.post_sweeps = 3;
    amg_case("pcg_unequal_sweeps", good, SolverKind::AmgPcg, o);
  }
  {
    AmgOptions o;
    o.aggregation_passes = 9;
    amg_case("aggregation_passes", good, SolverKind::AmgPcg, o);
  }
  {
    AmgOptions o;
    o.strength_threshold = 1.5;
    amg_case("strength_threshold", good, SolverKind::AmgPcg, o);
  }
  {
    AmgOptions o;
    o.coarse_rows = 0;
    amg_case("coarse_rows", good, SolverKind::AmgPcg, o);
  }
  {
    AmgOptions o;
    o.cycle = static_cast<AmgCycle>(7);
    amg_case("cycle", good, SolverKind::AmgPcg, o);
  }
  {
    AmgOptions o;
    o.nullspace = static_cast<NullSpace>(5);
    amg_case("nullspace_value", good, SolverKind::AmgPcg, o);
  }
  {
    AmgOptions o;
    o.workspace = std::make_shared<KrylovWorkspace>(n + 1);
    amg_case("workspace_rows", good, SolverKind::AmgPcg, o);
  }
  {
    SolverOptions o;
    o.workspace = std::make_shared<KrylovWorkspace>(n - 1);
    plain_case("workspace_rows_plain", good, SolverKind::BicgstabJacobi, o);
  }
  {
    // Rows with nonzero sums and a constant null space: the row-sum check of
    // solver.cpp:13-30 is compiled only without NDEBUG, so both accept them.
    AmgOptions o;
    o.nullspace = NullSpace::Constant;
    amg_case("nullspace_row_sums", good, SolverKind::AmgPcg, o);
  }

  // The M-matrix checks (amg.cpp:362-378).
  {
    auto a = good;
    a.val[a.pattern.diag[10]] *= 0.5;
    amg_case("m_not_dominant", a, SolverKind::AmgPcg, m_matrix);
  }
  {
    auto a = good;
    const Index j = a.pattern.diag[30] + 1;  // (30, 31) positive, (31, 30) left
    a.val[j] = 0.25;
    amg_case("m_positive_edge", a, SolverKind::AmgPcg, m_matrix);
  }
  {
    auto a = good;
    const Index j = a.pattern.diag[40] + 1;  // (40, 41) only
    a.val[j] *= 2.0;
    a.val[a.pattern.diag[40]] += 1.0;
    amg_case("m_not_symmetric", a, SolverKind::AmgPcg, m_matrix);
  }

  // Setup values (amg.cpp:248-256 through the first refresh; solver.cpp:37-53).
  {
    auto a = good;
    for (Index j = a.pattern.row_ptr[50]; j < a.pattern.row_ptr[51]; ++j) a.val[j] = -a.val[j];
    amg_case("negative_diagonal", a, SolverKind::AmgBicgstab, AmgOptions{});
  }
  {
    auto a = good;
    a.val[a.pattern.diag[60]] = 0.0;
    plain_case("zero_diagonal_jacobi", a, SolverKind::PcgJacobi, SolverOptions{});
  }

  // The mixed-precision factory against the pressure solver it replaces.
  {
    SolverOptions pressure;
    pressure.structure = OperatorStructure::SymmetricMMatrix;
    mixed_case("mixed_valid", good, pressure);
    auto a = good;
    a.val[a.pattern.diag[10]] *= 0.5;
    mixed_case("mixed_m_not_dominant", a, pressure);
    a = good;
    a.val[3] = std::numeric_limits<double>::infinity();
    mixed_case("mixed_infinite_value", a, pressure);
    a = good;
    a.pattern.col[a.pattern.row_ptr[n - 1]] = n;
    mixed_case("mixed_column_out_of_range", a, pressure);
    a = good;
    a.val.pop_back();
    mixed_case("mixed_value_count", a, pressure);
    SolverOptions bad = pressure;
    bad.nullspace = static_cast<NullSpace>(4);
    mixed_case("mixed_nullspace_value", good, bad);
  }
  return 0;
}
