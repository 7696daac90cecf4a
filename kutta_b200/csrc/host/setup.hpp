// Host-side AMG setup: CSR validation, pairwise aggregation and the coarse
// operators with their Galerkin entry maps. Pure C++ (no CUDA), so it runs and is
// tested without a GPU.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace kb2 {

// kutta::Error / kutta::NonfiniteError (src/kutta/core/types.hpp:24-33).
class Error : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};
class NonfiniteError : public Error {
 public:
  using Error::Error;
};
class DeviceError : public Error {
 public:
  using Error::Error;
};
class TimeoutError : public Error {
 public:
  using Error::Error;
};

#define KB2_REQUIRE(cond, msg) \
  do {                         \
    if (!(cond)) throw ::kb2::Error(msg); \
  } while (0)

enum class Kind : int { Jacobi = 0, PcgJacobi = 1, BicgstabJacobi = 2, AmgPcg = 3, AmgBicgstab = 4 };
enum class Cycle : int { V = 0, K = 1 };

struct Options {  // AmgOptions, src/kutta/linalg/amg.hpp:8-20
  Cycle cycle = Cycle::V;
  int pre_sweeps = 5, post_sweeps = 5, coarse_sweeps = 32;
  int coarse_rows = 24, max_levels = 24, aggregation_passes = 3;
  double strength_threshold = 0.25;
  bool nullspace = false;  // NullSpace::Constant
  bool m_matrix = false;   // OperatorStructure::SymmetricMMatrix
  // Mixed-precision hierarchy only (no reference counterpart): after each
  // pairing pass, a row left unpaired joins the pair of its strongest paired
  // neighbour, so coarsening does not stall on singletons.
  bool absorb_singletons = false;
  // Mixed-precision V-cycle: levels >= 1 stored as BF16 x row scales, and the
  // coarsest level (<= 1024 rows) solved with a dense FP64 inverse.
  bool coarse_bf16 = false;
  bool dense_coarsest = false;
  // Mixed V-cycle: the coarse levels below 16,384 rows run as one
  // thread-block-cluster launch (needs coarse_bf16, no nullspace, and no
  // K-cycle inner step on those levels).
  bool fused_tail = false;
  // K-cycle depth: coarse levels 1..k_levels take the inner Krylov step and
  // the levels below them a V-cycle; 0 means every level (the reference).
  int k_levels = 0;
  // Replay each AMG preconditioner application as a captured CUDA graph (the
  // same kernels with the same arguments, so the same results).
  bool graphs = false;
  // Mixed solve: the fine level's residual, post-sweep and SpMV read a packed
  // copy of the operator (packed rows: int16 column offsets, the diagonal
  // apart; the same results bit for bit), refreshed from the values at every
  // refresh. Used when every row has at most 8 off-diagonal entries within
  // 32,767 columns of the diagonal.
  bool packed_fine = false;
  // Build the hierarchy on the device (same aggregates, patterns and values as
  // the host setup) when the pattern is structurally symmetric.
  bool device_setup = true;
};

// CsrMatrixHost (src/kutta/linalg/csr.hpp:16-28). val holds float-representable
// doubles for the input; coarse operators store their float values.
struct HostCsr {
  int n = 0;
  std::vector<int> row_ptr{0}, col, diag;
  std::vector<double> val;
  int nnz() const { return static_cast<int>(col.size()); }
};

// Borrowed view of a caller's host CSR (avoids copying the fine matrix).
struct CsrView {
  int n = 0, nnz = 0;
  const int* row_ptr = nullptr;
  const int* col = nullptr;
  const int* diag = nullptr;
  const double* val = nullptr;
  static CsrView of(const HostCsr& a) {
    return {a.n, a.nnz(), a.row_ptr.data(), a.col.data(), a.diag.data(), a.val.data()};
  }
};

// Transfer from one level to the next (amg.cpp:176-178): aggregate[n_f] (-1 for
// rows left out), members grouped by coarse row, and the Galerkin entry map.
struct Transfer {
  std::vector<int> aggregate, member_offsets, members, entry_offsets, entries;
};

struct HostLevel {
  HostCsr matrix;            // empty for level 0 (the caller's matrix)
  std::vector<float> l1;     // inverse L1 diagonal (solver.cpp:37-53)
  Transfer transfer;         // to level + 1 (empty on the coarsest)
};

struct Hierarchy {
  std::vector<HostLevel> levels;
  double complexity = 0;
};

// csr.cpp:11-31 + :58-64 (pattern and finite float-range values).
void validate_host(const CsrView& a);
// solver.cpp:37-53.
std::vector<float> diagonal_values(const CsrView& a, bool l1, bool nullspace);
// The option and operator checks of make_amg_solver (amg.cpp:347-379).
void check_amg(Kind kind, const CsrView& a, const Options& o);
// Aggregation ctor (amg.cpp:200-226): levels until coarse_rows, max_levels or stall.
Hierarchy build_hierarchy(const CsrView& a, const Options& o);

// Exposed for tests.
std::vector<int> pairs(const CsrView& a, double threshold, bool exclude_isolated,
                       bool absorb_singletons = false);

}  // namespace kb2
