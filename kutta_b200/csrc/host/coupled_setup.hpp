// Host setup of the Coupled (4x4-block) solve: the pressure-force
// sensitivities of each cell from its geometry and least-squares fit, the
// aggregation hierarchy over the geometric pressure-Laplacian graph and the
// coarse block-CSR patterns (src/kutta/fv/coupled_solver.cpp:27-290). Pure
// C++ (no CUDA), so it runs and is tested without a GPU.
#pragma once

#include <cstddef>
#include <vector>

#include "setup.hpp"

namespace kb2 {

// Host arrays of the mesh, stencil and pressure least-squares fit; the field
// meanings follow the reference's DeviceMesh, Stencil and BoundaryLeastSquares
// (src/kutta/fv/device_mesh.hpp:36-60, src/kutta/fv/operators.hpp:16-47).
struct CoupledMeshHost {
  int n_cells = 0, n_faces = 0, n_internal = 0;
  const int* owner = nullptr;      // n_faces
  const int* neighbour = nullptr;  // n_internal
  const int* cell_face_offsets = nullptr;  // n_cells + 1
  const int* cell_faces = nullptr;         // per entry
  const float* cell_face_sign = nullptr;   // per entry
  const int* adjacent = nullptr;           // per entry
  const float *area_x = nullptr, *area_y = nullptr, *area_z = nullptr;  // n_faces
  const double* face_area = nullptr;      // 3 n_faces (x, y, z per face), double
  const double* cell_centroid = nullptr;  // 3 n_cells, double
  const float *owner_to_face_x = nullptr, *owner_to_face_y = nullptr, *owner_to_face_z = nullptr;
  const float *neighbour_to_face_x = nullptr, *neighbour_to_face_y = nullptr,
              *neighbour_to_face_z = nullptr;  // n_internal
  const float *lsq_x = nullptr, *lsq_y = nullptr, *lsq_z = nullptr;  // per entry
  const float *boundary_delta_x = nullptr, *boundary_delta_y = nullptr,
              *boundary_delta_z = nullptr;  // per boundary face
  const float* lsq_inverse = nullptr;       // 6 n_cells planes: xx xy xz yy yz zz
  const float* diffusion = nullptr;         // n_faces
  const float* volume = nullptr;            // n_cells
  const int* boundary_kind = nullptr;       // per boundary face (fv_flow.kern.h:3-4)
  const int* pattern_row_ptr = nullptr;     // the stencil's sorted cell adjacency with
  const int* pattern_col = nullptr;         // its diagonal (the momentum rows' pattern)
  const int* pattern_diag = nullptr;
  const int* low_order = nullptr;           // n_cells flags, or null (none)
  int entries() const { return cell_face_offsets ? cell_face_offsets[n_cells] : 0; }
  int pattern_nnz() const { return pattern_row_ptr ? pattern_row_ptr[n_cells] : 0; }
};

struct CoupledOptions {  // CoupledOptions, src/kutta/fv/coupled_solver.hpp:26-38
  int pre_sweeps = 1, post_sweeps = 2, coarsest_sweeps = 8;
  float smoother_damping = 0.7f;
  double courant = 200;
  int coarsest_rows = 48;
  int aggregation_passes = 3;
  // The reference's memory-limited operator (CoupledEdgeStorage::Recompute)
  // gives the same results as the cached one; the edge cache always fits here.
  int recompute = 0;
};

// Symmetric weighted graph without self loops.
struct CoupledGraph {
  std::vector<int> row_ptr{0}, col;
  std::vector<double> weight;
  int rows() const { return static_cast<int>(row_ptr.size()) - 1; }
};

struct CoupledSetup {
  int n = 0;
  // 27 planes of n floats: the pressure-force sensitivities in slots 4-6 (G)
  // and 10-18 (Q, row major), every other slot zero.
  std::vector<float> cell;
  struct Level {
    int n = 0, nnz = 0;
    std::vector<int> rows, cols, diag;
  };
  struct Transfer {
    std::vector<int> aggregate, offsets, members;
  };
  std::vector<Level> levels;        // coarse levels 1..L
  std::vector<Transfer> transfers;  // transfers[k]: level k -> k + 1
  int width = 0;                    // most internal faces of one cell
};

// Greedy strongest-unassigned pairing with index tie-breaking: a row pairs
// only through an edge of at least threshold x its strongest edge.
std::vector<int> coupled_pair_rows(const CoupledGraph& g, double threshold, int& count);
// Member lists of each aggregate, in row order.
void coupled_members(const std::vector<int>& map, int count, std::vector<int>& offsets,
                     std::vector<int>& members);
// The graph of the aggregates: weights between two aggregates summed in
// increasing (target, weight) order.
CoupledGraph coupled_contract(const CoupledGraph& g, const std::vector<int>& map, int count);
// The cell graph weighted by the geometric pressure Laplacian |S|^2 / |S.d|.
CoupledGraph coupled_graph(const CoupledMeshHost& m);

CoupledSetup coupled_setup(const CoupledMeshHost& m, const CoupledOptions& o);

}  // namespace kb2
