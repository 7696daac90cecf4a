// Test infrastructure only: the reference's own Coupled (4x4-block) solve,
// src/kutta/fv/coupled_solver.cpp with src/kutta/kernels/fv_coupled.kern.h,
// run on the serial CPU device of a structured box mesh that the reference
// itself generates (src/kutta/io/generators.cpp, make_box_hex / make_box_tet),
// with the reference's geometry, device mesh, stencil and least-squares fit
// (src/kutta/mesh/mesh.cpp, src/kutta/fv/device_mesh.cpp,
// src/kutta/fv/operators.cpp). Built into oracle/_ref/libkutta_ref.so by
// oracle/build_ref.sh; the product never loads it.
//
//   kref_coupled_mesh   build the mesh and every array a Coupled solver reads;
//   kref_coupled_solve  construct CoupledSolver on it, capture the three
//                       momentum diagonals, solve once and record what its
//                       kernels saw and wrote (the packed cell data, the face
//                       coefficients, the edge cache, the right-hand side, each
//                       coarse level's operator and transfer, the solution);
//   kref_coupled_array  copy one named array out (size query with out = null).
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "kernels.hpp"
#include "kutta/fv/coupled_solver.hpp"
#include "kutta/fv/device_mesh.hpp"
#include "kutta/fv/operators.hpp"
#include "kutta/io/mesh_io.hpp"
#include "kutta/linalg/csr.hpp"
#include "ref_watch.hpp"

using namespace kutta;
using namespace kutta::fv;
using kref::WatchDevice;

namespace {

struct Named {
  char type;  // 'i' int32, 'f' float32, 'd' float64
  std::vector<char> bytes;
};

struct Case {
  WatchDevice dev;
  PolyMesh host;
  MeshGeometry geom;
  DeviceMesh mesh;
  Stencil stencil;
  BoundaryLeastSquares lsq;
  Buffer<Index> kinds;
  std::vector<int> kind_host;
  std::map<std::string, Named> arrays;

  template <class T>
  void put(const std::string& name, const std::vector<T>& v) {
    Named a;
    a.type = sizeof(T) == 8 ? 'd' : (std::is_integral_v<T> ? 'i' : 'f');
    a.bytes.resize(v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(a.bytes.data(), v.data(), a.bytes.size());
    arrays[name] = std::move(a);
  }
  template <class T>
  void put_buffer(const std::string& name, const Buffer<T>& b) {
    put(name, dev.download(b));
  }
  void put_vec3(const std::string& name, const DeviceVec3& v) {
    put_buffer(name + "_x", v.x);
    put_buffer(name + "_y", v.y);
    put_buffer(name + "_z", v.z);
  }
};

thread_local std::string g_error;

}  // namespace

extern "C" {

const char* kref_coupled_last_error() { return g_error.c_str(); }

// tet = 0: hex box, else the six-tet split. patch_kind[6]: boundary kind of
// the xmin, xmax, ymin, ymax, zmin, zmax patches (fv_flow.kern.h:3-4: wall 0,
// inlet 1, outlet 2, symmetry 3, outlet with normal backflow 4).
void* kref_coupled_mesh(int tet, int nx, int ny, int nz, const double* lo, const double* hi,
                        const int* patch_kind) {
  try {
    auto c = std::make_unique<Case>();
    c->host = tet ? make_box_tet(nx, ny, nz, {lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]})
                  : make_box_hex(nx, ny, nz, {lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]});
    c->geom = compute_geometry(c->host);
    c->mesh = upload_mesh(c->dev, c->host, c->geom);
    c->stencil = make_stencil(c->dev, c->host, c->geom);
    const Index nb = c->host.n_faces() - c->host.n_internal_faces();
    c->kind_host.assign(nb, 0);
    for (std::size_t p = 0; p < c->host.patches.size() && p < 6; ++p) {
      const auto& patch = c->host.patches[p];
      for (Index f = patch.start; f < patch.start + patch.size; ++f)
        c->kind_host[f - c->host.n_internal_faces()] = patch_kind[p];
    }
    c->kinds = c->dev.upload<Index>(c->kind_host);
    // The steady solver's pressure fit with standard pressure interpolation
    // (steady_solver.cpp:348-356): face values at pressure-specified faces,
    // the cell value at the normal foot elsewhere.
    std::vector<BoundaryObservation> obs(nb);
    for (Index b = 0; b < nb; ++b)
      obs[b] = (c->kind_host[b] == 2 || c->kind_host[b] == 4) ? BoundaryObservation::FaceValue
                                                            : BoundaryObservation::NormalFootValue;
    c->lsq = boundary_least_squares(c->dev, c->host, c->geom, obs, &c->stencil,
                                    std::make_shared<LeastSquaresWorkspace>());
    auto& m = c->mesh;
    c->put<int>("sizes", {m.n_cells, m.n_faces, m.n_internal_faces,
                          static_cast<int>(m.cell_faces.size()),
                          static_cast<int>(c->stencil.pattern.col.size())});
    c->put_buffer("owner", m.owner);
    c->put_buffer("neighbour", m.neighbour);
    c->put_vec3("area", m.area);
    c->put_vec3("owner_to_face", m.owner_to_face);
    c->put_vec3("neighbour_to_face", m.neighbour_to_face);
    c->put_buffer("volume", m.volume);
    c->put_buffer("cell_face_offsets", m.cell_face_offsets);
    c->put_buffer("cell_faces", m.cell_faces);
    c->put_buffer("cell_face_sign", m.cell_face_sign);
    c->put_buffer("adjacent", c->stencil.adjacent);
    c->put_buffer("diffusion", c->stencil.diffusion);
    c->put<int>("pattern_row_ptr", c->stencil.pattern.row_ptr);
    c->put<int>("pattern_col", c->stencil.pattern.col);
    c->put<int>("pattern_diag", c->stencil.pattern.diag);
    c->put_vec3("lsq", c->lsq.rows());
    c->put_vec3("boundary_delta", c->lsq.boundary_delta);
    c->put_buffer("lsq_inverse", c->lsq.inverse_values(c->dev));
    c->put<int>("boundary_kind", c->kind_host);
    std::vector<double> area(3 * c->geom.face_area.size()), centroid(3 * c->geom.cell_centroid.size());
    for (std::size_t f = 0; f < c->geom.face_area.size(); ++f) {
      area[3 * f] = c->geom.face_area[f].x;
      area[3 * f + 1] = c->geom.face_area[f].y;
      area[3 * f + 2] = c->geom.face_area[f].z;
    }
    for (std::size_t i = 0; i < c->geom.cell_centroid.size(); ++i) {
      centroid[3 * i] = c->geom.cell_centroid[i].x;
      centroid[3 * i + 1] = c->geom.cell_centroid[i].y;
      centroid[3 * i + 2] = c->geom.cell_centroid[i].z;
    }
    c->put<double>("face_area", area);
    c->put<double>("cell_centroid", centroid);
    c->put<double>("cell_volume", c->geom.cell_volume);
    return c.release();
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

struct kref_coupled_options {
  int pre_sweeps, post_sweeps, coarsest_sweeps, coarsest_rows, aggregation_passes, recompute;
  double smoother_damping, courant;
};

// One Coupled solve (steady_solver.cpp:1268-1294): capture_diagonal for the
// three momentum rows (values over the stencil pattern; physical diagonals),
// solve(residuals) and update(alpha 1, 1) into zero fields. net_outflow may be
// null. reference < 0: open domain. capture = 0 records nothing (timing).
// low_order: n flags of cells with low-order pressure faces, or null. With
// pair_hi / pair_lo (planes u | v | w | p), the float-pair update is also run
// on those fields and recorded.
// residuals[4]: initial and final residual, construction and solve seconds
// (solve: the momentum-diagonal captures excluded, Jacobian assembly included).
int kref_coupled_solve(void* handle, const kref_coupled_options* o, const float* momentum_u,
                       const float* momentum_v, const float* momentum_w, const float* physical_u,
                       const float* physical_v, const float* physical_w, const float* ru,
                       const float* rv, const float* rw, const float* mass, const float* viscosity,
                       const float* physical_diagonal, const float* face_weights,
                       const float* net_outflow, double density, double velocity_scale,
                       int reference, double rel_tol, double abs_tol, int max_iter, int capture,
                       const int* low_order, const float* pair_hi, const float* pair_lo,
                       double pair_alpha_u, double pair_alpha_p, float velocity_slack,
                       float pressure_slack, int* iterations, int* converged, double* residuals,
                       char* describe, int describe_len) {
  try {
    auto& c = *static_cast<Case*>(handle);
    auto& dev = c.dev;
    const Index n = c.mesh.n_cells, nf = c.mesh.n_faces;
    const auto& pattern = c.stencil.pattern;
    const std::size_t nnz = pattern.col.size();
    CoupledOptions opt;
    opt.pre_sweeps = o->pre_sweeps;
    opt.post_sweeps = o->post_sweeps;
    opt.coarsest_sweeps = o->coarsest_sweeps;
    opt.coarsest_rows = o->coarsest_rows;
    opt.aggregation_passes = o->aggregation_passes;
    opt.smoother_damping = static_cast<float>(o->smoother_damping);
    opt.courant = o->courant;
    opt.edge_storage = o->recompute ? CoupledEdgeStorage::Recompute : CoupledEdgeStorage::Cached;

    // Capture what the solver's kernels read and wrote; argument positions
    // follow the kernel signatures in fv_coupled.kern.h.
    std::map<int, bool> seen;
    dev.observer = [&](KernelId id, std::size_t count, std::span<const KernelArg> args) {
      const auto once = [&](int key) { return seen.emplace(key, true).second; };
      if (id == KernelId::coupled_face_coefficient && once(0))
        c.put("coefficient", dev.read<float>(args[6].buffer));
      if (id == KernelId::coupled_rhs && once(1)) c.put("rhs", dev.read<float>(args[10].buffer));
      if ((id == KernelId::coupled_fine_coefficients || id == KernelId::coupled_fine_prepare) &&
          once(2)) {
        const int cell_arg = id == KernelId::coupled_fine_coefficients ? 14 : 0;
        c.put("cell", dev.read<float>(args[cell_arg].buffer));
        if (id == KernelId::coupled_fine_coefficients)
          c.put("edge", dev.read<float>(args[15].buffer));
      }
      if (id == KernelId::coupled_coarse_smooth && once(1000 + static_cast<int>(count))) {
        const std::string l = "level" + std::to_string(count) + "_";
        const char* names[] = {"rows", "cols", "diag"};
        for (int k = 0; k < 3; ++k) c.put(l + names[k], dev.read<int>(args[k].buffer));
        const char* values[] = {"a", "c", "g", "h", "d"};
        for (int k = 0; k < 5; ++k) c.put(l + values[k], dev.read<float>(args[3 + k].buffer));
      }
      if (id == KernelId::coupled_restrict && once(2000000000 - static_cast<int>(count))) {
        const std::string l = "restrict" + std::to_string(count) + "_";
        c.put(l + "offsets", dev.read<int>(args[0].buffer));
        c.put(l + "members", dev.read<int>(args[1].buffer));
      }
      if (id == KernelId::coupled_prolong && once(-1 - static_cast<int>(count)))
        c.put("aggregate" + std::to_string(count), dev.read<int>(args[0].buffer));
      if (id == KernelId::coupled_update) c.put("x", dev.read<float>(args[0].buffer));
    };

    if (!capture) dev.observer = nullptr;
    using Clock = std::chrono::steady_clock;
    const auto t0 = Clock::now();
    std::vector<Index> low(low_order ? low_order : nullptr, low_order ? low_order + n : nullptr);
    CoupledSolver solver(dev, c.mesh, c.stencil, c.host, c.geom, c.kinds, c.lsq, reference, low,
                         opt);
    const float* momentum[] = {momentum_u, momentum_v, momentum_w};
    const float* physical[] = {physical_u, physical_v, physical_w};
    for (int k = 0; k < 3; ++k) {
      CsrMatrixHost h;
      h.pattern = pattern;
      h.val.assign(momentum[k], momentum[k] + nnz);
      auto a = upload(dev, h);
      auto p = dev.upload<float>(std::span<const float>(physical[k], n));
      solver.capture_diagonal(k, a, p);
    }
    auto d_ru = dev.upload<float>(std::span<const float>(ru, n));
    auto d_rv = dev.upload<float>(std::span<const float>(rv, n));
    auto d_rw = dev.upload<float>(std::span<const float>(rw, n));
    auto d_mass = dev.upload<float>(std::span<const float>(mass, nf));
    auto d_mu = dev.upload<float>(std::span<const float>(viscosity, nf));
    auto d_phys = dev.upload<float>(std::span<const float>(physical_diagonal, n));
    auto d_weight = dev.upload<float>(std::span<const float>(face_weights, n));
    Buffer<float> d_net;
    if (net_outflow) d_net = dev.upload<float>(std::span<const float>(net_outflow, n));
    CoupledResiduals in{d_ru, d_rv, d_rw, d_mass, d_mu, d_phys, d_weight, density, velocity_scale,
                        net_outflow ? &d_net : nullptr};
    const auto t1 = Clock::now();
    const auto st = solver.solve(in, {rel_tol, abs_tol, max_iter, 8});
    const auto t2 = Clock::now();
    DeviceVec3 velocity{dev.alloc<float>(n), dev.alloc<float>(n), dev.alloc<float>(n)};
    auto pressure = dev.alloc<float>(n);
    for (auto* b : {&velocity.x, &velocity.y, &velocity.z, &pressure}) dev.fill(*b, 0.0f);
    solver.update(velocity, pressure, 1.0, 1.0);
    c.put_buffer("updated_u", velocity.x);
    c.put_buffer("updated_p", pressure);
    if (pair_hi && pair_lo) {
      // The float-pair update (coupled_solver.cpp:524-535) from given hi/lo
      // fields (planes u | v | w | p of n each).
      const auto plane = [&](const float* base, int k) {
        return dev.upload<float>(std::span<const float>(base + static_cast<std::size_t>(k) * n, n));
      };
      DeviceVec3 vh{plane(pair_hi, 0), plane(pair_hi, 1), plane(pair_hi, 2)};
      DeviceVec3 vl{plane(pair_lo, 0), plane(pair_lo, 1), plane(pair_lo, 2)};
      auto ph = plane(pair_hi, 3), pl = plane(pair_lo, 3);
      solver.update(vh, ph, CoupledPairs{vl, pl, velocity_slack, pressure_slack}, pair_alpha_u,
                    pair_alpha_p);
      const char* hi_names[] = {"paired_u", "paired_v", "paired_w", "paired_p"};
      const char* lo_names[] = {"paired_u_lo", "paired_v_lo", "paired_w_lo", "paired_p_lo"};
      const Buffer<float>* his[] = {&vh.x, &vh.y, &vh.z, &ph};
      const Buffer<float>* los[] = {&vl.x, &vl.y, &vl.z, &pl};
      for (int k = 0; k < 4; ++k) {
        c.put_buffer(hi_names[k], *his[k]);
        c.put_buffer(lo_names[k], *los[k]);
      }
    }
    dev.observer = nullptr;
    *iterations = st.iterations;
    *converged = st.converged ? 1 : 0;
    residuals[0] = st.initial_residual;
    residuals[1] = st.final_residual;
    residuals[2] = std::chrono::duration<double>(t1 - t0).count();
    residuals[3] = std::chrono::duration<double>(t2 - t1).count();
    if (describe && describe_len > 0) std::snprintf(describe, describe_len, "%s", solver.describe().c_str());
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return -1;
  }
}

// Bytes of array `name` (copied to out unless out is null), or -1 if absent.
// type receives its element type: 'i', 'f' or 'd'.
long long kref_coupled_array(void* handle, const char* name, void* out, char* type) {
  auto& c = *static_cast<Case*>(handle);
  const auto it = c.arrays.find(name);
  if (it == c.arrays.end()) return -1;
  if (type) *type = it->second.type;
  if (out && !it->second.bytes.empty())
    std::memcpy(out, it->second.bytes.data(), it->second.bytes.size());
  return static_cast<long long>(it->second.bytes.size());
}

// Names of every array, separated by spaces (size query with out = null).
int kref_coupled_names(void* handle, char* out, int len) {
  auto& c = *static_cast<Case*>(handle);
  std::string all;
  for (const auto& [k, v] : c.arrays) all += k + " ";
  if (out && len > 0) std::snprintf(out, len, "%s", all.c_str());
  return static_cast<int>(all.size()) + 1;
}

void kref_coupled_free(void* handle) { delete static_cast<Case*>(handle); }

}  // extern "C"
