// The Coupled (4x4-block) solve on the device. Control flow follows
// src/kutta/fv/coupled_solver.cpp:290-546 (smoothing, V-cycle, Galerkin
// refresh, block BiCGStab with verified restarts and the bounded fallback);
// the scalar Krylov epilogues are this library's reference-parity ones.
#include "coupled.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <sstream>
#include <utility>

namespace kb2 {

namespace {
template <class T>
std::vector<T> copy_of(const T* p, std::size_t n) {
  return std::vector<T>(p, p + n);
}
}  // namespace

CoupledSolver::CoupledSolver(const CoupledMeshHost& m, int reference,
                             const CoupledOptions& options, cudaStream_t s)
    : stream_(s), options_(options), n_(m.n_cells), reference_(reference) {
  // KUTTA_B200_COUPLED_GRAPHS=0 launches every kernel of an iteration
  // directly instead of replaying a graph (the same results), for comparisons.
  const char* graphs = std::getenv("KUTTA_B200_COUPLED_GRAPHS");
  graphs_enabled_ = !(graphs && std::string(graphs) == "0");
  KB2_REQUIRE(reference < m.n_cells, "coupled: reference cell out of range");
  CoupledSetup setup = coupled_setup(m, options);
  width_ = setup.width;
  const std::size_t n = n_, nf = m.n_faces, ni = m.n_internal, nb = nf - ni;
  const std::size_t entries = m.entries();
  own(owner_, copy_of(m.owner, nf), s);
  own(neighbour_, copy_of(m.neighbour, ni), s);
  own(offsets_, copy_of(m.cell_face_offsets, n + 1), s);
  own(faces_, copy_of(m.cell_faces, entries), s);
  own(adjacent_, copy_of(m.adjacent, entries), s);
  own(kind_, nb ? copy_of(m.boundary_kind, nb) : std::vector<int>(), s);
  own(sign_, copy_of(m.cell_face_sign, entries), s);
  own(sx_, copy_of(m.area_x, nf), s);
  own(sy_, copy_of(m.area_y, nf), s);
  own(sz_, copy_of(m.area_z, nf), s);
  own(dx_, copy_of(m.lsq_x, entries), s);
  own(dy_, copy_of(m.lsq_y, entries), s);
  own(dz_, copy_of(m.lsq_z, entries), s);
  own(diffusion_, copy_of(m.diffusion, nf), s);
  own(volume_, copy_of(m.volume, n), s);
  mesh_.n = n_;
  mesh_.n_faces = m.n_faces;
  mesh_.n_internal = m.n_internal;
  mesh_.width = width_;
  mesh_.owner = owner_.get();
  mesh_.neighbour = neighbour_.get();
  mesh_.offsets = offsets_.get();
  mesh_.faces = faces_.get();
  mesh_.sign = sign_.get();
  mesh_.adjacent = adjacent_.get();
  mesh_.kind = kind_.get();
  mesh_.sx = sx_.get();
  mesh_.sy = sy_.get();
  mesh_.sz = sz_.get();
  mesh_.dx = dx_.get();
  mesh_.dy = dy_.get();
  mesh_.dz = dz_.get();
  mesh_.diffusion = diffusion_.get();
  mesh_.volume = volume_.get();

  own(cell_, setup.cell, s);
  own(coefficient_, nf);
  own(scratch_, 3 * n);
  own(diag_, n);
  own(coupling_, n);
  own(coupling_yz_, n);
  own(inverse_, n);
  own(inverse_h_, n);
  const std::size_t slots = static_cast<std::size_t>(width_) * n;
  own(edge_, slots);
  own(edge_h_, slots);
  own(link_, slots);
  own(face_, nf);

  // A level whose longest row has at least this many entries gets a warp per
  // row in its separately launched row kernels (KUTTA_B200_COUPLED_WIDE_ROWS,
  // 0 for never; the same bits either way; the one-block tail keeps a thread
  // per row): a thread walking a hub row of ~150 entries stalls a whole sweep
  // behind it.
  const char* wide_env = std::getenv("KUTTA_B200_COUPLED_WIDE_ROWS");
  const int wide_rows = wide_env ? std::atoi(wide_env) : 32;
  for (std::size_t k = 0; k < setup.levels.size(); ++k) {
    auto& src = setup.levels[k];
    int longest = 0;
    for (int i = 0; i < src.n; ++i) longest = std::max(longest, src.rows[i + 1] - src.rows[i]);
    Level l;
    own(l.rows, src.rows, s);
    own(l.cols, src.cols, s);
    own(l.diag, src.diag, s);
    const std::size_t cn = src.n, nnz = src.nnz;
    own(l.a, nnz);
    own(l.c, nnz);
    own(l.g, 3 * nnz);
    own(l.h, 3 * nnz);
    own(l.d, 11 * cn);
    own(l.b, cn);
    own(l.store[0], cn);
    own(l.store[1], cn);
    l.x = l.store[0].get();
    l.tmp = l.store[1].get();
    l.op = CoupledLevel{src.n, src.nnz, l.rows.get(), l.cols.get(), l.diag.get(),
                        l.a.get(),  l.c.get(),   l.g.get(),    l.h.get(),    l.d.get()};
    l.op.wide = wide_rows > 0 && longest >= wide_rows ? 1 : 0;
    levels_.push_back(std::move(l));
    auto& tsrc = setup.transfers[k];
    Transfer t;
    own(t.aggregate, tsrc.aggregate, s);
    own(t.offsets, tsrc.offsets, s);
    own(t.members, tsrc.members, s);
    t.view = CoupledTransfer{t.aggregate.get(), t.offsets.get(), t.members.get()};
    transfers_.push_back(std::move(t));
  }
  // Levels from `tail_` down are small enough for the one-block V-cycle
  // (KUTTA_B200_COUPLED_TAIL=0: separate launches, the same results;
  // KUTTA_B200_COUPLED_TAIL_ROWS: the largest level it takes).
  const char* tail = std::getenv("KUTTA_B200_COUPLED_TAIL");
  const char* tail_rows = std::getenv("KUTTA_B200_COUPLED_TAIL_ROWS");
  const int max_rows = tail_rows ? std::atoi(tail_rows) : CoupledTail::kMaxRows;
  tail_ = levels_.size();
  if (!(tail && std::string(tail) == "0"))
    while (tail_ > 0 && levels_[tail_ - 1].op.n <= max_rows &&
           levels_.size() - (tail_ - 1) <= static_cast<std::size_t>(CoupledTail::kMaxLevels))
      --tail_;
  for (auto* v : {&b_, &r_, &shadow_, &p_, &q_, &sv_, &t_}) own(*v, n);
  for (auto& v : store_) own(v, n);
  x_ = store_[0].get();
  z_ = store_[1].get();
  zs_ = store_[2].get();
  tmp_ = store_[3].get();
  own(scalars_, 24);
  own(gauge_, 2);
  own(status_, 3);
  own(partials_, kReducePartials);
  own(values_, 8);
  own(ticket_, 1);
  cuda_check(cudaMemsetAsync(ticket_.get(), 0, sizeof(unsigned), s), "memset");
  cuda_check(cudaMemsetAsync(scalars_.get(), 0, 24 * sizeof(float), s), "memset");
  cuda_check(cudaMemsetAsync(status_.get(), 0, 3 * sizeof(int), s), "memset");
  cuda_check(cudaMemsetAsync(x_, 0, n * sizeof(float4), s), "memset");
  cuda_check(cudaMemsetAsync(link_.get(), 0xff, slots * sizeof(int2), s), "memset");
  cuda_check(cudaGetLastError(), "coupled setup");
}

CoupledSolver::~CoupledSolver() {
  for (auto& g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (capture_) cudaStreamDestroy(capture_);
}

std::vector<float4*> CoupledSolver::roles() const {
  std::vector<float4*> r{x_, z_, zs_, tmp_};
  for (const auto& l : levels_) {
    r.push_back(l.x);
    r.push_back(l.tmp);
  }
  return r;
}

void CoupledSolver::set_roles(const std::vector<float4*>& r) {
  x_ = r[0];
  z_ = r[1];
  zs_ = r[2];
  tmp_ = r[3];
  for (std::size_t k = 0; k < levels_.size(); ++k) {
    levels_[k].x = r[4 + 2 * k];
    levels_[k].tmp = r[5 + 2 * k];
  }
}

// The iteration's ~100 launches cost more host time than several of its
// kernels take on the device, and the solve waits on the host after every
// iteration (the status read), so the GPU idles while they are enqueued.
// Captured once per buffer-role state (the smoother's ping-pong cycles
// through three), each iteration is then one graph launch. A capture runs on
// an internal stream and executes nothing; the graph is launched on the
// solve stream.
template <class Body>
void CoupledSolver::iteration(Body body) {
  if (!graphs_enabled_) {
    body();
    return;
  }
  const auto before = roles();
  for (const auto& g : graphs_)
    if (g.before == before) {
      cuda_check(cudaGraphLaunch(g.exec, stream_), "cudaGraphLaunch");
      launch::counter += g.launches;
      set_roles(g.after);
      return;
    }
  if (capture_ == nullptr)
    cuda_check(cudaStreamCreateWithFlags(&capture_, cudaStreamNonBlocking), "cudaStreamCreate");
  const cudaStream_t solve = stream_;
  stream_ = capture_;
  const long long launches0 = launch::counter.load();
  cudaGraph_t graph = nullptr;
  cuda_check(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal), "capture");
  try {
    body();
  } catch (...) {
    cudaStreamEndCapture(capture_, &graph);
    if (graph) cudaGraphDestroy(graph);
    stream_ = solve;
    set_roles(before);
    throw;
  }
  const cudaError_t ended = cudaStreamEndCapture(capture_, &graph);
  stream_ = solve;
  cuda_check(ended, "capture");
  IterationGraph g;
  g.before = before;
  g.after = roles();
  g.launches = launch::counter.load() - launches0;
  launch::counter -= g.launches;  // counted when launched
  const cudaError_t made = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  cuda_check(made, "cudaGraphInstantiate");
  cuda_check(cudaGraphLaunch(g.exec, stream_), "cudaGraphLaunch");
  launch::counter += g.launches;
  if (graphs_.size() < 8)
    graphs_.push_back(std::move(g));
  else
    cudaGraphExecDestroy(g.exec);  // deferred by CUDA until the launch ends
}

CoupledFine CoupledSolver::fine() const {
  return CoupledFine{diag_.get(),   coupling_.get(), coupling_yz_.get(), inverse_.get(),
                     inverse_h_.get(), edge_.get(), edge_h_.get(),      link_.get(),
                     face_.get()};
}

void CoupledSolver::capture_diagonal(int component, const int* rows, const int* diag,
                                     const float* values, const float* physical, cudaStream_t s) {
  KB2_REQUIRE(component >= 0 && component < 3, "coupled: invalid momentum component");
  launch::cpl_copy_diagonal(n_, rows, diag, values, physical,
                            cell_.get() + static_cast<std::size_t>(component) * n_,
                            static_cast<float>(1 / options_.courant), s);
  cuda_check(cudaGetLastError(), "capture_diagonal");
}

// ---- multigrid -----------------------------------------------------------------

// Damped block-Jacobi sweeps, double buffered through tmp_
// (coupled_solver.cpp:307-329).
void CoupledSolver::fine_smooth(float4*& out, const float4* rhs, int sweeps, bool first) {
  for (int k = 0; k < sweeps; ++k) {
    launch::cpl_fine_smooth(n_, fine(), width_, out, rhs, tmp_, options_.smoother_damping,
                            first && k == 0, stream_);
    // The sweep's output becomes the iterate; the old iterate is scratch.
    std::swap(tmp_, out);
  }
}

void CoupledSolver::coarse_smooth(Level& l, int sweeps, bool first) {
  for (int k = 0; k < sweeps; ++k) {
    launch::cpl_coarse_smooth(l.op, l.x, l.b.get(), l.tmp, options_.smoother_damping,
                              first && k == 0, stream_);
    std::swap(l.x, l.tmp);
  }
}

// Coarse level k receives its right-hand side in levels_[k].b
// (coupled_solver.cpp:331-347).
void CoupledSolver::cycle(std::size_t k) {
  if (k == tail_) {
    CoupledTail t;
    t.levels = static_cast<int>(levels_.size() - k);
    t.pre = options_.pre_sweeps;
    t.post = options_.post_sweeps;
    t.coarsest = options_.coarsest_sweeps;
    t.omega = options_.smoother_damping;
    for (int j = 0; j < t.levels; ++j) {
      auto& l = levels_[k + j];
      t.op[j] = l.op;
      t.x[j] = l.x;
      t.tmp[j] = l.tmp;
      t.b[j] = l.b.get();
      if (j + 1 < t.levels) t.down[j] = transfers_[k + j + 1].view;
    }
    launch::cpl_tail(t, stream_);
    // The roles the separate launches would leave: each level swaps once per
    // sweep.
    for (int j = 0; j < t.levels; ++j) {
      const int sweeps = j + 1 < t.levels ? t.pre + t.post : t.coarsest;
      if (sweeps % 2) std::swap(levels_[k + j].x, levels_[k + j].tmp);
    }
    return;
  }
  auto& l = levels_[k];
  if (k + 1 == levels_.size()) {
    coarse_smooth(l, options_.coarsest_sweeps, true);
    return;
  }
  auto& c = levels_[k + 1];
  coarse_smooth(l, options_.pre_sweeps, true);
  launch::cpl_coarse_residual(l.op, l.x, l.b.get(), l.tmp, stream_);
  const auto& t = transfers_[k + 1].view;
  launch::cpl_restrict(c.op.n, t.offsets, t.members, l.tmp, c.b.get(), stream_);
  cycle(k + 1);
  launch::cpl_prolong(l.op.n, t.aggregate, c.x, l.x, stream_);
  coarse_smooth(l, options_.post_sweeps, false);
}

// out = V-cycle(rhs), a fixed linear preconditioner (coupled_solver.cpp:349-360).
void CoupledSolver::precondition(const float4* rhs, float4*& out) {
  fine_smooth(out, rhs, options_.pre_sweeps, true);
  if (!levels_.empty()) {
    auto& c = levels_[0];
    const auto& t = transfers_[0].view;
    launch::cpl_fine_residual(n_, fine(), width_, out, rhs, tmp_, stream_);
    launch::cpl_restrict(c.op.n, t.offsets, t.members, tmp_, c.b.get(), stream_);
    cycle(0);
    launch::cpl_prolong(n_, t.aggregate, c.x, out, stream_);
  }
  fine_smooth(out, rhs, options_.post_sweeps, false);
}

// Galerkin operators from the fine level down, then each level's smoother
// bound and block inverse (coupled_solver.cpp:361-384).
void CoupledSolver::galerkin(const CoupledSolveInputs& in) {
  if (levels_.empty()) return;
  launch::cpl_galerkin_fine(levels_[0].op, transfers_[0].view, mesh_, in, coefficient_.get(),
                            cell_.get(), wc_, stream_);
  for (std::size_t k = 1; k < levels_.size(); ++k)
    launch::cpl_galerkin_coarse(levels_[k].op, transfers_[k].view, levels_[k - 1].op, stream_);
  for (auto& l : levels_)
    launch::cpl_coarse_prepare(l.op, reinterpret_cast<float*>(l.tmp), stream_);
}

double CoupledSolver::norm(const float4* v) {
  const float* f = reinterpret_cast<const float*>(v);
  launch::reduce_value(ReduceMode::Dot, 4 * n_, f, f, DeviceReducer{partials_.get(), ticket_.get()},
                       values_.get(), 0, stream_);
  cuda_check(cudaMemcpyAsync(host_value_.get(), values_.get(), sizeof(double),
                             cudaMemcpyDeviceToHost, stream_),
             "norm readback");
  wait(stream_);
  cuda_check(cudaGetLastError(), "coupled norm");
  return std::sqrt(host_value_[0]);
}

// ---- the block BiCGStab (coupled_solver.cpp:389-451) -----------------------------

Stats CoupledSolver::bicgstab(const Control& c) {
  const int n4 = 4 * n_;
  const auto F = [](const DArray<float4>& a) { return reinterpret_cast<float*>(a.get()); };
  const DeviceReducer red{partials_.get(), ticket_.get()};
  float* sc = scalars_.get();
  int* st = status_.get();
  Stats stats;
  cuda_check(cudaMemsetAsync(x_, 0, static_cast<std::size_t>(n_) * sizeof(float4), stream_),
             "memset");
  cuda_check(cudaMemcpyAsync(r_.get(), b_.get(), static_cast<std::size_t>(n_) * sizeof(float4),
                             cudaMemcpyDeviceToDevice, stream_),
             "copy");
  stats.initial_residual = stats.final_residual = norm(r_.get());
  if (!std::isfinite(stats.initial_residual)) throw NonfiniteError("coupled: nonfinite residual");
  const double target = std::max(c.abs_tol, c.rel_tol * stats.initial_residual);
  if (stats.initial_residual <= target) {
    stats.converged = true;
    return stats;
  }
  const auto pair = [](double value, float& hi, float& lo) {
    hi = static_cast<float>(value);
    lo = std::isfinite(hi) ? static_cast<float>(value - static_cast<double>(hi)) : 0.0f;
  };
  float th, tl, dh, dl;
  pair(target * target, th, tl);
  pair(1e6 * stats.initial_residual * stats.initial_residual, dh, dl);
  launch::solver_limits(sc, th, tl, dh, dl, stream_);
  const auto restart = [&] {
    launch::solver_reset(sc, st, stats.iterations, stream_);
    cuda_check(cudaMemcpyAsync(shadow_.get(), r_.get(), static_cast<std::size_t>(n_) * sizeof(float4),
                               cudaMemcpyDeviceToDevice, stream_),
               "copy");
    launch::fill(n4, F(p_), 0.0f, stream_);
    launch::fill(n4, F(q_), 0.0f, stream_);
  };
  restart();
  int restarts = 0;
  Pinned<int>& state = host_status_;
  while (stats.iterations < c.max_iter) {
    iteration([&] {
      launch::reduce_into(ReduceMode::Dot, n4, F(shadow_), F(r_), F(shadow_), F(r_), red, sc, 0, st,
                          true, Epilogue::BicgBeta, stream_);
      launch::bicg_direction(n4, F(r_), F(q_), F(p_), sc, st, stream_);
      precondition(p_.get(), z_);
      launch::cpl_fine_spmv(n_, fine(), width_, z_, q_.get(), stream_);
      launch::reduce_into(ReduceMode::Dot, n4, F(shadow_), F(q_), F(shadow_), F(q_), red, sc, 2, st,
                          true, Epilogue::BicgAlpha, stream_);
      launch::bicg_difference(n4, F(r_), F(q_), F(sv_), sc, st, stream_);
      launch::reduce_into(ReduceMode::Dot, n4, F(sv_), F(sv_), F(sv_), F(sv_), red, sc, 16, st, true,
                          Epilogue::BicgS, stream_);
      precondition(sv_.get(), zs_);
      launch::cpl_fine_spmv(n_, fine(), width_, zs_, t_.get(), stream_);
      launch::reduce_into(ReduceMode::Dot2, n4, F(t_), F(t_), F(t_), F(sv_), red, sc, 2, st, true,
                          Epilogue::BicgOmega, stream_);
      launch::bicg_step(n4, reinterpret_cast<float*>(x_), F(r_), reinterpret_cast<float*>(z_),
                        reinterpret_cast<float*>(zs_), F(sv_), F(t_), sc, st, stream_);
      launch::reduce_into(ReduceMode::Dot, n4, F(r_), F(r_), F(r_), F(r_), red, sc, 18, st, true,
                          Epilogue::CheckBicg, stream_);
    });
    cuda_check(cudaMemcpyAsync(state.get(), st, 3 * sizeof(int), cudaMemcpyDeviceToHost, stream_),
               "status readback");
    wait(stream_);
    cuda_check(cudaGetLastError(), "coupled iteration");
    stats.iterations = state[1];
    if (state[0] == 0) continue;
    // A candidate: verify it against the true residual b - J x.
    launch::cpl_fine_residual(n_, fine(), width_, x_, b_.get(), r_.get(), stream_);
    stats.final_residual = norm(r_.get());
    stats.converged = std::isfinite(stats.final_residual) && stats.final_residual <= target;
    if (stats.converged || state[0] == 2 || !std::isfinite(stats.final_residual) ||
        stats.final_residual > 1e3 * stats.initial_residual || ++restarts > 4)
      return bounded(stats, target);
    restart();
  }
  launch::cpl_fine_residual(n_, fine(), width_, x_, b_.get(), r_.get(), stream_);
  stats.final_residual = norm(r_.get());
  stats.converged = stats.final_residual <= target;
  return bounded(stats, target);
}

// A Krylov breakdown must not reach the flow field: an iterate that grew the
// residual is replaced by one multigrid cycle (coupled_solver.cpp:453-462).
Stats CoupledSolver::bounded(Stats stats, double target) {
  if (std::isfinite(stats.final_residual) && stats.final_residual <= stats.initial_residual)
    return stats;
  precondition(b_.get(), x_);
  launch::cpl_fine_residual(n_, fine(), width_, x_, b_.get(), r_.get(), stream_);
  stats.final_residual = norm(r_.get());
  if (!std::isfinite(stats.final_residual)) throw NonfiniteError("coupled: nonfinite update");
  stats.converged = stats.final_residual <= target;
  return stats;
}

Stats CoupledSolver::solve(const CoupledSolveInputs& in, double density, double velocity_scale,
                           const Control& control, cudaStream_t s) {
  KB2_REQUIRE(density > 0 && velocity_scale > 0 && std::isfinite(velocity_scale),
              "coupled: invalid scales");
  KB2_REQUIRE(control.max_iter >= 0 && control.rel_tol >= 0 && control.abs_tol >= 0,
              "coupled: invalid control");
  KB2_REQUIRE(in.ru && in.rv && in.rw && in.mass && in.viscosity && in.physical_diagonal &&
                  in.face_weights,
              "coupled: missing solve input");
  stream_ = s;
  inputs_ = in;
  // Continuity rows in momentum units: volume flux times rho U.
  const double wc = density * velocity_scale;
  wc_ = static_cast<float>(wc);
  launch::cpl_assemble(mesh_, in, cell_.get(), coefficient_.get(), b_.get(),
                       scratch_.get(), fine(), wc_, static_cast<float>(wc * wc),
                       static_cast<float>(wc / density), reference_, s);
  galerkin(in);
  cuda_check(cudaGetLastError(), "coupled assembly");
  return bicgstab(control);
}

void CoupledSolver::update(float* u, float* v, float* w, float* p, double alpha_u, double alpha_p,
                           cudaStream_t s) {
  launch::cpl_update(n_, x_, u, v, w, p, static_cast<float>(alpha_u),
                     static_cast<float>(alpha_p * static_cast<double>(wc_)), s);
  if (reference_ >= 0) launch::cpl_gauge(n_, p, nullptr, 0.0f, gauge_.get(), reference_, s);
  cuda_check(cudaGetLastError(), "coupled update");
}

void CoupledSolver::paired_update(float* u, float* v, float* w, float* p, float* u_lo,
                                  float* v_lo, float* w_lo, float* p_lo, double alpha_u,
                                  double alpha_p, float velocity_slack, float pressure_slack,
                                  cudaStream_t s) {
  launch::cpl_paired_update(n_, x_, u, v, w, p, u_lo, v_lo, w_lo, p_lo,
                            static_cast<float>(alpha_u),
                            static_cast<float>(alpha_p * static_cast<double>(wc_)),
                            velocity_slack, pressure_slack, s);
  if (reference_ >= 0) launch::cpl_gauge(n_, p, p_lo, pressure_slack, gauge_.get(), reference_, s);
  cuda_check(cudaGetLastError(), "coupled update");
}

void CoupledSolver::apply(const float* x, float* y, cudaStream_t s) {
  launch::cpl_fine_spmv(n_, fine(), width_, reinterpret_cast<const float4*>(x),
                        reinterpret_cast<float4*>(y), s);
}
void CoupledSolver::residual(const float* x, const float* b, float* r, cudaStream_t s) {
  launch::cpl_fine_residual(n_, fine(), width_, reinterpret_cast<const float4*>(x),
                            reinterpret_cast<const float4*>(b), reinterpret_cast<float4*>(r), s);
}
void CoupledSolver::smooth(const float* x, const float* b, float* next, bool first,
                           cudaStream_t s) {
  launch::cpl_fine_smooth(n_, fine(), width_, reinterpret_cast<const float4*>(x),
                          reinterpret_cast<const float4*>(b), reinterpret_cast<float4*>(next),
                          options_.smoother_damping, first, s);
}

void CoupledSolver::level_apply(int k, int op, const float* x, const float* b, float* y,
                                cudaStream_t s) {
  KB2_REQUIRE(k >= 1 && k < levels(), "coupled: level out of range");
  const auto& l = levels_[k - 1].op;
  const auto* x4 = reinterpret_cast<const float4*>(x);
  const auto* b4 = reinterpret_cast<const float4*>(b);
  auto* y4 = reinterpret_cast<float4*>(y);
  const auto& t = transfers_[k - 1].view;
  switch (op) {
    case 1: launch::cpl_coarse_residual(l, x4, b4, y4, s); break;
    case 2:
    case 3:
      launch::cpl_coarse_smooth(l, x4, b4, y4, options_.smoother_damping, op == 3, s);
      break;
    case 4: launch::cpl_restrict(l.n, t.offsets, t.members, x4, y4, s); break;
    case 5: launch::cpl_prolong(level_rows(k - 1), t.aggregate, x4, y4, s); break;
    default: KB2_REQUIRE(false, "coupled: unknown level operator");
  }
}

void CoupledSolver::copy_inverse(float* inverse, float* inverse_h, cudaStream_t s) const {
  const std::size_t bytes = static_cast<std::size_t>(n_) * sizeof(float4);
  cuda_check(cudaMemcpyAsync(inverse, inverse_.get(), bytes, cudaMemcpyDeviceToHost, s), "copy");
  cuda_check(cudaMemcpyAsync(inverse_h, inverse_h_.get(), bytes, cudaMemcpyDeviceToHost, s),
             "copy");
}

std::string CoupledSolver::describe() const {
  std::ostringstream out;
  out << "coupled block BiCGStab, aggregation AMG V-cycle, " << levels_.size() + 1 << " levels (";
  out << n_;
  for (const auto& l : levels_) out << '/' << l.op.n;
  out << " rows), block Jacobi smoother";
  return out.str();
}

}  // namespace kb2
