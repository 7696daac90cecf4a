// Learned preconditioner stage: parameters, activations, forward, training.
#include "learned.hpp"

#include <cmath>

#include "../cuda/kernels.hpp"
#include "setup.hpp"

namespace kb2 {

namespace {
std::uint64_t mix(std::uint64_t& state) {
  std::uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
double uniform(std::uint64_t& state) { return static_cast<double>(mix(state) >> 11) * 0x1.0p-53; }

int cin(int layer) { return layer == 0 ? 1 : Gnn::kHidden; }
}  // namespace

int Gnn::parameter_count() {
  int count = kHidden + kGate;  // wo, theta
  for (int l = 0; l < kLayers; ++l) count += 2 * kHidden * cin(l) + kHidden;
  return count;
}

Gnn::Slices Gnn::slices(float* base) const {
  Slices s{};
  float* p = base;
  for (int l = 0; l < kLayers; ++l) {
    s.ws[l] = p;
    p += kHidden * cin(l);
    s.wn[l] = p;
    p += kHidden * cin(l);
    s.b[l] = p;
    p += kHidden;
  }
  s.wo = p;
  return s;
}

// Uniform Glorot-style initialisation (fan-in 2 Cin for the two halves of a
// layer), zero biases, small output weights.
Gnn::Gnn(std::uint64_t seed) {
  cuda_check(cudaGetDevice(&device_), "cudaGetDevice");
  const int count = parameter_count();
  std::vector<float> w(static_cast<std::size_t>(count), 0.0f);
  std::uint64_t state = seed * 0x2545F4914F6CDD1DULL + 1;
  std::size_t k = 0;
  for (int l = 0; l < kLayers; ++l) {
    const double limit = std::sqrt(6.0 / (2.0 * cin(l) + kHidden));
    for (int half = 0; half < 2; ++half)
      for (int e = 0; e < kHidden * cin(l); ++e)
        w[k++] = static_cast<float>((2.0 * uniform(state) - 1.0) * limit);
    k += kHidden;  // biases stay 0
  }
  for (int c = 0; c < kHidden; ++c) w[k++] = static_cast<float>((2.0 * uniform(state) - 1.0) * 0.1);
  w[k++] = 0.0f;               // theta_0: the gate starts at exactly 1
  w[k++] = kGateSlope;         // theta_1: nonzero, so theta_0's gradient is not 0
  params_.upload(w, nullptr);
  grads_.reset(static_cast<std::size_t>(count));
  m_.reset(static_cast<std::size_t>(count));
  v_.reset(static_cast<std::size_t>(count));
  cuda_check(cudaMemset(m_.get(), 0, sizeof(float) * count), "memset");
  cuda_check(cudaMemset(v_.get(), 0, sizeof(float) * count), "memset");
  loss_.reset(1);
  partials_.reset(kReducePartials);
  ticket_.reset(1);
  cuda_check(cudaMemset(ticket_.get(), 0, sizeof(unsigned)), "memset");
  sums_.reset(6);
  fault_.reset(1);
  cuda_check(cudaMemset(fault_.get(), 0, sizeof(int)), "memset");
}

void Gnn::check_device() const {
  int device = 0;
  cuda_check(cudaGetDevice(&device), "cudaGetDevice");
  KB2_REQUIRE(device == device_, "learned stage: called on another device than its own");
}

void Gnn::bind(int n, const int* rows, const int* cols, const int* diag, const float* vals,
               cudaStream_t s) {
  KB2_REQUIRE(n > 0 && rows && cols && diag && vals, "learned stage: invalid matrix");
  check_device();
  if (n != n_) {
    const auto rows_n = static_cast<std::size_t>(n);
    const auto wide = rows_n * kHidden;
    h_[0].reset(rows_n);
    for (int l = 1; l <= kLayers; ++l) h_[l].reset(wide);
    m_agg_[0].reset(rows_n);
    for (int l = 1; l < kLayers; ++l) m_agg_[l].reset(wide);
    dz_.reset(rows_n);
    z_.reset(rows_n);
    q_.reset(rows_n);
    dh_.reset(wide);
    dhs_.reset(wide);
    dm_.reset(wide);
    dagg_.reset(wide);
    scale_.reset(rows_n);
    uv_.reset(2 * rows_n);
    h2_.reset(wide);
  }
  int nnz = 0;
  cuda_check(cudaMemcpy(&nnz, rows + n, sizeof(int), cudaMemcpyDeviceToHost), "learned stage");
  if (edge_.size() != static_cast<std::size_t>(nnz)) {
    edge_.reset(static_cast<std::size_t>(nnz));
    lift_.reset(static_cast<std::size_t>(nnz));
  }
  n_ = n;
  nnz_ = nnz;
  rows_ = rows;
  cols_ = cols;
  vals_ = vals;
  gated_ = geometry_ != nullptr;
  if (!gated_) {
    launch::gnn_graph(n, rows, cols, diag, vals, edge_.get(), lift_.get(), scale_.get(), s);
    return;
  }
  const auto count = static_cast<std::size_t>(nnz);
  for (auto* a : {&edge_w_, &lift_w_, &rho_, &dedge_, &gate_fa_, &gate_fb_})
    if (a->size() != count) a->reset(count);
  if (node_g_.size() != static_cast<std::size_t>(n)) node_g_.reset(static_cast<std::size_t>(n));
  launch::gnn_graph(n, rows, cols, diag, vals, edge_w_.get(), lift_w_.get(), scale_.get(), s);
  launch::gnn_geometry(n, rows, cols, geometry_, edge_w_.get(), node_g_.get(), rho_.get(), s);
  regate(s);
}

void Gnn::regate(cudaStream_t s) {
  if (!gated_) return;
  launch::gnn_gate(nnz_, edge_w_.get(), lift_w_.get(), rho_.get(),
                   params_.get() + base_parameter_count(), edge_.get(), lift_.get(), s);
}

void Gnn::forward(const float* r, float* z, float beta, cudaStream_t s) {
  KB2_REQUIRE(n_ > 0, "learned stage: no matrix bound");
  check_device();
  const Slices p = slices(params_.get());
  float2* uv = reinterpret_cast<float2*>(uv_.get());
  launch::gnn_lift(n_, rows_, cols_, lift_.get(), r, scale_.get(), uv,
                   DeviceReducer{partials_.get(), ticket_.get()}, sums_.get(), s);
  launch::gnn_layer_a(n_, rows_, cols_, edge_.get(), uv, params_.get(), p.ws[1], p.wn[1], p.b[1],
                      sums_.get(), h2_.get(), fault_.get(), wait_polls_, s);
  launch::gnn_layer_b(n_, rows_, cols_, edge_.get(), h2_.get(), p.ws[2], p.wn[2], p.b[2], p.wo,
                      scale_.get(), sums_.get(), z, beta, fault_.get(), wait_polls_, s);
}

void Gnn::check(cudaStream_t s) {
  int fault = 0;
  cuda_check(cudaMemcpyAsync(&fault, fault_.get(), sizeof(int), cudaMemcpyDeviceToHost, s),
             "learned stage fault readback");
  wait(s);
  if (fault != 0) {
    cuda_check(cudaMemsetAsync(fault_.get(), 0, sizeof(int), s), "memset");
    throw TimeoutError("learned stage: a tensor-core tile did not complete");
  }
}

void Gnn::forward32(const float* r, float* z, cudaStream_t s) {
  KB2_REQUIRE(n_ > 0, "learned stage: no matrix bound");
  const Slices p = slices(params_.get());
  launch::gnn_input(n_, r, scale_.get(), h_[0].get(), s);
  launch::reduce_value(ReduceMode::Dot, n_, h_[0].get(), h_[0].get(),
                       DeviceReducer{partials_.get(), ticket_.get()}, sums_.get(), 0, s);
  launch::gnn_normalize(n_, h_[0].get(), sums_.get(), s);
  for (int l = 0; l < kLayers; ++l) {
    launch::gnn_aggregate(n_, cin(l), rows_, cols_, edge_.get(), h_[l].get(), m_agg_[l].get(), s);
    launch::gnn_dense(n_, cin(l), h_[l].get(), m_agg_[l].get(), p.ws[l], p.wn[l], p.b[l],
                      h_[l + 1].get(), s);
  }
  launch::gnn_output(n_, h_[kLayers].get(), p.wo, scale_.get(), sums_.get(), z, 0.0f, s);
}

// The energy loss's gradient at the current weights into grads_ (and the loss
// into loss_): the FP32 forward keeping every layer's activations, then the
// backward, whose two 32-wide layers run on the tensor cores when asked
// (gnn_dense_back_tc, BF16 operands, FP32 accumulation) and the 1-wide input
// layer on CUDA cores.
void Gnn::backward(const float* t, const float* e, bool tensor_cores, cudaStream_t s) {
  KB2_REQUIRE(n_ > 0, "learned stage: no matrix bound");
  KB2_REQUIRE(t != nullptr && e != nullptr, "learned stage: null training vector");
  check_device();
  const int count = parameter_count();
  const DeviceReducer red{partials_.get(), ticket_.get()};
  float* c = z_.get();
  forward32(t, c, s);
  launch::spmv(n_, rows_, cols_, vals_, c, q_.get(), nullptr, s);
  launch::reduce_value(ReduceMode::Dot, n_, c, t, red, sums_.get(), 1, s);
  launch::reduce_value(ReduceMode::Dot, n_, c, q_.get(), red, sums_.get(), 2, s);
  launch::reduce_value(ReduceMode::Dot, n_, t, e, red, sums_.get(), 3, s);
  cuda_check(cudaMemsetAsync(grads_.get(), 0, sizeof(float) * count, s), "memset");
  const Slices p = slices(params_.get());
  const Slices g = slices(grads_.get());
  launch::gnn_energy(n_, t, q_.get(), sums_.get() + 1, dz_.get(), loss_.get(), s);
  launch::gnn_output_back(n_, h_[kLayers].get(), p.wo, scale_.get(), sums_.get(), dz_.get(),
                          dh_.get(), g.wo, s);
  for (int l = kLayers - 1; l >= 0; --l) {
    if (tensor_cores && cin(l) == kHidden) {
      if (!back_partials_.allocated())
        back_partials_.reset(static_cast<std::size_t>(launch::gnn_back_partials_floats()));
      launch::gnn_dense_back_tc(n_, h_[l].get(), m_agg_[l].get(), h_[l + 1].get(), dh_.get(),
                                p.ws[l], p.wn[l], dhs_.get(), dm_.get(), g.ws[l], g.wn[l],
                                g.b[l], back_partials_.get(), fault_.get(), s);
    } else {
      launch::gnn_dense_back(n_, cin(l), h_[l].get(), m_agg_[l].get(), h_[l + 1].get(),
                             dh_.get(), p.ws[l], p.wn[l], dhs_.get(), dm_.get(), g.ws[l],
                             g.wn[l], g.b[l], s);
    }
    if (gated_)  // dL/dE from this layer's aggregation M = E h[l]
      launch::gnn_edge_grad(n_, cin(l), rows_, cols_, dm_.get(), h_[l].get(), dedge_.get(),
                            l != kLayers - 1, s);
    if (l > 0) {
      // dL/dh[l] = Ws^T G + W^T (Wn^T G); W is symmetric.
      launch::gnn_aggregate(n_, cin(l), rows_, cols_, edge_.get(), dm_.get(), dagg_.get(), s);
      launch::gnn_add(static_cast<std::size_t>(n_) * cin(l), dhs_.get(), dagg_.get(), dh_.get(), s);
    }
  }
  if (gated_) {
    // dL/dtheta = sum over edges of dL/dE dE/dtheta (FP64 dots).
    const float* theta = params_.get() + base_parameter_count();
    launch::gnn_gate_factors(nnz_, edge_.get(), rho_.get(), theta, gate_fa_.get(),
                             gate_fb_.get(), s);
    launch::reduce_value(ReduceMode::Dot, nnz_, dedge_.get(), gate_fa_.get(), red, sums_.get(), 4,
                         s);
    launch::reduce_value(ReduceMode::Dot, nnz_, dedge_.get(), gate_fb_.get(), red, sums_.get(), 5,
                         s);
    launch::gnn_store_gate_grad(sums_.get() + 4, grads_.get() + base_parameter_count(), s);
  }
}

float Gnn::train_step(const float* t, const float* e, float lr, cudaStream_t s) {
  backward(t, e, true, s);
  const int count = parameter_count();
  ++step_;
  const float beta1 = 0.9f, beta2 = 0.999f;
  launch::gnn_adam(count, params_.get(), grads_.get(), m_.get(), v_.get(), lr, beta1, beta2, 1e-8f,
                   1.0f - std::pow(beta1, static_cast<float>(step_)),
                   1.0f - std::pow(beta2, static_cast<float>(step_)), s);
  regate(s);  // the gate's theta moved
  float loss = 0;
  cuda_check(cudaMemcpyAsync(&loss, loss_.get(), sizeof(float), cudaMemcpyDeviceToHost, s),
             "loss readback");
  check(s);  // waits; a tensor-core tile that did not complete raises a timeout
  return loss;
}

std::vector<float> Gnn::gradient(const float* t, const float* e, bool tensor_cores, float* loss,
                                 cudaStream_t s) {
  backward(t, e, tensor_cores, s);
  std::vector<float> out(static_cast<std::size_t>(parameter_count()));
  cuda_check(cudaMemcpyAsync(out.data(), grads_.get(), sizeof(float) * out.size(),
                             cudaMemcpyDeviceToHost, s),
             "gradient readback");
  float value = 0;
  cuda_check(cudaMemcpyAsync(&value, loss_.get(), sizeof(float), cudaMemcpyDeviceToHost, s),
             "loss readback");
  check(s);
  if (loss) *loss = value;
  return out;
}

std::vector<float> Gnn::weights() const {
  std::vector<float> w(static_cast<std::size_t>(parameter_count()));
  cuda_check(cudaMemcpy(w.data(), params_.get(), sizeof(float) * w.size(), cudaMemcpyDeviceToHost),
             "weights");
  return w;
}

void Gnn::set_weights(const std::vector<float>& w) {
  const auto count = static_cast<std::size_t>(parameter_count());
  KB2_REQUIRE(w.size() == count || w.size() == static_cast<std::size_t>(base_parameter_count()),
              "learned stage: wrong number of weights");
  std::vector<float> all(w);
  if (all.size() < count) {  // weights without the gate: gate exactly 1, as at creation
    all.resize(count, 0.0f);
    all[count - 1] = kGateSlope;
  }
  cuda_check(cudaMemcpy(params_.get(), all.data(), sizeof(float) * count, cudaMemcpyHostToDevice),
             "weights");
  step_ = 0;
  cuda_check(cudaMemset(m_.get(), 0, sizeof(float) * count), "memset");
  cuda_check(cudaMemset(v_.get(), 0, sizeof(float) * count), "memset");
  if (n_ > 0) {
    regate(nullptr);
    cuda_check(cudaStreamSynchronize(nullptr), "regate");
  }
}

}  // namespace kb2
