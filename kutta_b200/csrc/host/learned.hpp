// The learned preconditioner stage (no reference counterpart): a 3-layer
// message-passing network, hidden width 32, over the graph of the fine matrix,
// mapping a residual r to a correction direction G(r) (positively homogeneous:
// the input is normalised by its RMS and the output scaled back). It is used
// inside the mixed solve's flexible PCG as z = M(r) + alpha G(t), t = r - A M(r)
// and alpha the energy-optimal step, and as a warm-start correction. Training
// takes (residual t, error e) pairs with A e = t, made by the solvers
// themselves, and minimises the fraction of the error's A-energy that the best
// step along G(t) leaves: 1 - (c.t)^2 / ((c.Ac)(t.e)), c = G(t).
#pragma once

#include <cstdint>
#include <vector>

#include "device.hpp"

namespace kb2 {

class Gnn {
 public:
  static constexpr int kHidden = 32;
  static constexpr int kLayers = 3;
  static constexpr int kGate = 2;  // the geometry gate's theta (last parameters)
  // theta_1 at creation. At theta = (0, 0) both gate gradients vanish (a
  // saddle: dE/dtheta_0 carries tanh(theta_1 rho), dE/dtheta_1 carries
  // theta_0), so theta_1 starts nonzero; the gate is exactly 1 while theta_0
  // is 0.
  static constexpr float kGateSlope = 0.25f;
  explicit Gnn(std::uint64_t seed);
  // Parameters: per layer Ws [32][Cin], Wn [32][Cin], b [32] (Cin = 1, 32,
  // 32), then wo [32], then the geometry gate's theta [2] (initially
  // (0, kGateSlope): a gate of exactly 1).
  static int parameter_count();
  // The count without the gate (weights saved before it existed; loading
  // them leaves theta at 0).
  static int base_parameter_count() { return parameter_count() - kGate; }
  // Per-entry geometric coefficients of the matrices bound from now on (a
  // device array over the bound CSR pattern: |A_f| / |c_N - c_P| per
  // off-diagonal entry, 0 on the diagonal), or null for none. With them each
  // edge weight is gated, E_ij = w_ij exp(theta_0 tanh(theta_1 rho_ij)),
  // rho_ij = log((g_ij / sqrt(G_i G_j)) / w_ij), G_i = sum_j g_ij; takes effect
  // at the next bind; the array must stay valid while bound.
  void set_geometry(const float* geometry) { geometry_ = geometry; }
  // Binds the matrix graph (device CSR of the fine level): edge weights and
  // node scales from the values, activation buffers for n rows. The pattern
  // arrays must stay valid while bound; call again after values change.
  void bind(int n, const int* rows, const int* cols, const int* diag, const float* vals,
            cudaStream_t s);
  // z = beta z + G(r) (beta 0 or 1), kernels only: the tensor-core forward
  // (BF16 operands, FP32 accumulation) of learned_tc.cu.
  void forward(const float* r, float* z, float beta, cudaStream_t s);
  // Throws TimeoutError if a tensor-core launch recorded an MMA that did not
  // complete (host wait on s).
  void check(cudaStream_t s);
  // One Adam step on the energy loss of G(t) for A e = t (the bound matrix);
  // returns that loss before the step (host wait). The backward's two 32-wide
  // layers run on the tensor cores.
  float train_step(const float* t, const float* e, float lr, cudaStream_t s);
  // The energy loss's gradient at the current weights (no step), with the
  // 32-wide layers' backward on the tensor cores or on CUDA cores in FP32;
  // *loss (if not null) receives the loss. Host wait.
  std::vector<float> gradient(const float* t, const float* e, bool tensor_cores, float* loss,
                              cudaStream_t s);
  std::vector<float> weights() const;
  void set_weights(const std::vector<float>& w);
  int rows() const { return n_; }
  // The device the stage's arrays live on (current at construction).
  int device() const { return device_; }
  // Polls of each tensor-core tile's first wait for its MMA before the CTA
  // gives up and the forward reports a timeout (< 0: the built-in bound). A
  // test sets 0 to take the timeout path with a healthy MMA.
  void set_wait_polls(long long polls) { wait_polls_ = polls; }

 private:
  // Throws unless the current device is the stage's own.
  void check_device() const;
  struct Slices {
    float *ws[kLayers], *wn[kLayers], *b[kLayers], *wo;
  };
  Slices slices(float* base) const;
  // The FP32 forward of learned.cu, keeping every layer's activations for
  // the backward pass of training.
  void forward32(const float* r, float* z, cudaStream_t s);
  // Gradient of the energy loss into grads_, the loss into loss_.
  void backward(const float* t, const float* e, bool tensor_cores, cudaStream_t s);
  DArray<float> back_partials_;  // per-CTA partial weight gradients (tensor-core backward)
  int n_ = 0;
  int device_ = 0;
  const int* rows_ = nullptr;
  const int* cols_ = nullptr;
  const float* vals_ = nullptr;
  const float* geometry_ = nullptr;   // set for the next bind
  bool gated_ = false;                // the bound graph carries the geometry gate
  int nnz_ = 0;
  DArray<float> edge_w_, lift_w_, rho_, node_g_, dedge_, gate_fa_, gate_fb_;
  // E and lift from the ungated weights and the current theta.
  void regate(cudaStream_t s);
  DArray<double> partials_;
  DArray<unsigned> ticket_;
  DArray<double> sums_;  // [0] input sum of squares; [1..3] energy-loss dots
  DArray<float> params_, grads_, m_, v_, loss_;
  DArray<float> edge_, lift_, scale_;
  DArray<float> uv_;             // (u, v) pairs of the tensor-core forward
  DArray<unsigned short> h2_;    // its BF16 hidden rows (n x 32)
  DArray<int> fault_;
  // h[0] = input (n), h[l] = layer l output (n x 32); m[l] = aggregation of h[l].
  DArray<float> h_[kLayers + 1], m_agg_[kLayers];
  DArray<float> dz_, z_, q_, dh_, dhs_, dm_, dagg_;
  int step_ = 0;
  long long wait_polls_ = -1;
};

}  // namespace kb2
