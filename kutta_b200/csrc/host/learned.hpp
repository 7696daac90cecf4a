// The learned preconditioner stage (no reference counterpart): a 3-layer
// message-passing network, hidden width 32, over the graph of the fine matrix,
// mapping a residual r to an approximate correction G(r) ~ A^-1 r. It is
// trained on (matrix, right-hand side, solution) triples produced by the
// solvers themselves, with the loss |G(b) - x|^2 / |x|^2, and used inside the
// mixed solve's flexible PCG as z = M_amg(r) + G(r - A M_amg(r)).
#pragma once

#include <cstdint>
#include <vector>

#include "device.hpp"

namespace kb2 {

class Gnn {
 public:
  static constexpr int kHidden = 32;
  static constexpr int kLayers = 3;
  explicit Gnn(std::uint64_t seed);
  // Parameters: per layer Ws [32][Cin], Wn [32][Cin], b [32] (Cin = 1, 32,
  // 32), then wo [32].
  static int parameter_count();
  // Binds the matrix graph (device CSR of the fine level): edge weights and
  // node scales from the values, activation buffers for n rows. The pattern
  // arrays must stay valid while bound; call again after values change.
  void bind(int n, const int* rows, const int* cols, const int* diag, const float* vals,
            cudaStream_t s);
  // z = beta z + G(r) (beta 0 or 1), kernels only.
  void forward(const float* r, float* z, float beta, cudaStream_t s);
  // One Adam step on |G(b) - x|^2 / x_norm2; returns that loss (host wait).
  float train_step(const float* b, const float* x, double x_norm2, float lr, cudaStream_t s);
  std::vector<float> weights() const;
  void set_weights(const std::vector<float>& w);
  int rows() const { return n_; }

 private:
  struct Slices {
    float *ws[kLayers], *wn[kLayers], *b[kLayers], *wo;
  };
  Slices slices(float* base) const;
  int n_ = 0;
  const int* rows_ = nullptr;
  const int* cols_ = nullptr;
  DArray<float> params_, grads_, m_, v_, loss_;
  DArray<float> edge_, scale_;
  // h[0] = input (n), h[l] = layer l output (n x 32); m[l] = aggregation of h[l].
  DArray<float> h_[kLayers + 1], m_agg_[kLayers];
  DArray<float> dz_, z_, dh_, dhs_, dm_, dagg_;
  int step_ = 0;
};

}  // namespace kb2
