// Small RAII helpers over the CUDA runtime: owned device arrays, pinned host
// staging, and bounded host waits.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "setup.hpp"

namespace kb2 {

inline void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    throw DeviceError(std::string("out of device memory: ") + what);
  }
  throw DeviceError(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

template <class T>
class DArray {
 public:
  DArray() = default;
  explicit DArray(std::size_t n) { reset(n); }
  DArray(const DArray&) = delete;
  DArray& operator=(const DArray&) = delete;
  DArray(DArray&& o) noexcept : p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)) {}
  DArray& operator=(DArray&& o) noexcept {
    if (this != &o) {
      release();
      p_ = std::exchange(o.p_, nullptr);
      n_ = std::exchange(o.n_, 0);
    }
    return *this;
  }
  ~DArray() { release(); }
  void reset(std::size_t n) {
    release();
    n_ = n;
    // A handle even when empty, as the reference's buffers (one word minimum).
    cuda_check(cudaMalloc(&p_, std::max<std::size_t>(n, 1) * sizeof(T)), "cudaMalloc");
  }
  void upload(const T* host, std::size_t n, cudaStream_t s) {
    if (n) cuda_check(cudaMemcpyAsync(p_, host, n * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
  }
  void upload(const std::vector<T>& v, cudaStream_t s) {
    reset(v.size());
    upload(v.data(), v.size(), s);
  }
  T* get() const { return p_; }
  std::size_t size() const { return n_; }
  bool allocated() const { return p_ != nullptr; }

 private:
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
  T* p_ = nullptr;
  std::size_t n_ = 0;
};

// A stream-ordered device array: cudaMallocAsync on its stream, released with
// cudaFreeAsync on the same stream, so the release waits for that stream's
// queued work without synchronising the device, and the memory pool makes
// repeated allocations cheap. For scratch whose every use is on one stream.
template <class T>
class SArray {
 public:
  SArray() = default;
  SArray(std::size_t n, cudaStream_t s) { reset(n, s); }
  SArray(const SArray&) = delete;
  SArray& operator=(const SArray&) = delete;
  SArray(SArray&& o) noexcept
      : p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)), s_(o.s_) {}
  SArray& operator=(SArray&& o) noexcept {
    if (this != &o) {
      release();
      p_ = std::exchange(o.p_, nullptr);
      n_ = std::exchange(o.n_, 0);
      s_ = o.s_;
    }
    return *this;
  }
  ~SArray() { release(); }
  void reset(std::size_t n, cudaStream_t s) {
    release();
    n_ = n;
    s_ = s;
    void* p = nullptr;
    cuda_check(cudaMallocAsync(&p, std::max<std::size_t>(n, 1) * sizeof(T), s), "cudaMallocAsync");
    p_ = static_cast<T*>(p);
  }
  T* get() const { return p_; }
  std::size_t size() const { return n_; }
  bool allocated() const { return p_ != nullptr; }

 private:
  void release() {
    if (p_) cudaFreeAsync(p_, s_);
    p_ = nullptr;
    n_ = 0;
  }
  T* p_ = nullptr;
  std::size_t n_ = 0;
  cudaStream_t s_ = nullptr;
};

template <class T>
class Pinned {
 public:
  explicit Pinned(std::size_t n) : n_(n) {
    cuda_check(cudaMallocHost(&p_, std::max<std::size_t>(n, 1) * sizeof(T)), "cudaMallocHost");
  }
  Pinned(const Pinned&) = delete;
  Pinned& operator=(const Pinned&) = delete;
  ~Pinned() {
    if (p_) cudaFreeHost(p_);
  }
  T* get() const { return p_; }
  T& operator[](std::size_t i) { return p_[i]; }

 private:
  T* p_ = nullptr;
  std::size_t n_;
};

// Waits for all work queued on `s`, polling with a wall-clock limit so a device
// that stops answering turns into an error instead of a hang.
inline void wait(cudaStream_t s) {
  static const double limit = [] {
    const char* e = std::getenv("KUTTA_B200_WAIT_SECONDS");
    return e ? std::atof(e) : 300.0;
  }();
  const auto start = std::chrono::steady_clock::now();
  for (std::size_t spin = 0;; ++spin) {
    const cudaError_t e = cudaStreamQuery(s);
    if (e == cudaSuccess) return;
    if (e != cudaErrorNotReady) cuda_check(e, "stream");
    if ((spin & 1023) == 0) {
      const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
      if (t > limit) throw TimeoutError("device wait exceeded its time limit");
    }
  }
}

}  // namespace kb2
