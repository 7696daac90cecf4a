// Test infrastructure only (see oracle/ref_shim.cpp): a Device that forwards
// every call to the reference's serial CPU backend and lets the shim observe
// each kernel launch after it ran, with its arguments.
#pragma once

#include <cstring>
#include <functional>
#include <memory>
#include <span>
#include <string>
#include <vector>

#include "kernels.hpp"
#include "kutta/runtime/device.hpp"

namespace kref {
using namespace kutta;

// Forwards every Device call to the serial CPU backend while letting the shim
// observe kernel launches. Buffers are wrapped so the wrapper owns the handle
// identity the solver sees; launches translate them back.
class WatchDevice final : public Device {
  struct Wrapped final : BufferHandle {
    Buffer<float> inner;
    explicit Wrapped(Buffer<float> b) : inner(std::move(b)) {}
    std::size_t bytes() const override { return inner.size() * sizeof(float); }
  };
  static Buffer<float>& in(const BufferHandle& h) {
    return const_cast<Wrapped&>(static_cast<const Wrapped&>(h)).inner;
  }

 public:
  WatchDevice() : cpu_(Device::create(Backend::Cpu)) {}
  Backend backend() const override { return Backend::Cpu; }
  std::string name() const override { return cpu_->name(); }
  double sum(const Buffer<float>& x, std::size_t n) override { return cpu_->sum(in(*x.handle()), n); }
  double dot(const Buffer<float>& x, const Buffer<float>& y, std::size_t n) override {
    return cpu_->dot(in(*x.handle()), in(*y.handle()), n);
  }
  double max_abs(const Buffer<float>& x, std::size_t n) override {
    return cpu_->max_abs(in(*x.handle()), n);
  }
  void launch(KernelId id, std::size_t n, std::span<const KernelArg> args) override {
    std::vector<KernelArg> inner(args.begin(), args.end());
    for (auto& a : inner)
      if (a.kind == KernelArg::Kind::Buffer) a.buffer = in(*a.buffer).handle();
    cpu_->launch(id, n, inner);
    if (observer) observer(id, n, args);
  }
  void synchronize() override { cpu_->synchronize(); }
  template <class T>
  std::vector<T> read(const BufferHandle* h) {
    const auto words = cpu_->download(in(*h));
    std::vector<T> out(words.size());
    if (!words.empty()) std::memcpy(out.data(), words.data(), words.size() * sizeof(float));
    return out;
  }
  std::function<void(KernelId, std::size_t, std::span<const KernelArg>)> observer;

 protected:
  void reduce_into(const Buffer<float>& x, const Buffer<float>& y, const Buffer<float>& u,
                   const Buffer<float>& v, std::size_t n, Buffer<float>& dst,
                   std::size_t offset, Reduction mode) override {
    check_reduction(x, y, u, v, n, dst, offset, mode);
    auto& out = in(*dst.handle());
    if (mode == Reduction::Sum) cpu_->sum_into(in(*x.handle()), n, out, offset);
    else if (mode == Reduction::Dot) cpu_->dot_into(in(*x.handle()), in(*y.handle()), n, out, offset);
    else cpu_->dot2_into(in(*x.handle()), in(*y.handle()), in(*u.handle()), in(*v.handle()), n, out, offset);
  }
  void host_reductions(std::span<const HostReduction> requests, std::span<double> out) override {
    std::vector<HostReduction> inner(requests.begin(), requests.end());
    for (auto& r : inner) { r.x = &in(*r.x->handle()); r.y = &in(*r.y->handle()); }
    const auto values = cpu_->reduce_many(inner);
    std::copy(values.begin(), values.end(), out.begin());
  }
  std::unique_ptr<BufferHandle> alloc_bytes(std::size_t bytes) override {
    return std::make_unique<Wrapped>(cpu_->alloc<float>((bytes + 3) / 4));
  }
  void upload_bytes(BufferHandle& dst, const void* src, std::size_t bytes) override {
    std::vector<float> words(in(dst).size());
    if (bytes) std::memcpy(words.data(), src, bytes);
    cpu_->upload<float>(in(dst), words);
  }
  void download_bytes(const BufferHandle& src, void* dst, std::size_t bytes) override {
    const auto words = cpu_->download(in(src));
    if (bytes) std::memcpy(dst, words.data(), bytes);
  }
  void copy_bytes(BufferHandle& dst, const BufferHandle& src, std::size_t) override {
    cpu_->copy(in(dst), in(src));
  }
  void fill_bytes(BufferHandle& dst, const void* value, std::size_t size, std::size_t) override {
    float word = 0;
    std::memcpy(&word, value, size);
    cpu_->fill(in(dst), word);
  }

 private:
  std::unique_ptr<Device> cpu_;
};


}  // namespace kref
