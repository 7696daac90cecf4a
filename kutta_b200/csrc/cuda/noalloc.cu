// Dense coarsest-level inverse for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they need this step:
// code running while a CUDA stream or graph is being recorded by someone else,
// hosts that hand the library a fixed memory budget (pre-sized pools, no growth
// after start-up), or real-time loops that must not take the allocator's locks
// or risk an out-of-memory failure mid-iteration. For them this entry point
// takes its n x n factor scratch from one array compiled into the library
// instead of allocating it. The caller still provides the inputs and outputs.
//
// Limits and sharing:
// - n <= kNoAllocRows (512): the scratch is 512 x 512 doubles = 2 MiB, reserved
//   on every GPU that loads this library, for as long as the process runs.
// - Operators of n > 236 rows are factored through the array. Every such call
//   uses the same array: the kernel clears the part it uses before filling
//   it, so leftovers from an earlier call never reach the result, but calls
//   whose work overlaps on the GPU (different streams, or different threads on
//   one device without ordering) race on the array and must be ordered by the
//   caller. Operators of n <= 236 rows are factored in shared memory and never
//   touch the array, so they need no ordering.
// - The device address of the array is looked up once per device, on that
//   device's first call (cudaGetSymbolAddress, which may load this library's
//   device code). Make that first call before any stream capture begins.
//   Later calls read the cached address without taking a lock. A device reset
//   (cudaDeviceReset) unloads the library's device code, which can move the
//   array; a process that resets a device must not call this entry point on
//   that device afterwards.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>

#include "kernels.hpp"
#include "kutta_b200.h"

namespace kb2 {
int report_error(int code, const char* message);  // capi.cpp: sets b2_last_error()

namespace {
constexpr int kNoAllocRows = 512;
constexpr int kMaxDevices = 64;

// Host code sees only a stand-in for this name; the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) double g_dense_scratch[kNoAllocRows * kNoAllocRows];

std::mutex g_lock;  // taken only by a device's first lookup
std::atomic<double*> g_scratch_address[kMaxDevices] = {};

// Device address of the scratch on the current device (looked up once).
int scratch_address(double** out) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return report_error(B2_DEVICE_ERROR, cudaGetErrorString(e));
  if (device < 0 || device >= kMaxDevices)
    return report_error(B2_DEVICE_ERROR, "dense inverse (no allocation): device ordinal out of range");
  if (double* cached = g_scratch_address[device].load(std::memory_order_acquire)) {
    *out = cached;
    return B2_OK;
  }
  std::lock_guard<std::mutex> hold(g_lock);
  if (!g_scratch_address[device].load(std::memory_order_relaxed)) {
    void* address = nullptr;
    e = cudaGetSymbolAddress(&address, g_dense_scratch);
    if (e != cudaSuccess || address == nullptr) {
      char message[256];
      std::snprintf(message, sizeof message,
                    "dense inverse (no allocation): cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
      return report_error(B2_DEVICE_ERROR, message);
    }
    g_scratch_address[device].store(static_cast<double*>(address), std::memory_order_release);
  }
  *out = g_scratch_address[device].load(std::memory_order_relaxed);
  return B2_OK;
}
}  // namespace
}  // namespace kb2

extern "C" int b2_dense_inverse_noalloc(int n, const int32_t* d_row_ptr, const int32_t* d_col,
                                        const float* d_val, double* d_inverse, double* d_not_spd,
                                        void* stream) {
  if (n < 1 || n > kb2::kNoAllocRows) {
    char message[160];
    std::snprintf(message, sizeof message,
                  "dense inverse (no allocation): n = %d is outside [1, %d], the size of its "
                  "built-in scratch", n, kb2::kNoAllocRows);
    return kb2::report_error(B2_INVALID_ARGUMENT, message);
  }
  if (!d_row_ptr || !d_col || !d_val || !d_inverse || !d_not_spd)
    return kb2::report_error(B2_INVALID_ARGUMENT, "dense inverse (no allocation): null argument");
  double* scratch = nullptr;
  const int status = kb2::scratch_address(&scratch);
  if (status != B2_OK) return status;
  kb2::launch::dense_inverse(n, d_row_ptr, d_col, d_val, scratch, d_inverse, d_not_spd,
                             static_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return kb2::report_error(B2_DEVICE_ERROR, cudaGetErrorString(e));
  return B2_OK;
}
