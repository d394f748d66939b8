// Shared device/host utilities for the B200 fastPLS fitting library.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace fpls {

// ---------------------------------------------------------------------------
// host-side error handling
// ---------------------------------------------------------------------------
inline void check(cudaError_t status, const char* what) {
  if (status != cudaSuccess) {
    cudaGetLastError();  // clear a sticky launch error so the context stays usable
    throw std::runtime_error(std::string(what) + ": " +
                             cudaGetErrorString(status));
  }
}
#define FPLS_CHECK(expr) ::fpls::check((expr), #expr)
#define FPLS_LAUNCH(what) ::fpls::check(cudaGetLastError(), what)

inline void require(bool ok, const char* message) {
  if (!ok) throw std::invalid_argument(message);
}

// Let the device's stream-ordered pool keep freed memory (up to half the
// device) instead of returning it to the driver at every synchronisation:
// repeated fits then reuse mapped pages rather than remapping gigabytes.
void keep_pool_memory();

// Device buffer owned by the host object that allocated it (stream-ordered).
template <class T>
class DeviceArray {
 public:
  DeviceArray() = default;
  DeviceArray(std::size_t count, cudaStream_t stream) { allocate(count, stream); }
  ~DeviceArray() { release(); }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& o) noexcept { swap(o); }
  DeviceArray& operator=(DeviceArray&& o) noexcept {
    if (this != &o) {
      release();
      swap(o);
    }
    return *this;
  }
  void allocate(std::size_t count, cudaStream_t stream) {
    release();
    keep_pool_memory();
    stream_ = stream;
    count_ = count;
    if (count) FPLS_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&ptr_),
                                          count * sizeof(T), stream));
  }
  // Keep the allocation when it is already large enough.
  void reserve(std::size_t count, cudaStream_t stream) {
    if (count > count_ || stream != stream_) allocate(count, stream);
  }
  void zero(cudaStream_t stream) {
    if (count_) FPLS_CHECK(cudaMemsetAsync(ptr_, 0, count_ * sizeof(T), stream));
  }
  void release() noexcept {
    if (ptr_) cudaFreeAsync(ptr_, stream_);
    ptr_ = nullptr;
    count_ = 0;
  }
  T* get() const { return ptr_; }
  std::size_t size() const { return count_; }
  explicit operator bool() const { return ptr_ != nullptr; }

 private:
  void swap(DeviceArray& o) noexcept {
    std::swap(ptr_, o.ptr_);
    std::swap(count_, o.count_);
    std::swap(stream_, o.stream_);
  }
  T* ptr_ = nullptr;
  std::size_t count_ = 0;
  cudaStream_t stream_ = nullptr;
};

// Launch accounting: every kernel launch of this library goes through
// count_launch() so callers (benchmarks) can report how many ran.
void count_launch(unsigned n = 1);
// Takes back launches counted while a CUDA graph was being captured (they
// are counted again each time the graph is replayed).
void uncount_launch(unsigned long long n);
unsigned long long launch_count();

inline int num_sms() {
  static int sms = [] {
    int dev = 0, value = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&value, cudaDevAttrMultiProcessorCount, dev);
    return value > 0 ? value : 148;
  }();
  return sms;
}

inline unsigned ceil_div(std::size_t a, std::size_t b) {
  return static_cast<unsigned>((a + b - 1) / b);
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ double as_f64(T v) {
  return static_cast<double>(v);
}

// BF16 storage of the predictors (precision 16): widened exactly to FP64
using bf16 = __nv_bfloat16;
__device__ __forceinline__ double as_f64(bf16 v) {
  return static_cast<double>(__bfloat162float(v));
}

// type of responses and results for a predictor storage type: BF16
// predictors take FP32 responses and return FP32 results
template <class T> struct io_type { using type = T; };
template <> struct io_type<bf16> { using type = float; };

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; every thread receives the total. scratch: >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warps = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double total = 0.0;
  for (int w = 0; w < warps; ++w) total += scratch[w];
  __syncthreads();
  return total;
}

// Non-finite / failure flag shared by the kernels of one call.
__device__ __forceinline__ void flag_error(int* flag, int code) {
  if (flag) atomicExch(flag, code);
}

}  // namespace fpls
