// Cross-product X^T V with no memory allocation by the library.
//
// Some callers cannot let a library call cudaMalloc: hosts that own every
// byte of device memory through their own pool or budget (an R or Python
// runtime with a fixed GPU memory plan, a serving process that admits work
// by its memory footprint and must not be surprised by a library's own
// allocations), code that runs when the device is already close to full, and
// real-time loops that must not stall on the allocator. This entry point
// serves them: the caller passes device pointers for X, V and the output,
// and the per-chunk partial sums live in a fixed, file-scope device array.
//
// The array holds kNoAllocScratchDoubles doubles (16 MiB). Every GPU that
// loads the library keeps it for the lifetime of the process. Its address is
// looked up once per device (cudaGetSymbolAddress, on the first call made
// while that device is current), so that first call should happen before any
// stream capture starts. The looked-up address is kept for the process: after
// cudaDeviceReset the module is loaded again and the array may move, so a
// process that resets a device must not call this entry point again. Each
// call waits for its stream before returning. All calls share the array and
// every call overwrites
// the slots it uses before reading them (nothing has to start at zero), so
// calls that overlap on the GPU -- on different streams, or from different
// host threads -- race on it and must be serialised by the caller.
#include "../../include/fastpls_b200.h"
#include "common.cuh"
#include "kernels.cuh"

#include <algorithm>
#include <cstdio>
#include <mutex>

namespace fpls {

namespace {

constexpr long kNoAllocScratchDoubles = 2L * 1024 * 1024;  // 16 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// One warp per column j of the block's 32-column tile, lanes over the rows of
// this block's row chunk, V staged through shared memory `sub` rows at a time.
// partial[(chunk * p + j) * nb + c] = sum_{i in chunk} X[i, j] * V[i, c]; the
// first sub-tile writes the slot, later ones add to it (same block, fixed
// order), so no slot needs to start at zero.
template <class T>
__global__ void __launch_bounds__(256)
    xtv_chunks_noalloc(const T* __restrict__ X, int n, int p, long ld,
                       const double* __restrict__ V, long ldv, int nb, int rc,
                       int sub, double* __restrict__ partial) {
  extern __shared__ double vs[];  // sub x nb
  const int chunk = blockIdx.y;
  const int r0 = chunk * rc;
  const int rows = min(rc, n - r0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int s0 = 0; s0 < rows; s0 += sub) {
    const int cnt = min(sub, rows - s0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < cnt * nb; idx += blockDim.x) {
      const int r = idx % cnt, c = idx / cnt;
      vs[r + c * sub] = V[(r0 + s0 + r) + (long)c * ldv];
    }
    __syncthreads();
    for (int jj = warp; jj < 32; jj += 8) {
      const int j = blockIdx.x * 32 + jj;
      if (j >= p) break;
      const T* col = X + (long)j * ld + r0 + s0;
      for (int c = 0; c < nb; ++c) {
        double acc = 0.0;
        for (int r = lane; r < cnt; r += 32) acc = fma(as_f64(col[r]), vs[r + c * sub], acc);
        acc = warp_sum(acc);
        if (lane == 0) {
          double* slot = partial + ((long)chunk * p + j) * nb + c;
          *slot = s0 == 0 ? acc : *slot + acc;
        }
      }
    }
  }
}

__global__ void sum_chunks_noalloc(const double* __restrict__ partial,
                                   int chunks, int p, int nb, double* out,
                                   long ldo) {
  const long total = (long)p * nb;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int j = (int)(idx / nb), c = (int)(idx % nb);
    double s = 0.0;
    for (int k = 0; k < chunks; ++k) s += partial[((long)k * p + j) * nb + c];
    out[j + (long)c * ldo] = s;
  }
}

// Device address of the scratch array for the current device, looked up on
// the first call on that device.
double* scratch_address() {
  static std::mutex mu;
  static double* cached[kMaxDevices] = {};
  int dev = 0;
  FPLS_CHECK(cudaGetDevice(&dev));
  require(dev >= 0 && dev < kMaxDevices, "device index beyond the no-allocation table");
  std::lock_guard<std::mutex> lock(mu);
  if (!cached[dev]) {
    void* ptr = nullptr;
    FPLS_CHECK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    cached[dev] = static_cast<double*>(ptr);
  }
  return cached[dev];
}

template <class T>
void crossprod_noalloc(const T* X, int n, int p, long ld, const double* V,
                       long ldv, int nb, double* out, long ldo,
                       cudaStream_t stream) {
  require(X && V && out && n >= 1 && p >= 1 && nb >= 1 && nb <= 32 &&
              ld >= n && ldv >= n && ldo >= p,
          "invalid no-allocation cross-product input");
  const long per_chunk = (long)p * nb;
  if (per_chunk > kNoAllocScratchDoubles)
    throw std::invalid_argument(
        "p * nb exceeds the no-allocation scratch capacity of 2097152 doubles");
  double* scratch = scratch_address();
  const int rc = 1024;
  int chunks = (int)ceil_div(n, rc);
  // chunks run along gridDim.y (at most 65535), and their partials must fit
  const long fit = std::min(kNoAllocScratchDoubles / per_chunk, 65535L);
  int rows_per_chunk = rc;
  if (chunks > fit) {  // fewer, taller chunks so the partials fit
    rows_per_chunk = (int)ceil_div(n, fit);
    chunks = (int)ceil_div(n, rows_per_chunk);
  }
  const int sub = std::max(32, std::min(rows_per_chunk, (48 * 1024 / 8) / nb));
  const size_t smem = (size_t)sub * nb * sizeof(double);
  xtv_chunks_noalloc<T><<<dim3(ceil_div(p, 32), chunks), 256, smem, stream>>>(
      X, n, p, ld, V, ldv, nb, rows_per_chunk, sub, scratch);
  FPLS_LAUNCH("xtv_chunks_noalloc");
  const long total = per_chunk;
  sum_chunks_noalloc<<<(unsigned)std::min<long>((total + 255) / 256, 8L * num_sms()), 256, 0, stream>>>(
      scratch, chunks, p, nb, out, ldo);
  FPLS_LAUNCH("sum_chunks_noalloc");
  count_launch(2);
}

}  // namespace

}  // namespace fpls

extern "C" FASTPLS_B200_API int fastpls_b200_crossprod_noalloc(
    const void* x, int precision, int n, int p, long ldx, const double* v,
    long ldv, int nb, double* out, long ldo, void* stream, char* error,
    size_t error_capacity) {
  if (error && error_capacity) error[0] = '\0';
  try {
    if (precision != 32 && precision != 64)
      throw std::invalid_argument("invalid no-allocation cross-product precision");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == 32)
      fpls::crossprod_noalloc(static_cast<const float*>(x), n, p, ldx, v, ldv, nb, out, ldo, s);
    else
      fpls::crossprod_noalloc(static_cast<const double*>(x), n, p, ldx, v, ldv, nb, out, ldo, s);
    fpls::check(cudaStreamSynchronize(s), "no-allocation cross-product");
    return 0;
  } catch (const std::exception& e) {
    if (error && error_capacity) std::snprintf(error, error_capacity, "%s", e.what());
    return 1;
  } catch (...) {
    if (error && error_capacity) std::snprintf(error, error_capacity, "%s", "unknown no-allocation error");
    return 1;
  }
}
