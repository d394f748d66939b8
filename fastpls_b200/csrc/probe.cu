// FP64 FMA throughput probe: the roofline denominator for the FP64-bound
// kernels of this library, measured on the running device (the measured
// peak file holds HBM copy and BF16 GEMM figures only).
#include "common.cuh"
#include "kernels.cuh"

namespace fpls {

namespace {

// 8 independent FMA chains per thread, `iters` rounds; the result is written
// so the chains are not eliminated.
__global__ void __launch_bounds__(256) fma_chains(int iters, double seed, double* out) {
  double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
  double a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const double m = 0.999999999, c = 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
      a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
  }
  const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678) out[blockIdx.x] = s;  // practically never true
}

}  // namespace

double fp64_fma_tflops() {
  cudaStream_t s = nullptr;
  FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  DeviceArray<double> out(4096, s);
  const int blocks = num_sms() * 8, iters = 2048;
  cudaEvent_t e0, e1;
  FPLS_CHECK(cudaEventCreate(&e0));
  FPLS_CHECK(cudaEventCreate(&e1));
  fma_chains<<<blocks, 256, 0, s>>>(iters / 8, 1.0, out.get());  // warm-up
  FPLS_CHECK(cudaEventRecord(e0, s));
  fma_chains<<<blocks, 256, 0, s>>>(iters, 1.0, out.get());
  FPLS_CHECK(cudaEventRecord(e1, s));
  count_launch(2);
  FPLS_LAUNCH("fma_chains");
  FPLS_CHECK(cudaEventSynchronize(e1));
  float ms = 0.f;
  FPLS_CHECK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  out.release();
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace fpls
