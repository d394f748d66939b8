// FP64-accumulating tiled GEMM on the CUDA cores (DFMA), sm_100a.
//
//   C[M x N] = alpha * op(A)[M x K] * diag(kscale) * op(B)[K x N] (+ beta C)
//
// A and B are column-major and may be float or double (converted to double as
// they are staged into shared memory), so FP32-stored predictors are consumed
// in place without a conversion pass. Every product and sum is FP64: this is
// the precision contract of the fitting path (results track the FP64 CPU
// reference to ~1e-12 rather than to FP32 rounding).
//
// Tiling: 128 x 128 block tile, BK = 8, 256 threads, 8 x 8 register tile per
// thread, double-buffered shared memory with register prefetch of the next
// k-slab. Split-K over blockIdx.z writes partial tiles to disjoint slices of
// `C` (slice stride `split_stride`) which gemm_reduce_splits sums in a fixed
// order, so results are bitwise deterministic run to run.
#include "common.cuh"
#include "kernels.cuh"

#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

namespace fpls {

namespace {

constexpr int BM = 128, BN = 128, BK = 8, THREADS = 256;

template <class T, bool TRANS>
struct TileLoader;

// Loads a BM x BK slab of op(A) (or, transposed roles, a BK x BN slab of
// op(B)) into registers. `rows` indexes the M (or N) dimension, `ks` the K
// dimension. Element (r, k) of op(X) lives at X[r + k*ld] when !TRANS and at
// X[k + r*ld] when TRANS.
template <class T>
struct TileLoader<T, false> {  // contiguous along rows
  static __device__ __forceinline__ void load(const T* X, long ld, int rows,
                                              int ks, int r0, int k0,
                                              double (&reg)[4]) {
    const int t = threadIdx.x;
    const int r = r0 + (t & 127);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = k0 + (t >> 7) + 2 * q;
      reg[q] = (r < rows && k < ks) ? as_f64(X[r + (long)k * ld]) : 0.0;
    }
  }
  static __device__ __forceinline__ void store(double (*S)[BM + 4],
                                               const double (&reg)[4]) {
    const int t = threadIdx.x;
#pragma unroll
    for (int q = 0; q < 4; ++q) S[(t >> 7) + 2 * q][t & 127] = reg[q];
  }
};

template <class T>
struct TileLoader<T, true> {  // contiguous along k
  static __device__ __forceinline__ void load(const T* X, long ld, int rows,
                                              int ks, int r0, int k0,
                                              double (&reg)[4]) {
    const int t = threadIdx.x;
    const int k = k0 + (t & 7);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = r0 + (t >> 3) + 32 * q;
      reg[q] = (r < rows && k < ks) ? as_f64(X[k + (long)r * ld]) : 0.0;
    }
  }
  static __device__ __forceinline__ void store(double (*S)[BM + 4],
                                               const double (&reg)[4]) {
    const int t = threadIdx.x;
#pragma unroll
    for (int q = 0; q < 4; ++q) S[t & 7][(t >> 3) + 32 * q] = reg[q];
  }
};

template <class TA, class TB, bool TA_T, bool TB_T>
__global__ void __launch_bounds__(THREADS)
    dgemm_tiled(int M, int N, int K, const TA* __restrict__ A, long lda,
                const TB* __restrict__ B, long ldb,
                const double* __restrict__ kscale, double alpha, double beta,
                double* __restrict__ C, long ldc, long split_stride,
                int k_per_split) {
  __shared__ __align__(16) double As[2][BK][BM + 4];
  __shared__ __align__(16) double Bs[2][BK][BN + 4];

  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  double* Cz = C + (long)blockIdx.z * split_stride;

  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;

  double ra[4], rb[4];
  auto load_slab = [&](int k0) {
    TileLoader<TA, TA_T>::load(A, lda, M, kend, m0, k0, ra);
    TileLoader<TB, !TB_T>::load(B, ldb, N, kend, n0, k0, rb);
    if (kscale) {
      // scale the K index of op(A): recompute which k each register holds
      const int t = threadIdx.x;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = TA_T ? k0 + (t & 7) : k0 + (t >> 7) + 2 * q;
        if (k < kend) ra[q] *= kscale[k];
      }
    }
  };

  int buf = 0;
  if (kbeg < kend) {
    load_slab(kbeg);
    TileLoader<TA, TA_T>::store(As[0], ra);
    TileLoader<TB, !TB_T>::store(Bs[0], rb);
  }
  __syncthreads();

  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    const bool more = k0 + BK < kend;
    if (more) load_slab(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double a[8], b[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 va = *reinterpret_cast<const double2*>(&As[buf][kk][ty * 4 + 2 * (i & 1) + 64 * (i >> 1)]);
        a[2 * i] = va.x;
        a[2 * i + 1] = va.y;
        const double2 vb = *reinterpret_cast<const double2*>(&Bs[buf][kk][tx * 4 + 2 * (i & 1) + 64 * (i >> 1)]);
        b[2 * i] = vb.x;
        b[2 * i + 1] = vb.y;
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (more) {
      TileLoader<TA, TA_T>::store(As[buf ^ 1], ra);
      TileLoader<TB, !TB_T>::store(Bs[buf ^ 1], rb);
    }
    __syncthreads();
    buf ^= 1;
  }

  // thread (ty, tx) owns rows ty*4 + {0..3} and ty*4 + 64 + {0..3},
  // columns tx*4 + {0..3} and tx*4 + 64 + {0..3}
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int col = n0 + tx * 4 + (j & 3) + 64 * (j >> 2);
    if (col >= N) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int row = m0 + ty * 4 + (i & 3) + 64 * (i >> 2);
      if (row >= M) continue;
      double* dst = Cz + row + (long)col * ldc;
      const double v = alpha * acc[i][j];
      *dst = (beta != 0.0) ? fma(beta, *dst, v) : v;
    }
  }
}

__global__ void gemm_reduce_splits(int M, int N, double* C, long ldc,
                                   long split_stride, int splits) {
  const long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int row = (int)(idx % M);
    const long col = idx / M;
    double* dst = C + row + col * ldc;
    double s = *dst;
    for (int z = 1; z < splits; ++z) s += dst[z * split_stride];
    *dst = s;
  }
}

// C[:, :] = sum of `splits` contiguous M x N slices (fixed order)
__global__ void sum_slices(const double* __restrict__ slices, int splits, int M,
                           int N, double* C, long ldc) {
  const long total = (long)M * N;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    double v = slices[idx];
    for (int z = 1; z < splits; ++z) v += slices[idx + z * total];
    C[(idx % M) + (idx / M) * ldc] = v;
  }
}

// Split-K factor (1..4) that best fills whole waves of SMs for an MMA tile
// grid, each split keeping at least 512 of K; 1 when no split helps.
int gemm_mma_wave_splits(int M, int N, int K) {
  const double tiles = (double)ceil_div(M, 128) * ceil_div(N, 128);
  const double sms = num_sms();
  int best = 1;
  double best_score = 0.0;
  for (int s = 1; s <= 4; ++s) {
    if (s > 1 && K / s < 512) break;
    const double waves = tiles * s / sms;
    const double eff = waves / std::ceil(waves);
    const double score = eff - 0.01 * (s - 1);
    if (score > best_score + 1e-9) {
      best_score = score;
      best = s;
    }
  }
  return best;
}

template <class TA, class TB, bool TA_T, bool TB_T>
void launch(const GemmArgs& g, const TA* A, const TB* B, cudaStream_t stream) {
  const dim3 grid(ceil_div(g.N, BN), ceil_div(g.M, BM), g.splits);
  const int kps = ((g.K + g.splits - 1) / g.splits + BK - 1) / BK * BK;
  dgemm_tiled<TA, TB, TA_T, TB_T><<<grid, THREADS, 0, stream>>>(
      g.M, g.N, g.K, A, g.lda, B, g.ldb, g.kscale, g.alpha, g.beta, g.C,
      g.ldc, g.split_stride, kps);
  count_launch();
  FPLS_LAUNCH("dgemm_tiled");
}

template <class TA, class TB>
void dispatch(const GemmArgs& g, const TA* A, const TB* B, cudaStream_t s) {
  if (!g.trans_a && !g.trans_b) launch<TA, TB, false, false>(g, A, B, s);
  else if (!g.trans_a && g.trans_b) launch<TA, TB, false, true>(g, A, B, s);
  else if (g.trans_a && !g.trans_b) launch<TA, TB, true, false>(g, A, B, s);
  else launch<TA, TB, true, true>(g, A, B, s);
}

}  // namespace

// Live timing of GEMM launches (benchmark instrumentation): when enabled,
// every gemm_f64 call is bracketed by CUDA events on its own stream.
namespace {
struct GemmTiming {
  bool enabled = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
  std::vector<double> flops;
};
GemmTiming& timing() {
  static GemmTiming t;
  return t;
}
}  // namespace

void gemm_profile_enable(bool on) { timing().enabled = on; }

void gemm_profile_read(double* ms, double* flops, unsigned long long* launches) {
  GemmTiming& t = timing();
  double total_ms = 0.0, total_flops = 0.0;
  for (size_t k = 0; k < t.events.size(); ++k) {
    float e = 0.f;
    cudaEventSynchronize(t.events[k].second);
    cudaEventElapsedTime(&e, t.events[k].first, t.events[k].second);
    total_ms += e;
    total_flops += t.flops[k];
    cudaEventDestroy(t.events[k].first);
    cudaEventDestroy(t.events[k].second);
  }
  if (ms) *ms = total_ms;
  if (flops) *flops = total_flops;
  if (launches) *launches = t.events.size();
  t.events.clear();
  t.flops.clear();
}

void gemm_f64(const GemmArgs& g, cudaStream_t stream) {
  require(g.M >= 0 && g.N >= 0 && g.K >= 0, "invalid GEMM dimensions");
  if (g.M == 0 || g.N == 0) return;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (timing().enabled) {
    FPLS_CHECK(cudaEventCreate(&ev0));
    FPLS_CHECK(cudaEventCreate(&ev1));
    FPLS_CHECK(cudaEventRecord(ev0, stream));
  }
  require(g.splits >= 1, "invalid GEMM split count");
  require(g.splits == 1 || g.beta == 0.0, "split-K GEMM requires beta == 0");
  const bool use_mma = gemm_mma_supported(g);
  require(!g.lower || (g.M == g.N && use_mma && g.splits == 1 && g.beta == 0.0),
          "symmetric GEMM needs the FP64 tensor-core path");
  const int wave_splits = use_mma && !g.lower && g.splits == 1 && g.beta == 0.0
                              ? gemm_mma_wave_splits(g.M, g.N, g.K) : 1;
  DeviceArray<double> slices;
  if (wave_splits > 1) {
    // split K so the tile count fills whole waves of SMs; the slices are
    // summed in a fixed order afterwards (deterministic)
    slices.allocate((size_t)wave_splits * g.M * g.N, stream);
    GemmArgs h = g;
    h.C = slices.get();
    h.ldc = g.M;
    h.splits = wave_splits;
    h.split_stride = (long)g.M * g.N;
    gemm_mma_launch(h, false, stream);
    const long total = (long)g.M * g.N;
    sum_slices<<<(unsigned)std::min<long>((total + 255) / 256, 16L * num_sms()), 256, 0, stream>>>(
        slices.get(), wave_splits, g.M, g.N, g.C, g.ldc);
    count_launch();
    FPLS_LAUNCH("sum_slices");
  } else if (use_mma)
    gemm_mma_launch(g, g.lower, stream);
  else if (g.a_f32 && g.b_f32)
    dispatch(g, static_cast<const float*>(g.A), static_cast<const float*>(g.B), stream);
  else if (g.a_f32)
    dispatch(g, static_cast<const float*>(g.A), static_cast<const double*>(g.B), stream);
  else if (g.b_f32)
    dispatch(g, static_cast<const double*>(g.A), static_cast<const float*>(g.B), stream);
  else
    dispatch(g, static_cast<const double*>(g.A), static_cast<const double*>(g.B), stream);
  if (g.lower) mirror_lower_triangle(g.C, g.M, g.ldc, stream);
  if (g.splits > 1) {
    const long total = (long)g.M * g.N;
    const unsigned blocks = (unsigned)std::min<long>((total + 255) / 256, 4L * num_sms());
    gemm_reduce_splits<<<blocks, 256, 0, stream>>>(g.M, g.N, g.C, g.ldc,
                                                   g.split_stride, g.splits);
    count_launch();
    FPLS_LAUNCH("gemm_reduce_splits");
  }
  if (ev0) {
    FPLS_CHECK(cudaEventRecord(ev1, stream));
    timing().events.emplace_back(ev0, ev1);
    // algorithmic FLOPs: a symmetric product needs only its lower triangle
    timing().flops.push_back(g.lower ? (double)g.M * (g.M + 1.0) * g.K
                                     : 2.0 * g.M * (double)g.N * g.K);
  }
}

int gemm_pick_splits(int M, int N, int K) {
  const long tiles = (long)ceil_div(M, BM) * ceil_div(N, BN);
  const long want = 2L * num_sms();
  if (tiles >= want || K < 4 * BK * 8) return 1;
  long s = (want + tiles - 1) / tiles;
  s = std::min<long>(s, K / (BK * 8));
  return (int)std::max<long>(1, std::min<long>(s, 64));
}

}  // namespace fpls
