// fastcor and fastsvd on the device (FP64).
//
// fastcor (reference: R/main.R:12799-12817, src/r_api.cpp:4054-4166): every
// unit (row when byrow, else column) is centred and scaled to unit norm in
// FP64 (NaN when it has a non-finite value or zero spread); the correlation
// matrix is L R^T on the FP64 tensor path (symmetric when b is absent), or the
// per-unit dot products when diag is requested.
//
// fastsvd (reference: R/main.R:8181-8202 over the CPU randomized operator SVD,
// inst/include/fastpls/core/rsvd.hpp:185-237 and operator_rsvd.hpp:204-272):
// randomized subspace iteration in FP64 -- Gaussian sketch Omega (p x l,
// l = min(k + oversample, min(n, p))), Y = X Omega, `power` rounds of
// orthonormalise / X^T / orthonormalise / X, then B = Q^T X and the small SVD
// of B from the Jacobi eigen-decomposition of B B^T. Orthonormalisation is
// CholeskyQR2 (two Cholesky passes on the l x l Gram). When l reaches
// min(n, p) the sketch spans the whole range and the result is the exact
// truncated SVD. The Gaussian draws come from a counter-based generator
// (SplitMix64 hashing of (seed, index) into Box-Muller pairs), so a seed
// reproduces the sketch on any device.
#include "../../include/fastpls_b200.h"
#include "kernels.cuh"
#include "small.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

namespace fpls {

namespace {

constexpr int TB = 256;

unsigned grid_for(long total) {
  return (unsigned)std::min<long>((total + TB - 1) / TB, 16L * num_sms());
}

// ------------------------------------------------------------------ fastcor
template <class T>
__global__ void unit_normalize(const T* __restrict__ X, int rows, int cols,
                               bool byrow, double* L, int units, int features) {
  __shared__ double scratch[32];
  for (int u = blockIdx.x; u < units; u += gridDim.x) {
    double s = 0.0;
    int bad = 0;
    for (int f = threadIdx.x; f < features; f += blockDim.x) {
      const double v = as_f64(byrow ? X[u + (long)f * rows] : X[f + (long)u * rows]);
      if (!isfinite(v)) bad = 1;
      s += v;
    }
    const double mean = block_sum(s, scratch) / features;
    const double anybad = block_sum((double)bad, scratch);
    double ss = 0.0;
    for (int f = threadIdx.x; f < features; f += blockDim.x) {
      const double v = as_f64(byrow ? X[u + (long)f * rows] : X[f + (long)u * rows]) - mean;
      ss = fma(v, v, ss);
    }
    const double norm = sqrt(block_sum(ss, scratch));
    const bool ok = anybad == 0.0 && norm > 0.0;
    for (int f = threadIdx.x; f < features; f += blockDim.x) {
      const double v = as_f64(byrow ? X[u + (long)f * rows] : X[f + (long)u * rows]) - mean;
      L[u + (long)f * units] = ok ? v / norm : nan("");
    }
  }
}

__global__ void rowwise_dot(const double* __restrict__ L, const double* __restrict__ R,
                            int units, int features, double* out) {
  for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < units; u += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int f = 0; f < features; ++f) s = fma(L[u + (long)f * units], R[u + (long)f * units], s);
    out[u] = s;
  }
}

template <class T>
void fastcor_impl(const T* a, const T* b, int rows_a, int cols_a, int rows_b,
                  int cols_b, bool byrow, bool diag, double* out) {
  const int units_a = byrow ? rows_a : cols_a, feats = byrow ? cols_a : rows_a;
  const int units_b = b ? (byrow ? rows_b : cols_b) : units_a;
  const int feats_b = b ? (byrow ? cols_b : rows_b) : feats;
  if (b && feats_b != feats)
    throw std::invalid_argument("a and b must contain the same number of correlated features");
  if (!b) diag = false;
  if (diag && units_a != units_b)
    throw std::invalid_argument("diag = TRUE requires matching numbers of rows or columns");
  cudaStream_t s = nullptr;
  FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct Guard {
    cudaStream_t s;
    ~Guard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } guard{s};
  DeviceArray<T> da((size_t)rows_a * cols_a, s), db;
  FPLS_CHECK(cudaMemcpyAsync(da.get(), a, sizeof(T) * rows_a * cols_a, cudaMemcpyHostToDevice, s));
  DeviceArray<double> L((size_t)units_a * feats, s), R;
  unit_normalize<T><<<std::min(units_a, 8 * num_sms()), TB, 0, s>>>(da.get(), rows_a, cols_a, byrow,
                                                                      L.get(), units_a, feats);
  count_launch();
  if (b) {
    db.allocate((size_t)rows_b * cols_b, s);
    FPLS_CHECK(cudaMemcpyAsync(db.get(), b, sizeof(T) * rows_b * cols_b, cudaMemcpyHostToDevice, s));
    R.allocate((size_t)units_b * feats, s);
    unit_normalize<T><<<std::min(units_b, 8 * num_sms()), TB, 0, s>>>(db.get(), rows_b, cols_b, byrow,
                                                                        R.get(), units_b, feats);
    count_launch();
  }
  FPLS_LAUNCH("unit_normalize");
  const size_t count = diag ? (size_t)units_a : (size_t)units_a * units_b;
  DeviceArray<double> C(count, s);
  if (diag) {
    rowwise_dot<<<grid_for(units_a), TB, 0, s>>>(L.get(), R.get(), units_a, feats, C.get());
    count_launch();
    FPLS_LAUNCH("rowwise_dot");
  } else {
    GemmArgs g;
    g.M = units_a;
    g.N = units_b;
    g.K = feats;
    g.A = L.get();
    g.lda = units_a;
    g.B = b ? R.get() : L.get();
    g.ldb = units_b;
    g.trans_b = true;
    g.C = C.get();
    g.ldc = units_a;
    g.lower = !b && gemm_mma_supported(g);
    gemm_f64(g, s);
  }
  FPLS_CHECK(cudaMemcpyAsync(out, C.get(), sizeof(double) * count, cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaStreamSynchronize(s));
}

// ------------------------------------------------------------------ fastsvd
template <class T>
__global__ void widen_kernel(const T* __restrict__ in, long count, double* out) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < count;
       k += (long)gridDim.x * blockDim.x)
    out[k] = as_f64(in[k]);
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// standard normal draws, element k from (seed, k) only
__global__ void gaussian_fill(double* out, long count, unsigned long long seed) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < count;
       k += (long)gridDim.x * blockDim.x) {
    const long pair = k >> 1;
    const unsigned long long h1 = splitmix64(seed * 0x100000001B3ull + 2 * pair);
    const unsigned long long h2 = splitmix64(seed * 0x100000001B3ull + 2 * pair + 1);
    const double u1 = ((h1 >> 11) + 1.0) * 0x1.0p-53;  // (0, 1]
    const double u2 = (h2 >> 11) * 0x1.0p-53;
    const double r = sqrt(-2.0 * log(u1));
    out[k] = (k & 1) ? r * sin(2.0 * M_PI * u2) : r * cos(2.0 * M_PI * u2);
  }
}

// R^-1 of the Cholesky factor of the l x l Gram (one thread; l <= 256):
// G = L L^T, Q = Y L^-T. Writes Linv^T (upper) into out.
__global__ void chol_inverse_upper(const double* __restrict__ G, int l, double* work,
                                   double* out, int* flag) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < l * l; ++k) work[k] = G[k];
  double scale = 0.0;
  for (int i = 0; i < l; ++i) scale = fmax(scale, fabs(G[i + i * l]));
  if (!cholesky_serial(work, l, 1e-30 * scale)) {
    flag_error(flag, 7);
    for (int k = 0; k < l * l; ++k) out[k] = 0.0;
    return;
  }
  // out = (L^-1)^T: solve L Z = I column by column, Z lower; out = Z^T
  for (int c = 0; c < l; ++c) {
    for (int i = 0; i < l; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int q = 0; q < i; ++q) v -= work[i + q * l] * out[c + q * l];
      out[c + i * l] = v / work[i + i * l];  // out[c, i] = Z[i, c]
    }
  }
}

// eigen-decomposition of the small l x l Gram B B^T -> sorted d (k), Ub (l x k)
__global__ void small_svd_from_gram(const double* __restrict__ G, int l, int k,
                                    double* d, double* Ub, double* Uinv_d) {
  extern __shared__ double sm[];
  double* A = sm;
  double* E = sm + l * l;
  int* order = reinterpret_cast<int*>(E + l * l);
  for (int idx = threadIdx.x; idx < l * l; idx += blockDim.x) A[idx] = G[idx];
  __syncthreads();
  jacobi_eigen_warp<4>(A, E, l, 60);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < l; ++i) order[i] = i;
    for (int i = 1; i < l; ++i) {
      const int key = order[i];
      int j = i - 1;
      while (j >= 0 && A[order[j] + order[j] * l] < A[key + key * l]) {
        order[j + 1] = order[j];
        --j;
      }
      order[j + 1] = key;
    }
    for (int c = 0; c < k; ++c) {
      const int src = order[c];
      const double lam = fmax(A[src + src * l], 0.0);
      const double sv = sqrt(lam);
      int arg = 0;
      for (int r = 1; r < l; ++r)
        if (fabs(E[r + src * l]) > fabs(E[arg + src * l])) arg = r;
      const double sgn = E[arg + src * l] < 0.0 ? -1.0 : 1.0;
      d[c] = sv;
      for (int r = 0; r < l; ++r) {
        const double v = sgn * E[r + src * l];
        Ub[r + c * l] = v;
        Uinv_d[r + c * l] = sv > 0.0 ? v / sv : 0.0;
      }
    }
  }
}

struct SvdScratch {
  DeviceArray<double> G, work, inv, tmp;
};

// Q (rows x l) <- orthonormal basis of Y via CholeskyQR2 (in place)
void orthonormalize(double* Y, int rows, int l, SvdScratch& w, int* flag, cudaStream_t s) {
  w.G.reserve((size_t)l * l, s);
  w.work.reserve((size_t)l * l, s);
  w.inv.reserve((size_t)l * l, s);
  w.tmp.reserve((size_t)rows * l, s);
  for (int pass = 0; pass < 2; ++pass) {
    GemmArgs g;
    g.M = l;
    g.N = l;
    g.K = rows;
    g.A = Y;
    g.lda = rows;
    g.trans_a = true;
    g.B = Y;
    g.ldb = rows;
    g.C = w.G.get();
    g.ldc = l;
    gemm_f64(g, s);
    chol_inverse_upper<<<1, 32, 0, s>>>(w.G.get(), l, w.work.get(), w.inv.get(), flag);
    count_launch();
    FPLS_LAUNCH("chol_inverse_upper");
    GemmArgs h;
    h.M = rows;
    h.N = l;
    h.K = l;
    h.A = Y;
    h.lda = rows;
    h.B = w.inv.get();
    h.ldb = l;
    h.C = w.tmp.get();
    h.ldc = rows;
    gemm_f64(h, s);
    FPLS_CHECK(cudaMemcpyAsync(Y, w.tmp.get(), sizeof(double) * rows * l, cudaMemcpyDeviceToDevice, s));
  }
}

template <class T>
void fastsvd_impl(const T* x, int n, int p, int k, int oversample, int power,
                  unsigned long long seed, double* U, double* d, double* V) {
  require(n >= 1 && p >= 1 && k >= 1 && k <= std::min(n, p), "invalid fastsvd rank");
  const int l = std::min(std::min(n, p), k + std::max(oversample, 0));
  require(l <= 256, "fastsvd on the device supports k + oversample <= 256");
  cudaStream_t s = nullptr;
  FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct Guard {
    cudaStream_t s;
    ~Guard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } guard{s};
  DeviceArray<T> xd((size_t)n * p, s);
  FPLS_CHECK(cudaMemcpyAsync(xd.get(), x, sizeof(T) * n * p, cudaMemcpyHostToDevice, s));
  // FP64 copy so every product takes the FP64 tensor path
  DeviceArray<double> X((size_t)n * p, s);
  widen_kernel<T><<<grid_for((long)n * p), TB, 0, s>>>(xd.get(), (long)n * p, X.get());
  count_launch();
  FPLS_LAUNCH("widen");
  DeviceArray<int> flag(1, s);
  FPLS_CHECK(cudaMemsetAsync(flag.get(), 0, sizeof(int), s));
  DeviceArray<double> Om((size_t)p * l, s), Y((size_t)n * l, s), Z((size_t)p * l, s);
  gaussian_fill<<<grid_for((long)p * l), TB, 0, s>>>(Om.get(), (long)p * l, seed);
  count_launch();
  FPLS_LAUNCH("gaussian_fill");
  SvdScratch w;
  auto XtimesB = [&](const double* B, int cols, double* out) {  // X (n x p) * B (p x cols)
    GemmArgs g;
    g.M = n;
    g.N = cols;
    g.K = p;
    g.A = X.get();
    g.lda = n;
    g.B = B;
    g.ldb = p;
    g.C = out;
    g.ldc = n;
    gemm_f64(g, s);
  };
  auto XtTimesB = [&](const double* B, int cols, double* out) {  // X^T (p x n) * B (n x cols)
    GemmArgs g;
    g.M = p;
    g.N = cols;
    g.K = n;
    g.A = X.get();
    g.lda = n;
    g.trans_a = true;
    g.B = B;
    g.ldb = n;
    g.C = out;
    g.ldc = p;
    gemm_f64(g, s);
  };
  XtimesB(Om.get(), l, Y.get());
  for (int it = 0; it < std::max(power, 0); ++it) {
    orthonormalize(Y.get(), n, l, w, flag.get(), s);
    XtTimesB(Y.get(), l, Z.get());
    orthonormalize(Z.get(), p, l, w, flag.get(), s);
    XtimesB(Z.get(), l, Y.get());
  }
  orthonormalize(Y.get(), n, l, w, flag.get(), s);
  // B^T = X^T Q (p x l); G = B B^T = Z^T Z (l x l)
  XtTimesB(Y.get(), l, Z.get());
  DeviceArray<double> G((size_t)l * l, s), dd(k, s), Ub((size_t)l * k, s), Ud((size_t)l * k, s);
  GemmArgs g;
  g.M = l;
  g.N = l;
  g.K = p;
  g.A = Z.get();
  g.lda = p;
  g.trans_a = true;
  g.B = Z.get();
  g.ldb = p;
  g.C = G.get();
  g.ldc = l;
  gemm_f64(g, s);
  const size_t smem = 2 * (size_t)l * l * sizeof(double) + l * sizeof(int) + 16;
  if (smem > 48 * 1024)
    FPLS_CHECK(cudaFuncSetAttribute(small_svd_from_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  require(smem <= 227 * 1024, "fastsvd sketch too wide for one block");
  small_svd_from_gram<<<1, 64, smem, s>>>(G.get(), l, k, dd.get(), Ub.get(), Ud.get());
  count_launch();
  FPLS_LAUNCH("small_svd_from_gram");
  // U = Q Ub (n x k); V = B^T Ub / d = Z Ud (p x k)
  DeviceArray<double> Uo((size_t)n * k, s), Vo((size_t)p * k, s);
  GemmArgs gu;
  gu.M = n;
  gu.N = k;
  gu.K = l;
  gu.A = Y.get();
  gu.lda = n;
  gu.B = Ub.get();
  gu.ldb = l;
  gu.C = Uo.get();
  gu.ldc = n;
  gemm_f64(gu, s);
  GemmArgs gv = gu;
  gv.M = p;
  gv.A = Z.get();
  gv.lda = p;
  gv.B = Ud.get();
  gv.C = Vo.get();
  gv.ldc = p;
  gemm_f64(gv, s);
  int bad = 0;
  FPLS_CHECK(cudaMemcpyAsync(&bad, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  if (U) FPLS_CHECK(cudaMemcpyAsync(U, Uo.get(), sizeof(double) * n * k, cudaMemcpyDeviceToHost, s));
  if (V) FPLS_CHECK(cudaMemcpyAsync(V, Vo.get(), sizeof(double) * p * k, cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaMemcpyAsync(d, dd.get(), sizeof(double) * k, cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaStreamSynchronize(s));
  if (bad) throw std::runtime_error("fastPLS rSVD sketch orthogonalization failed");
}

}  // namespace
}  // namespace fpls

extern "C" {

FASTPLS_B200_API int fastpls_b200_fastcor(const void* a, const void* b, int precision,
                                          int rows_a, int cols_a, int rows_b, int cols_b,
                                          int byrow, int diag, double* out, char* error,
                                          size_t error_capacity) {
  if (error && error_capacity) error[0] = '\0';
  try {
    if (!a || !out || (precision != 32 && precision != 64) || rows_a < 1 || cols_a < 1 ||
        (b && (rows_b < 1 || cols_b < 1)))
      throw std::invalid_argument("invalid fast Pearson correlation input");
    if (precision == 32)
      fpls::fastcor_impl(static_cast<const float*>(a), static_cast<const float*>(b), rows_a, cols_a,
                         rows_b, cols_b, byrow != 0, diag != 0, out);
    else
      fpls::fastcor_impl(static_cast<const double*>(a), static_cast<const double*>(b), rows_a, cols_a,
                         rows_b, cols_b, byrow != 0, diag != 0, out);
    return 0;
  } catch (const std::exception& e) {
    if (error && error_capacity) std::snprintf(error, error_capacity, "%s", e.what());
    return 1;
  }
}

FASTPLS_B200_API int fastpls_b200_fastsvd(const void* x, int precision, int n, int p, int k,
                                          int oversample, int power, unsigned long long seed,
                                          double* u, double* d, double* v, char* error,
                                          size_t error_capacity) {
  if (error && error_capacity) error[0] = '\0';
  try {
    if (!x || !d || (precision != 32 && precision != 64))
      throw std::invalid_argument("invalid fastsvd input");
    if (precision == 32)
      fpls::fastsvd_impl(static_cast<const float*>(x), n, p, k, oversample, power, seed, u, d, v);
    else
      fpls::fastsvd_impl(static_cast<const double*>(x), n, p, k, oversample, power, seed, u, d, v);
    return 0;
  } catch (const std::exception& e) {
    if (error && error_capacity) std::snprintf(error, error_capacity, "%s", e.what());
    return 1;
  }
}

}  // extern "C"
