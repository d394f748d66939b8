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
#include "upload.cuh"
#include "../../include/fastpls_b200.h"
#include "kernels.cuh"
#include "small.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>
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
  upload_h2d(da.get(), a, sizeof(T) * rows_a * cols_a, s);
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
  jacobi_eigen(A, E, l, 60);
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

constexpr int kSketchMaxWidth = 120;  // 2 l^2 doubles + l ints <= 227 KB

// column sums of squares of (A - diag(scale) B), one block per column:
// out[j] = sum_i (A_ij - scale_j B_ij)^2 (scale / B may be null: sum A_ij^2)
__global__ void column_residual_sq(const double* __restrict__ A, const double* __restrict__ B,
                                   const double* __restrict__ scale, int rows, int cols,
                                   double* out) {
  __shared__ double scratch[32];
  for (int j = blockIdx.x; j < cols; j += gridDim.x) {
    const double sc = scale ? scale[j] : 0.0;
    double acc = 0.0;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
      const double r = B ? A[i + (long)j * rows] - sc * B[i + (long)j * rows] : A[i + (long)j * rows];
      acc = fma(r, r, acc);
    }
    acc = block_sum(acc, scratch);
    if (threadIdx.x == 0) out[j] = acc;
  }
}

// columns scaled to unit norm; a column whose norm is not above `tiny` is
// set to zero and reported with norm 0
__global__ void normalize_columns(double* A, int rows, int cols, double tiny, double* norms) {
  __shared__ double scratch[32];
  for (int j = blockIdx.x; j < cols; j += gridDim.x) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) acc = fma(A[i + (long)j * rows], A[i + (long)j * rows], acc);
    const double nrm = sqrt(block_sum(acc, scratch));
    const bool ok = isfinite(nrm) && nrm > tiny;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) A[i + (long)j * rows] = ok ? A[i + (long)j * rows] / nrm : 0.0;
    if (threadIdx.x == 0 && norms) norms[j] = ok ? nrm : 0.0;
  }
}

// Singular triplets on the device: U (n x r), V (p x r), d (r, decreasing).
struct Triplets {
  DeviceArray<double> U, V, d;
  std::vector<double> hd;
  int r = 0;
};

// X (FP64, n x p, resident) with the randomized SVD and the audit quantities
// of the reference's audited operator SVD (audited_rsvd.hpp).
class SvdOperator {
 public:
  SvdOperator(const double* X, int n, int p, cudaStream_t s) : X_(X), n_(n), p_(p), s_(s) {
    flag_.allocate(1, s);
    FPLS_CHECK(cudaMemsetAsync(flag_.get(), 0, sizeof(int), s));
  }

  // out (n x cols) = X B (p x cols) ; out (p x cols) = X^T B (n x cols)
  void times(const double* B, int cols, double* out, bool trans) {
    GemmArgs g;
    g.M = trans ? p_ : n_;
    g.N = cols;
    g.K = trans ? n_ : p_;
    g.A = X_;
    g.lda = n_;
    g.trans_a = trans;
    g.B = B;
    g.ldb = trans ? n_ : p_;
    g.C = out;
    g.ldc = trans ? p_ : n_;
    gemm_f64(g, s_);
  }

  // randomized SVD of rank r (rsvd.hpp:185-237): width l = min(r + os,
  // min(n, p)), `power` rounds, Gaussian sketch from `seed`
  Triplets rsvd(int r, int oversample, int power, unsigned long long seed) {
    const int n = n_, p = p_;
    const int l = std::min(std::min(n, p), r + std::max(oversample, 0));
    const size_t smem = 2 * (size_t)l * l * sizeof(double) + l * sizeof(int) + 16;
    require(l <= 256 && smem <= 227 * 1024, "fastsvd sketch too wide for one block");
    DeviceArray<double> Om((size_t)p * l, s_), Y((size_t)n * l, s_), Z((size_t)p * l, s_);
    gaussian_fill<<<grid_for((long)p * l), TB, 0, s_>>>(Om.get(), (long)p * l, seed);
    count_launch();
    FPLS_LAUNCH("gaussian_fill");
    times(Om.get(), l, Y.get(), false);
    for (int it = 0; it < std::max(power, 0); ++it) {
      orthonormalize(Y.get(), n, l, w_, flag_.get(), s_);
      times(Y.get(), l, Z.get(), true);
      orthonormalize(Z.get(), p, l, w_, flag_.get(), s_);
      times(Z.get(), l, Y.get(), false);
    }
    orthonormalize(Y.get(), n, l, w_, flag_.get(), s_);
    // B^T = X^T Q (p x l); G = B B^T = Z^T Z (l x l)
    times(Y.get(), l, Z.get(), true);
    DeviceArray<double> G((size_t)l * l, s_), Ub((size_t)l * r, s_), Ud((size_t)l * r, s_);
    Triplets t;
    t.r = r;
    t.d.allocate(r, s_);
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
    gemm_f64(g, s_);
    if (smem > 48 * 1024)
      FPLS_CHECK(cudaFuncSetAttribute(small_svd_from_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    small_svd_from_gram<<<1, jacobi_threads(l), smem, s_>>>(G.get(), l, r, t.d.get(), Ub.get(), Ud.get());
    count_launch();
    FPLS_LAUNCH("small_svd_from_gram");
    // U = Q Ub (n x r); V = B^T Ub / d = Z Ud (p x r)
    t.U.allocate((size_t)n * r, s_);
    t.V.allocate((size_t)p * r, s_);
    GemmArgs gu;
    gu.M = n;
    gu.N = r;
    gu.K = l;
    gu.A = Y.get();
    gu.lda = n;
    gu.B = Ub.get();
    gu.ldb = l;
    gu.C = t.U.get();
    gu.ldc = n;
    gemm_f64(gu, s_);
    GemmArgs gv = gu;
    gv.M = p;
    gv.A = Z.get();
    gv.lda = p;
    gv.B = Ud.get();
    gv.C = t.V.get();
    gv.ldc = p;
    gemm_f64(gv, s_);
    t.hd.resize(r);
    int bad = 0;
    FPLS_CHECK(cudaMemcpyAsync(&bad, flag_.get(), sizeof(int), cudaMemcpyDeviceToHost, s_));
    FPLS_CHECK(cudaMemcpyAsync(t.hd.data(), t.d.get(), sizeof(double) * r, cudaMemcpyDeviceToHost, s_));
    FPLS_CHECK(cudaStreamSynchronize(s_));
    if (bad) throw std::runtime_error("fastPLS rSVD sketch orthogonalization failed");
    return t;
  }

  // max_j max(||X v_j - d_j u_j||, ||X^T u_j - d_j v_j||) / max(|d_1|, eps)
  // (triplet_residual, audited_rsvd.hpp:103-143)
  double residual(const Triplets& t) {
    const int r = t.r;
    DeviceArray<double> F((size_t)n_ * r, s_), Rv((size_t)p_ * r, s_), sq((size_t)2 * r, s_);
    times(t.V.get(), r, F.get(), false);
    times(t.U.get(), r, Rv.get(), true);
    column_residual_sq<<<r, TB, 0, s_>>>(F.get(), t.U.get(), t.d.get(), n_, r, sq.get());
    column_residual_sq<<<r, TB, 0, s_>>>(Rv.get(), t.V.get(), t.d.get(), p_, r, sq.get() + r);
    count_launch(2);
    FPLS_LAUNCH("column_residual_sq");
    std::vector<double> h((size_t)2 * r);
    FPLS_CHECK(cudaMemcpyAsync(h.data(), sq.get(), sizeof(double) * 2 * r, cudaMemcpyDeviceToHost, s_));
    FPLS_CHECK(cudaStreamSynchronize(s_));
    const double scale = std::max(std::fabs(t.hd[0]), std::numeric_limits<double>::epsilon());
    double worst = 0.0;
    for (int j = 0; j < r; ++j) {
      const double a = std::sqrt(h[j]), b = std::sqrt(h[r + j]);
      if (!std::isfinite(a) || !std::isfinite(b)) return std::numeric_limits<double>::infinity();
      worst = std::max(worst, std::max(a, b) / scale);
    }
    return worst;
  }

  // largest component of X outside span(U[:, :retained]) found by three
  // random probes with two power steps each, over d_retained
  // (omitted_ratio, audited_rsvd.hpp:145-177; the probe draws come from the
  // device generator, not the reference's mt19937)
  double omitted(const Triplets& t, int retained, unsigned long long seed) {
    const int probes = 3;
    const double eps = std::numeric_limits<double>::epsilon();
    DeviceArray<double> right((size_t)p_ * probes, s_), left((size_t)n_ * probes, s_),
        coef((size_t)retained * probes, s_), norms(probes, s_);
    gaussian_fill<<<grid_for((long)p_ * probes), TB, 0, s_>>>(right.get(), (long)p_ * probes, seed);
    normalize_columns<<<probes, TB, 0, s_>>>(right.get(), p_, probes, eps, nullptr);
    count_launch(2);
    auto project_away = [&](double* L) {  // L -= U_r (U_r^T L)
      GemmArgs g;
      g.M = retained;
      g.N = probes;
      g.K = n_;
      g.A = t.U.get();
      g.lda = n_;
      g.trans_a = true;
      g.B = L;
      g.ldb = n_;
      g.C = coef.get();
      g.ldc = retained;
      gemm_f64(g, s_);
      GemmArgs h;
      h.M = n_;
      h.N = probes;
      h.K = retained;
      h.A = t.U.get();
      h.lda = n_;
      h.B = coef.get();
      h.ldb = retained;
      h.C = L;
      h.ldc = n_;
      h.alpha = -1.0;
      h.beta = 1.0;
      gemm_f64(h, s_);
    };
    for (int it = 0; it < 2; ++it) {
      times(right.get(), probes, left.get(), false);
      project_away(left.get());
      normalize_columns<<<probes, TB, 0, s_>>>(left.get(), n_, probes, eps, nullptr);
      times(left.get(), probes, right.get(), true);
      normalize_columns<<<probes, TB, 0, s_>>>(right.get(), p_, probes, eps, nullptr);
      count_launch(2);
    }
    times(right.get(), probes, left.get(), false);
    project_away(left.get());
    column_residual_sq<<<probes, TB, 0, s_>>>(left.get(), nullptr, nullptr, n_, probes, norms.get());
    count_launch();
    FPLS_LAUNCH("omitted_ratio");
    std::vector<double> h(probes);
    FPLS_CHECK(cudaMemcpyAsync(h.data(), norms.get(), sizeof(double) * probes, cudaMemcpyDeviceToHost, s_));
    FPLS_CHECK(cudaStreamSynchronize(s_));
    double largest = 0.0;
    for (double v : h) largest = std::max(largest, std::sqrt(v));
    const double boundary = std::max(std::fabs(t.hd[retained - 1]), eps);
    return largest / boundary;
  }

  // sqrt((r - ||U_a^T U_b||_F^2) / r)
  double subspace_error(const Triplets& a, const Triplets& b) {
    const int r = a.r;
    DeviceArray<double> O((size_t)r * r, s_), sq(r, s_);
    GemmArgs g;
    g.M = r;
    g.N = r;
    g.K = n_;
    g.A = a.U.get();
    g.lda = n_;
    g.trans_a = true;
    g.B = b.U.get();
    g.ldb = n_;
    g.C = O.get();
    g.ldc = r;
    gemm_f64(g, s_);
    column_residual_sq<<<r, TB, 0, s_>>>(O.get(), nullptr, nullptr, r, r, sq.get());
    count_launch();
    std::vector<double> h(r);
    FPLS_CHECK(cudaMemcpyAsync(h.data(), sq.get(), sizeof(double) * r, cudaMemcpyDeviceToHost, s_));
    FPLS_CHECK(cudaStreamSynchronize(s_));
    double overlap = 0.0;
    for (double v : h) overlap += v;
    overlap = std::min((double)r, overlap);
    return std::sqrt(std::max(0.0, ((double)r - overlap) / r));
  }

 private:
  const double* X_;
  int n_, p_;
  cudaStream_t s_;
  SvdScratch w_;
  DeviceArray<int> flag_;
};

bool finite_triplets(const Triplets& t) {
  for (double v : t.hd)
    if (!std::isfinite(v)) return false;
  return t.r > 0;
}

// audit_triplets (audited_rsvd.hpp:179-200): residual <= 1e-2 and omitted
// ratio (with the first dropped singular value) <= 1.01
bool audit_triplets(SvdOperator& op, const Triplets& t, int retained, uint32_t seed,
                    double& residual, double& omitted) {
  if (!finite_triplets(t) || t.r < retained) return false;
  residual = op.residual(t);
  omitted = op.omitted(t, retained, (uint32_t)(seed + 32452843u));
  const double eps = std::numeric_limits<double>::epsilon();
  if (t.r > retained) {
    const double boundary = std::max(std::fabs(t.hd[retained - 1]), eps);
    omitted = std::max(omitted, std::fabs(t.hd[retained] / boundary));
  }
  return std::isfinite(residual) && residual <= 1e-2 && std::isfinite(omitted) && omitted <= 1.01;
}

// consensus (audited_rsvd.hpp:202-241): subspace <= 1e-3, singular values
// <= 1e-5 (relative to the first), residual of the newer <= 1e-6
bool consensus(SvdOperator& op, const Triplets& a, const Triplets& b, double& subspace,
               double& singular, double& residual) {
  if (!finite_triplets(a) || !finite_triplets(b) || a.r != b.r) return false;
  subspace = op.subspace_error(a, b);
  const double scale = std::max(std::fabs(b.hd[0]), std::numeric_limits<double>::epsilon());
  double largest = 0.0;
  for (int j = 0; j < a.r; ++j) largest = std::max(largest, std::fabs(a.hd[j] - b.hd[j]));
  singular = largest / scale;
  residual = op.residual(b);
  return subspace <= 1e-3 && singular <= 1e-5 && residual <= 1e-6;
}

// Audited randomized SVD (audited_operator_rsvd, audited_rsvd.hpp:298-414):
// exact below 6 columns/rows; else up to three attempts at rank retained + 1
// with oversample >= (req, 32, 48), power >= (req, 3, 4) and seeds seed,
// seed + 104729, seed + 209759, accepted when the audit passes or two
// consecutive attempts agree; then up to four recoveries with a wider sketch
// and more power steps; an error when none is certified. audit (10 values):
// certified, deterministic fallback, attempts, oversample, power, seed,
// subspace error, singular value error, triplet residual, omitted ratio.
template <class T>
void fastsvd_impl(const T* x, int n, int p, int k, int oversample, int power,
                  unsigned long long seed64, double* U, double* d, double* V, double* audit) {
  require(n >= 1 && p >= 1 && k >= 1 && k <= std::min(n, p), "invalid fastsvd rank");
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
  xd.release();
  SvdOperator op(X.get(), n, p, s);
  const int maximum = std::min(n, p);
  const int retained = std::min(maximum, std::max(k, 1));
  const uint32_t seed = (uint32_t)seed64;
  double info[10] = {0};
  Triplets accepted;
  if (maximum < 6) {
    // exact: the sketch spans min(n, p) columns
    accepted = op.rsvd(retained, maximum, 0, seed);
    info[0] = 1;
    info[1] = 1;
    info[3] = std::max(oversample, 0);
    info[4] = std::max(power, 0);
    info[5] = seed;
  } else {
    const int audit_rank = std::min(maximum, retained + 1);
    const int oversamples[3] = {std::max(oversample, 0), std::max(oversample, 32), std::max(oversample, 48)};
    const int powers[3] = {std::max(power, 0), std::max(power, 3), std::max(power, 4)};
    const uint32_t seeds[3] = {seed, seed + 104729u, seed + 209759u};
    int os = 0, pw = 0;
    uint32_t sd = seed;
    double residual = std::numeric_limits<double>::infinity();
    double omitted = std::numeric_limits<double>::infinity();
    double subspace = 0.0, singular = 0.0;
    bool certified = false;
    int attempts = 0;
    Triplets previous;
    for (int attempt = 0; attempt < 3; ++attempt) {
      os = oversamples[attempt];
      pw = powers[attempt];
      sd = seeds[attempt];
      accepted = op.rsvd(audit_rank, os, pw, sd);
      ++attempts;
      const bool checked = audit_triplets(op, accepted, retained, sd, residual, omitted);
      bool agreed = false;
      if (attempt > 0) agreed = consensus(op, previous, accepted, subspace, singular, residual);
      certified = checked || agreed;
      if (certified) break;
      previous = std::move(accepted);
    }
    // widest sketch whose small l x l eigenproblem fits one block's shared
    // memory (2 l^2 doubles + l ints): recoveries widen up to it, then add
    // only power steps
    const int widest = std::max(audit_rank, std::min(maximum, kSketchMaxWidth));
    for (int recovery = 0; !certified && recovery < 4; ++recovery) {
      const int current = std::min(widest, audit_rank + std::max(os, 0));
      const int remaining = widest - current;
      const int enlarged = std::min(widest, std::max(current + std::min(32, remaining),
                                                     current + std::min(current, remaining)));
      os = enlarged - audit_rank;
      pw = std::max(pw, 6) + 2 * recovery;
      sd += 104729u * (uint32_t)(recovery + 1);
      accepted = op.rsvd(audit_rank, os, pw, sd);
      ++attempts;
      certified = audit_triplets(op, accepted, retained, sd, residual, omitted);
    }
    if (!certified)
      throw std::runtime_error(
          "rSVD recovery did not meet numerical tolerances within its workspace/iteration "
          "budget; no unchecked result was returned");
    info[0] = 1;
    info[2] = attempts;
    info[3] = os;
    info[4] = pw;
    info[5] = sd;
    info[6] = subspace;
    info[7] = singular;
    info[8] = residual;
    info[9] = omitted;
  }
  if (maximum < 6) info[2] = 1;
  // the first `retained` triplets (columns are contiguous: leading block)
  if (U) FPLS_CHECK(cudaMemcpyAsync(U, accepted.U.get(), sizeof(double) * n * retained, cudaMemcpyDeviceToHost, s));
  if (V) FPLS_CHECK(cudaMemcpyAsync(V, accepted.V.get(), sizeof(double) * p * retained, cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaStreamSynchronize(s));
  for (int j = 0; j < retained; ++j) d[j] = accepted.hd[j];
  if (audit)
    for (int j = 0; j < 10; ++j) audit[j] = info[j];
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
      fpls::fastsvd_impl(static_cast<const float*>(x), n, p, k, oversample, power, seed, u, d, v,
                         nullptr);
    else
      fpls::fastsvd_impl(static_cast<const double*>(x), n, p, k, oversample, power, seed, u, d, v,
                         nullptr);
    return 0;
  } catch (const std::exception& e) {
    if (error && error_capacity) std::snprintf(error, error_capacity, "%s", e.what());
    return 1;
  }
}

FASTPLS_B200_API int fastpls_b200_fastsvd_audited(const void* x, int precision, int n, int p,
                                                  int k, int oversample, int power,
                                                  unsigned long long seed, double* u, double* d,
                                                  double* v, double* audit, char* error,
                                                  size_t error_capacity) {
  if (error && error_capacity) error[0] = '\0';
  try {
    if (!x || !d || !audit || (precision != 32 && precision != 64))
      throw std::invalid_argument("invalid fastsvd input");
    if (precision == 32)
      fpls::fastsvd_impl(static_cast<const float*>(x), n, p, k, oversample, power, seed, u, d, v,
                         audit);
    else
      fpls::fastsvd_impl(static_cast<const double*>(x), n, p, k, oversample, power, seed, u, d, v,
                         audit);
    return 0;
  } catch (const std::exception& e) {
    if (error && error_capacity) std::snprintf(error, error_capacity, "%s", e.what());
    return 1;
  }
}

}  // extern "C"
