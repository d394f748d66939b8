// Pooled-covariance LDA on latent scores (FP64 on the device).
//
// Reference: train_lda_prefixes / finalize_lda_prefixes
// (inst/include/fastpls/core/lda.hpp:88-223) and ResidentLda
// (src/cuda_resident_lda.cuh:41-121): class means, pooled within-class
// covariance (T^T T - sum_c n_c mu_c mu_c^T) / max(1, n - c), ridge
// rho * trace / k for rho in {1e-8, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2} (first that
// factors), Cholesky solve, constants -0.5 mu^T Sigma^-1 mu + log prior.
// Moments come from two FP64 GEMMs (T^T T and onehot^T T); the per-prefix
// k x k factorisation runs in one block.
#include "lda.cuh"
#include "small.cuh"

#include <algorithm>
#include <cfloat>

namespace fpls {

namespace {

__global__ void one_hot_kernel(const int* __restrict__ labels, int n, int c,
                               double* oh) {
  const long total = (long)n * c;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), k = (int)(idx / n);
    oh[idx] = labels[i] == k + 1 ? 1.0 : 0.0;
  }
}

// One block: pooled covariance for the first k components, ridge retries,
// linear (c x k, row-major per class) and constants (c).
__global__ void lda_finalize(const double* __restrict__ gram, int a,
                             const double* __restrict__ sums, int c,
                             const double* __restrict__ counts, int n, int k,
                             double* linear, double* constants, double* ridge,
                             int* flag) {
  extern __shared__ double sm[];
  double* cov = sm;                 // k x k
  double* L = cov + k * k;          // k x k
  double* means = L + k * k;        // c x k (class-major)
  double* rhs = means + c * k;      // k
  const int t = threadIdx.x;
  for (int idx = t; idx < c * k; idx += blockDim.x) {
    const int cls = idx / k, j = idx % k;
    means[cls * k + j] = sums[cls + (long)j * c] / counts[cls];
  }
  __syncthreads();
  const double denom = (double)max(1, n > c ? n - c : 1);
  for (int idx = t; idx < k * k; idx += blockDim.x) {
    const int i = idx % k, j = idx / k;
    double v = gram[i + (long)j * a];
    for (int cls = 0; cls < c; ++cls) v -= counts[cls] * means[cls * k + i] * means[cls * k + j];
    cov[i + j * k] = v / denom;
  }
  __syncthreads();
  if (t == 0) {
    double scale = 0.0;
    for (int i = 0; i < k; ++i) scale += cov[i + i * k];
    scale /= k;
    if (!isfinite(scale) || scale <= 0.0) scale = 1.0;
    const double grid[6] = {1e-8, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2};
    bool solved = false;
    for (int g = 0; g < 6 && !solved; ++g) {
      for (int idx = 0; idx < k * k; ++idx) L[idx] = cov[idx];
      if (!cholesky_serial(L, k, grid[g] * scale)) continue;
      bool ok = true;
      for (int cls = 0; cls < c && ok; ++cls) {
        for (int j = 0; j < k; ++j) rhs[j] = means[cls * k + j];
        ok = cholesky_solve_serial(L, k, rhs);
        for (int j = 0; j < k; ++j) linear[cls + (long)j * c] = rhs[j];
      }
      if (!ok) continue;
      solved = true;
      *ridge = grid[g] * scale;
    }
    if (!solved) flag_error(flag, 5);
    for (int cls = 0; cls < c; ++cls) {
      double prod = 0.0;
      for (int j = 0; j < k; ++j) prod += means[cls * k + j] * linear[cls + (long)j * c];
      const double prior = counts[cls] / n;
      constants[cls] = -0.5 * prod + log(fmax(prior, DBL_MIN));
    }
  }
}

__global__ void fill_constants(double* out, int rows, int c, long ldo,
                               const double* constants) {
  const long total = (long)rows * c;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % rows), k = (int)(idx / rows);
    out[i + (long)k * ldo] = constants[k];
  }
}

}  // namespace

void LdaState::train(const double* scores, int n_, long lds, int a_,
                     const int* labels, int c_, const std::vector<int>& counts,
                     int* flag_, cudaStream_t stream) {
  n = n_;
  a = a_;
  c = c_;
  flag = flag_;
  std::vector<double> hc(c);
  for (int k = 0; k < c; ++k) {
    require(counts[k] > 0, "fastPLS LDA received an empty class");
    hc[k] = counts[k];
  }
  counts_dev.allocate(c, stream);
  FPLS_CHECK(cudaMemcpyAsync(counts_dev.get(), hc.data(), sizeof(double) * c,
                             cudaMemcpyHostToDevice, stream));
  gram.allocate((size_t)a * a, stream);
  sums.allocate((size_t)c * a, stream);
  DeviceArray<double> oh((size_t)n * c, stream);
  one_hot_kernel<<<std::min<unsigned>(ceil_div((size_t)n * c, 256), 8 * num_sms()), 256, 0, stream>>>(labels, n, c, oh.get());
  count_launch();
  FPLS_LAUNCH("one_hot");
  GemmArgs g;
  g.M = a;
  g.N = a;
  g.K = n;
  g.A = scores;
  g.lda = lds;
  g.trans_a = true;
  g.B = scores;
  g.ldb = lds;
  g.C = gram.get();
  g.ldc = a;
  g.splits = gemm_pick_splits(a, a, n);
  DeviceArray<double> split_buf;
  if (g.splits > 1) {
    split_buf.allocate((size_t)g.splits * a * a, stream);
    g.C = split_buf.get();
    g.split_stride = (long)a * a;
  }
  gemm_f64(g, stream);
  if (g.splits > 1)
    FPLS_CHECK(cudaMemcpyAsync(gram.get(), split_buf.get(), sizeof(double) * a * a,
                               cudaMemcpyDeviceToDevice, stream));
  GemmArgs h = g;
  h.M = c;
  h.N = a;
  h.A = oh.get();
  h.lda = n;
  h.splits = gemm_pick_splits(c, a, n);
  h.C = sums.get();
  h.ldc = c;
  DeviceArray<double> split_buf2;
  if (h.splits > 1) {
    split_buf2.allocate((size_t)h.splits * c * a, stream);
    h.C = split_buf2.get();
    h.split_stride = (long)c * a;
  }
  h.split_stride = h.splits > 1 ? (long)c * a : 0;
  gemm_f64(h, stream);
  if (h.splits > 1)
    FPLS_CHECK(cudaMemcpyAsync(sums.get(), split_buf2.get(), sizeof(double) * c * a,
                               cudaMemcpyDeviceToDevice, stream));
  prefixes.clear();
}

const LdaState::Prefix& LdaState::prefix(int k, cudaStream_t stream) {
  require(k >= 1 && k <= a, "invalid LDA prefix");
  for (auto& pr : prefixes)
    if (pr.k == k) return pr;
  prefixes.emplace_back();
  Prefix& pr = prefixes.back();
  pr.k = k;
  pr.linear.allocate((size_t)c * k, stream);
  pr.constants.allocate(c + 1, stream);
  const size_t smem = (2 * (size_t)k * k + (size_t)c * k + k) * sizeof(double);
  if (smem > 48 * 1024)
    FPLS_CHECK(cudaFuncSetAttribute(lda_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  lda_finalize<<<1, 256, smem, stream>>>(gram.get(), a, sums.get(), c,
                                         counts_dev.get(), n, k,
                                         pr.linear.get(), pr.constants.get(),
                                         pr.constants.get() + c, flag);
  count_launch();
  FPLS_LAUNCH("lda_finalize");
  return pr;
}

void LdaState::discriminants(const double* scores, int rows, long lds, int k,
                             double* out, long ldo, cudaStream_t stream) {
  const Prefix& pr = prefix(k, stream);
  const long total = (long)rows * c;
  fill_constants<<<(unsigned)std::min<long>((total + 255) / 256, 8L * num_sms()), 256, 0, stream>>>(
      out, rows, c, ldo, pr.constants.get());
  count_launch();
  FPLS_LAUNCH("fill_constants");
  GemmArgs g;
  g.M = rows;
  g.N = c;
  g.K = k;
  g.A = scores;
  g.lda = lds;
  g.B = pr.linear.get();  // c x k: op(B) = linear^T (k x c)
  g.ldb = c;
  g.trans_b = true;
  g.C = out;
  g.ldc = ldo;
  g.beta = 1.0;
  gemm_f64(g, stream);
}

}  // namespace fpls
