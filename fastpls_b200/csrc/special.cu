// OPLS and nonlinear kernel PLS on the device (FP64), both feeding the
// SIMPLS engine of fit.cu.
//
// OPLS (reference: src/cuda_resident_special.cuh:155-381; CPU
// inst/include/fastpls/core/opls.hpp:120-290): on the standardised FP64 copy
// Xf of X, each orthogonal filter takes the dominant left singular vector w of
// Xf^T Yc, t = Xf w, p = Xf^T t / t't, w_o = normalise(p - (w'p / w'w) w),
// t_o = Xf w_o, p_o = Xf^T t_o / t_o't_o, then deflates Xf -= t_o p_o^T. The
// predictive SIMPLS model is fitted on the filtered Xf and its weights are
// folded back through the filters (R_eff = R - w_o (R^T p_o)^T, last filter
// first), so new rows are projected from their standardised values with
// R_eff and every prediction path of the handle applies unchanged.
//
// Kernel PLS (reference: src/cuda_resident_special.cuh:383-543; CPU
// kernels.hpp, kernelpls.hpp:85-196): K = phi(Xs Xs^T) on the standardised
// rows (RBF exp(-gamma ||xi - xj||^2) or polynomial (gamma xi.xj + c)^d), the
// n x n Gram formed on the FP64 tensor path (lower tiles + mirror), double
// centred with its column means and grand mean, then SIMPLS on K (p := n).
// New rows use the same transform against the training rows and the training
// centring (row means of the new block, training column means, grand mean).
#include "kernels.cuh"
#include "model.cuh"
#include "reduce.cuh"

#include <algorithm>
#include <cmath>

namespace fpls {

namespace {

constexpr int TB = 256;

template <class T>
__global__ void standardize_f64(const T* __restrict__ X, int n, int p, long ld,
                                const double* __restrict__ mean,
                                const double* __restrict__ scale, double* out) {
  const long total = (long)n * p;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total;
       k += (long)gridDim.x * blockDim.x) {
    const int i = (int)(k % n);
    const long j = k / n;
    out[k] = (as_f64(X[i + j * ld]) - mean[j]) / scale[j];
  }
}

// dots[k] over len of a*b (last-block reduce into out[0])
__global__ void dot_kernel(const double* __restrict__ a,
                           const double* __restrict__ b, int len,
                           double* partial, unsigned* counter, double* out) {
  __shared__ double scratch[32];
  __shared__ double v[1];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
    s = fma(a[i], b[i], s);
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) v[0] = s;
  __syncthreads();
  last_block_reduce(v, 1, partial, counter, out);
}

// y[i] = (y[i] - coef * x[i]) * mul, coef = num/den (device scalars), mul = 1/sqrt(norm2) or 1/norm2
__global__ void scale_vec(double* y, int len, const double* by, int mode, int* flag) {
  const double d = by[0];
  const bool ok = d > 0.0 && isfinite(d);
  if (!ok && blockIdx.x == 0 && threadIdx.x == 0) flag_error(flag, 1);
  const double f = ok ? (mode == 0 ? 1.0 / sqrt(d) : 1.0 / d) : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) y[i] *= f;
}

// wo = p - (w.p / w.w) w
__global__ void opls_orthogonal(const double* __restrict__ p,
                                const double* __restrict__ w, int len,
                                const double* wp, const double* ww, double* wo,
                                int* flag) {
  const bool ok = ww[0] > 0.0 && isfinite(ww[0]);
  if (!ok && blockIdx.x == 0 && threadIdx.x == 0) flag_error(flag, 1);
  const double proj = ok ? wp[0] / ww[0] : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
    wo[i] = p[i] - proj * w[i];
}

// X (n x p) -= t p^T
__global__ void rank1_subtract(double* X, int n, int p, const double* __restrict__ t,
                               const double* __restrict__ pv) {
  const long total = (long)n * p;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total;
       k += (long)gridDim.x * blockDim.x) {
    const int i = (int)(k % n);
    const long j = k / n;
    X[k] = fma(-t[i], pv[j], X[k]);
  }
}

// R (fp x a) -= w (R^T p)^T, one block per column of R
__global__ void fold_filter(double* R, int fp, int a, const double* __restrict__ w,
                            const double* __restrict__ pv) {
  __shared__ double scratch[32];
  for (int c = blockIdx.x; c < a; c += gridDim.x) {
    double s = 0.0;
    for (int j = threadIdx.x; j < fp; j += blockDim.x) s = fma(R[j + (long)c * fp], pv[j], s);
    s = block_sum(s, scratch);
    for (int j = threadIdx.x; j < fp; j += blockDim.x) R[j + (long)c * fp] = fma(-w[j], s, R[j + (long)c * fp]);
  }
}

__global__ void row_sqnorms(const double* __restrict__ X, int n, int p, double* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < p; ++j) {
      const double v = X[i + (long)j * n];
      s = fma(v, v, s);
    }
    out[i] = s;
  }
}

__global__ void kernel_transform(double* K, int rows, int cols, long ld, int kind,
                                 double gamma, int degree, double coef0,
                                 const double* __restrict__ left,
                                 const double* __restrict__ right) {
  const long total = (long)rows * cols;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total;
       k += (long)gridDim.x * blockDim.x) {
    const int i = (int)(k % rows);
    const long j = k / rows;
    double* e = K + i + j * ld;
    const double dot = *e;
    if (kind == 2) {
      double d = left[i] + right[j] - 2.0 * dot;
      if (d < 0.0) d = 0.0;
      *e = exp(-gamma * d);
    } else {
      const double base = fma(gamma, dot, coef0);
      double v = 1.0;
      for (int q = 0; q < degree; ++q) v *= base;
      *e = v;
    }
  }
}

// mean of each column (block per column)
__global__ void col_means(const double* __restrict__ K, int rows, int cols, long ld,
                          double* out) {
  __shared__ double scratch[32];
  for (int j = blockIdx.x; j < cols; j += gridDim.x) {
    double s = 0.0;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) s += K[i + (long)j * ld];
    s = block_sum(s, scratch);
    if (threadIdx.x == 0) out[j] = s / rows;
  }
}

// mean of each row (thread per row, coalesced over rows)
__global__ void row_means_kernel(const double* __restrict__ K, int rows, int cols,
                                 long ld, double* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < cols; ++j) s += K[i + (long)j * ld];
    out[i] = s / cols;
  }
}

__global__ void grand_mean(const double* __restrict__ m, int len, double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < len; i += blockDim.x) s += m[i];
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) out[0] = s / len;
}

// K -= rmean[i] + cmean[j] - grand
__global__ void double_center(double* K, int rows, int cols, long ld,
                              const double* __restrict__ rmean,
                              const double* __restrict__ cmean,
                              const double* __restrict__ grand) {
  const double g = grand[0];
  const long total = (long)rows * cols;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total;
       k += (long)gridDim.x * blockDim.x) {
    const int i = (int)(k % rows);
    const long j = k / rows;
    K[i + j * ld] -= rmean[i] + cmean[j] - g;
  }
}

unsigned grid_for(long total) {
  return (unsigned)std::min<long>((total + TB - 1) / TB, 16L * num_sms());
}

// Standardisation statistics of X (sum, sumsq -> mean, scale) with the same
// rules as the linear fits.
__global__ void stats_from_moments(const double* __restrict__ sum,
                                   const double* __restrict__ sumsq, int n,
                                   int p, int scaling, double* mean,
                                   double* scale) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x) {
    const double mu = scaling != 3 ? sum[j] / n : 0.0;
    double sd = 1.0;
    if (scaling == 2) {
      sd = sqrt(fmax(0.0, sumsq[j] - n * mu * mu) / (double)max(n - 1, 1));
      if (!isfinite(sd) || sd <= 0.0) sd = 1.0;
    }
    mean[j] = mu;
    scale[j] = sd;
  }
}

template <class T>
void standardized_copy(const T* X, int n, int p, long ld, int scaling,
                       DeviceArray<double>& mean, DeviceArray<double>& scale,
                       DeviceArray<double>& xs, Workspace& ws, cudaStream_t s) {
  DeviceArray<double> mom((size_t)2 * p, s);
  column_moments<T>(X, n, p, ld, nullptr, 0, mom.get(), mom.get() + p, nullptr, ws.stream_partial, s);
  mean.allocate(p, s);
  scale.allocate(p, s);
  stats_from_moments<<<grid_for(p), TB, 0, s>>>(mom.get(), mom.get() + p, n, p, scaling, mean.get(), scale.get());
  xs.allocate((size_t)n * p, s);
  standardize_f64<T><<<grid_for((long)n * p), TB, 0, s>>>(X, n, p, ld, mean.get(), scale.get(), xs.get());
  count_launch(2);
  FPLS_LAUNCH("standardized_copy");
}

}  // namespace

template <class T>
void fit_opls(const T* X, int n, int p, long ld, const double* Yc,
              const double* ycsum, int m, int components, int scaling,
              int north, DeviceModel& model, Workspace& ws,
              DeviceArray<double>& design, cudaStream_t s) {
  require(north >= 0, "invalid resident CUDA OPLS input");
  ws.ensure(n, p, m, components, s);
  DeviceArray<double> mean, scale;
  standardized_copy<T>(X, n, p, ld, scaling, mean, scale, design, ws, s);
  double* xf = design.get();
  const int f = std::max(north, 0);
  DeviceArray<double> Wo((size_t)p * std::max(f, 1), s), Po((size_t)p * std::max(f, 1), s);
  DeviceArray<double> S((size_t)p * m, s), w(p, s), pv(p, s), t(n, s), sc(8, s);
  double* gpk = ws.small.get() + 8 + kMaxResponses;
  double* zs = ws.small.get() + 8;
  unsigned* ctr = ws.counters.get() + 16;
  double* part = ws.block_partial.get();
  const unsigned gd = std::min<unsigned>(ceil_div(std::max(n, p), TB), 2 * num_sms());
  for (int c = 0; c < f; ++c) {
    // dominant left direction of Xf^T Yc
    xtv_product<double>(xf, n, p, n, Yc, n, m, S.get(), p, ws.stream_partial, s);
    gram_of_columns(S.get(), p, m, gpk, ws, s);
    dominant_direction(S.get(), p, m, gpk, zs, w.get(), ws, s);
    // t = Xf w ; p = Xf^T t / t't ; wo = normalise(p - (w'p / w'w) w)
    xr_product<double>(xf, n, p, n, w.get(), p, 1, nullptr, t.get(), n, ws.stream_partial, s);
    xtv_product<double>(xf, n, p, n, t.get(), n, 1, pv.get(), p, ws.stream_partial, s);
    dot_kernel<<<gd, TB, 0, s>>>(t.get(), t.get(), n, part, ctr, sc.get());
    scale_vec<<<gd, TB, 0, s>>>(pv.get(), p, sc.get(), 1, ws.flag.get());
    dot_kernel<<<gd, TB, 0, s>>>(w.get(), pv.get(), p, part, ctr + 1, sc.get() + 1);
    dot_kernel<<<gd, TB, 0, s>>>(w.get(), w.get(), p, part, ctr + 2, sc.get() + 2);
    double* wo = Wo.get() + (size_t)c * p;
    opls_orthogonal<<<gd, TB, 0, s>>>(pv.get(), w.get(), p, sc.get() + 1, sc.get() + 2, wo, ws.flag.get());
    dot_kernel<<<gd, TB, 0, s>>>(wo, wo, p, part, ctr + 3, sc.get() + 3);
    scale_vec<<<gd, TB, 0, s>>>(wo, p, sc.get() + 3, 0, ws.flag.get());
    count_launch(7);
    FPLS_LAUNCH("opls filter direction");
    // t_o = Xf wo ; p_o = Xf^T t_o / t_o't_o ; Xf -= t_o p_o^T
    double* po = Po.get() + (size_t)c * p;
    xr_product<double>(xf, n, p, n, wo, p, 1, nullptr, t.get(), n, ws.stream_partial, s);
    xtv_product<double>(xf, n, p, n, t.get(), n, 1, po, p, ws.stream_partial, s);
    dot_kernel<<<gd, TB, 0, s>>>(t.get(), t.get(), n, part, ctr + 4, sc.get() + 4);
    scale_vec<<<gd, TB, 0, s>>>(po, p, sc.get() + 4, 1, ws.flag.get());
    rank1_subtract<<<grid_for((long)n * p), TB, 0, s>>>(xf, n, p, t.get(), po);
    count_launch(3);
    FPLS_LAUNCH("opls filter deflation");
  }
  // predictive SIMPLS on the filtered, already standardised predictors
  fit_simpls<double>(xf, n, p, n, Yc, ycsum, m, components, 3, model, ws, s,
                     simpls_block_size(n, p, m, components, model.classification,
                                       std::is_same<T, float>::value));
  for (int c = f - 1; c >= 0; --c) {
    fold_filter<<<std::min(components, 4 * num_sms()), TB, 0, s>>>(
        model.R.get(), p, components, Wo.get() + (size_t)c * p, Po.get() + (size_t)c * p);
    count_launch();
    FPLS_LAUNCH("fold_filter");
  }
  model.mean = std::move(mean);
  model.scale = std::move(scale);
  model.method = kOpls;
}

template <class T>
void fit_kernelpls(const T* X, int n, int p, long ld, const double* Yc,
                   const double* ycsum, int m, int components, int scaling,
                   int kind, double gamma, int degree, double coef0,
                   DeviceModel& model, Workspace& ws, DeviceArray<double>& design,
                   cudaStream_t s) {
  require((kind == 2 || kind == 3) && degree >= 1 && gamma > 0.0 && std::isfinite(gamma) &&
              std::isfinite(coef0),
          "invalid resident CUDA nonlinear kernel PLS dimensions or controls");
  require(components <= n - 1, "invalid resident CUDA nonlinear kernel PLS dimensions or controls");
  size_t free_b = 0, total_b = 0;
  FPLS_CHECK(cudaMemGetInfo(&free_b, &total_b));
  if ((double)n * n * 8.0 + (double)n * p * 8.0 > 0.6 * (double)free_b)
    throw std::runtime_error(
        "nonlinear kernel PLS requires an n-by-n Gram matrix that exceeds the guarded CUDA memory budget");
  ws.ensure(n, std::max(n, p), m, components, s);
  DeviceArray<double> mean, scale;
  standardized_copy<T>(X, n, p, ld, scaling, mean, scale, model.reference, ws, s);
  model.ref_norms.allocate(n, s);
  row_sqnorms<<<grid_for(n), TB, 0, s>>>(model.reference.get(), n, p, model.ref_norms.get());
  count_launch();
  design.allocate((size_t)n * n, s);
  GemmArgs g;
  g.M = n;
  g.N = n;
  g.K = p;
  g.A = model.reference.get();
  g.lda = n;
  g.B = model.reference.get();
  g.ldb = n;
  g.trans_b = true;
  g.C = design.get();
  g.ldc = n;
  g.lower = gemm_mma_supported(g);
  gemm_f64(g, s);
  kernel_transform<<<grid_for((long)n * n), TB, 0, s>>>(design.get(), n, n, n, kind, gamma, degree, coef0,
                                                         model.ref_norms.get(), model.ref_norms.get());
  model.kcol_means.allocate(n + 1, s);
  col_means<<<std::min(n, 8 * num_sms()), TB, 0, s>>>(design.get(), n, n, n, model.kcol_means.get());
  grand_mean<<<1, TB, 0, s>>>(model.kcol_means.get(), n, model.kcol_means.get() + n);
  double_center<<<grid_for((long)n * n), TB, 0, s>>>(design.get(), n, n, n, model.kcol_means.get(),
                                                      model.kcol_means.get(), model.kcol_means.get() + n);
  count_launch(4);
  FPLS_LAUNCH("kernel gram");
  fit_simpls<double>(design.get(), n, n, n, Yc, ycsum, m, components, 3, model, ws, s,
                     simpls_block_size(n, n, m, components, model.classification,
                                       std::is_same<T, float>::value));
  model.in_mean = std::move(mean);
  model.in_scale = std::move(scale);
  model.kernel_kind = kind;
  model.gamma = gamma;
  model.degree = degree;
  model.coef0 = coef0;
  model.method = kKernelPls;
  model.in_p = p;
}

template <class T>
void kernel_scores(const DeviceModel& model, const T* X, int rows, long ld, int k,
                   double* out, long ldo, Workspace& ws, cudaStream_t s) {
  const int n = model.n, p = model.in_p;
  size_t free_b = 0, total_b = 0;
  FPLS_CHECK(cudaMemGetInfo(&free_b, &total_b));
  if ((double)rows * n * 8.0 + (double)rows * p * 8.0 > 0.6 * (double)free_b)
    throw std::runtime_error(
        "nonlinear kernel prediction exceeds the guarded CUDA workspace; reduce the prediction block size or training sample count");
  DeviceArray<double> xs((size_t)rows * p, s), norms(rows, s), kt((size_t)rows * n, s), rm(rows, s);
  standardize_f64<T><<<grid_for((long)rows * p), TB, 0, s>>>(X, rows, p, ld, model.in_mean.get(),
                                                              model.in_scale.get(), xs.get());
  row_sqnorms<<<grid_for(rows), TB, 0, s>>>(xs.get(), rows, p, norms.get());
  count_launch(2);
  GemmArgs g;
  g.M = rows;
  g.N = n;
  g.K = p;
  g.A = xs.get();
  g.lda = rows;
  g.B = model.reference.get();
  g.ldb = n;
  g.trans_b = true;
  g.C = kt.get();
  g.ldc = rows;
  gemm_f64(g, s);
  kernel_transform<<<grid_for((long)rows * n), TB, 0, s>>>(kt.get(), rows, n, rows, model.kernel_kind,
                                                            model.gamma, model.degree, model.coef0,
                                                            norms.get(), model.ref_norms.get());
  row_means_kernel<<<grid_for(rows), TB, 0, s>>>(kt.get(), rows, n, rows, rm.get());
  double_center<<<grid_for((long)rows * n), TB, 0, s>>>(kt.get(), rows, n, rows, rm.get(),
                                                         model.kcol_means.get(), model.kcol_means.get() + n);
  count_launch(3);
  FPLS_LAUNCH("kernel test block");
  // scores = Kc R (inner design has zero mean / unit scale)
  project_rows<double>(model, kt.get(), rows, rows, k, out, ldo, ws, s);
}

#define FPLS_INSTANTIATE(T)                                                      \
  template void fit_opls<T>(const T*, int, int, long, const double*,            \
                            const double*, int, int, int, int, DeviceModel&,    \
                            Workspace&, DeviceArray<double>&, cudaStream_t);    \
  template void fit_kernelpls<T>(const T*, int, int, long, const double*,       \
                                 const double*, int, int, int, int, double, int, \
                                 double, DeviceModel&, Workspace&,              \
                                 DeviceArray<double>&, cudaStream_t);           \
  template void kernel_scores<T>(const DeviceModel&, const T*, int, long, int,  \
                                 double*, long, Workspace&, cudaStream_t);
FPLS_INSTANTIATE(float)
FPLS_INSTANTIATE(double)
FPLS_INSTANTIATE(bf16)
#undef FPLS_INSTANTIATE

}  // namespace fpls
