// Single-fit SIMPLS on the device (p-space, FP64 arithmetic, raw X).
//
// Reference algorithm: fit_simpls_preprocessed
// (inst/include/fastpls/core/simpls.hpp:479-763) and the resident CUDA
// component step (src/cuda_resident_component.cuh:94-130). Per component:
//   r = dominant left singular vector of the deflated cross-product S,
//   t = Xs r, r,t /= ||t||, p = Xs^T t, q = S0^T r,
//   v = p - V (V^T p), v /= ||v||, S -= v (v^T S).
//
// B200 design:
//  * X stays raw in HBM (FP32 or FP64). Centring and scaling are folded into
//    the two products, t = X (r / scale) - (mean . r / scale) and
//    p = (X^T t - mean * sum(t)) / scale, so X is never rewritten and each
//    component reads it exactly twice (stream.cu).
//  * The direction comes from the m x m Gram G = S^T S, recomputed from the
//    deflated S each component (no downdate drift) and diagonalised by
//    Jacobi in one block: r = S z / sqrt(lambda). The span of the
//    reference's randomized sketch equals the full response space in every
//    supported configuration, so this is the same dominant direction.
//  * Every p-length step is one kernel over 256-row blocks of S/V whose
//    cross-block sums finish in the last block to arrive (reduce.cuh):
//    deterministic, no atomics on data, no spin-waits.
#include "kernels.cuh"
#include "model.cuh"
#include "persistent.cuh"
#include "reduce.cuh"
#include "small.cuh"

#include <algorithm>
#include <memory>

namespace fpls {

namespace {

constexpr int TB = 256;

template <class T>
__global__ void center_dense(const T* __restrict__ Y, int n, int m,
                             double* __restrict__ Yc, double* ymean,
                             double* ycsum, int* flag) {
  __shared__ double scratch[32];
  const int c = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double y = as_f64(Y[i + (long)c * n]);
    if (!isfinite(y)) flag_error(flag, 3);
    s += y;
  }
  const double mu = block_sum(s, scratch) / n;
  double r = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = as_f64(Y[i + (long)c * n]) - mu;
    Yc[i + (long)c * n] = v;
    r += v;
  }
  r = block_sum(r, scratch);
  if (threadIdx.x == 0) {
    ymean[c] = mu;
    ycsum[c] = r;
  }
}

__global__ void center_labels(const int* __restrict__ labels, int n, int m,
                              double* __restrict__ Yc, double* ymean,
                              double* ycsum, int* flag) {
  __shared__ double scratch[32];
  const int c = blockIdx.x;
  double cnt = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int l = labels[i];
    if (l < 1 || l > m) flag_error(flag, 2);
    cnt += (l == c + 1) ? 1.0 : 0.0;
  }
  const double prior = block_sum(cnt, scratch) / n;
  double r = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = (labels[i] == c + 1 ? 1.0 : 0.0) - prior;
    Yc[i + (long)c * n] = v;
    r += v;
  }
  r = block_sum(r, scratch);
  if (threadIdx.x == 0) {
    ymean[c] = prior;
    ycsum[c] = r;
  }
}

// mean / scale per column (supervised.hpp:53-90) and the scaled centred
// cross-product S = D^-1 (X^T Yc - mean * colsum(Yc)).
__global__ void finish_moments(const double* __restrict__ sum,
                               const double* __restrict__ sumsq,
                               const double* __restrict__ cross,
                               const double* __restrict__ ycsum, int n, int p,
                               int m, int scaling, double* mean, double* scale,
                               double* S, double* S0, int* flag) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p;
       j += gridDim.x * blockDim.x) {
    const double mu = scaling != 3 ? sum[j] / n : 0.0;
    double sd = 1.0;
    if (scaling == 2) {
      const double cs = fmax(0.0, sumsq[j] - n * mu * mu);
      sd = sqrt(cs / (double)max(n - 1, 1));
      if (!isfinite(sd) || sd <= 0.0) sd = 1.0;
    }
    if (!isfinite(sum[j]) || !isfinite(sumsq[j])) flag_error(flag, 3);
    mean[j] = mu;
    scale[j] = sd;
    for (int c = 0; c < m; ++c) {
      const double s = (cross[j + (long)c * p] - mu * ycsum[c]) / sd;
      S[j + (long)c * p] = s;
      S0[j + (long)c * p] = s;
    }
  }
}

// Unpack the packed lower-triangular Gram, diagonalise, emit z / sqrt(lambda).
// The `count` dominant eigenpairs of the m x m right Gram (packed lower
// triangle), by decreasing eigenvalue (ties: lower index first):
// zs[k + j m] = z_j / sqrt(lambda_j), sign fixed so the largest-magnitude
// entry of z_j is positive; lambda_out = lambda_0.
__global__ void direction_kernel(const double* __restrict__ gpk, int m,
                                 double* zs, double* lambda_out, int* flag, int count) {
  extern __shared__ double sm[];
  double* A = sm;
  double* E = sm + m * m;
  for (int c = threadIdx.x; c < m; c += blockDim.x)
    for (int d = 0; d <= c; ++d) {
      const double v = gpk[c * (c + 1) / 2 + d];
      A[c + d * m] = v;
      A[d + c * m] = v;
    }
  __syncthreads();
  if (count == 1 && m <= kDominantMaxOrder) {
    // one direction: the dominant pair alone (repeated squaring)
    double* C = E + m * m;      // m^2 + 1
    double* v = C + m * m + 1;  // m + 1
    double lam = 0.0;
    const bool found = dominant_pair(A, E, C, v, m, lam);
    if (threadIdx.x == 0) {
      const bool ok = found && lam > 0.0 && isfinite(lam);
      if (!ok) flag_error(flag, 1);
      const double inv = ok ? 1.0 / sqrt(lam) : 0.0;
      int arg = 0;
      if (found)
        for (int k = 1; k < m; ++k)
          if (fabs(v[k]) > fabs(v[arg])) arg = k;
      const double sgn = found && v[arg] < 0.0 ? -1.0 : 1.0;
      for (int k = 0; k < m; ++k) zs[k] = found ? sgn * v[k] * inv : 0.0;
      if (lambda_out) *lambda_out = found ? lam : 0.0;
    }
    return;
  }
  jacobi_eigen(A, E, m);
  __syncthreads();
  if (threadIdx.x == 0) {
    double inv0 = 0.0;
    for (int j = 0; j < count; ++j) {
      int best = -1;
      for (int k = 0; k < m; ++k)
        if (best < 0 || A[k + k * m] > A[best + best * m]) best = k;
      const double lam = A[best + best * m];
      A[best + best * m] = -INFINITY;  // taken (A is scratch after the solve)
      const bool ok = lam > 0.0 && isfinite(lam);
      // The leading pair must exist (S not zero). A later candidate of a
      // block wider than the rank of S (a block of q classes, rank q - 1)
      // has a numerically zero eigenvalue: it takes the leading pair's scale
      // (R and T do not depend on the scale of r), as the reference's sketch
      // yields some unit direction there instead of failing.
      if (!ok && j == 0) flag_error(flag, 1);
      const double inv = ok ? 1.0 / sqrt(lam) : inv0;
      if (j == 0) inv0 = inv;
      // deterministic sign: largest-magnitude entry of z positive
      int arg = 0;
      for (int k = 1; k < m; ++k)
        if (fabs(E[k + best * m]) > fabs(E[arg + best * m])) arg = k;
      const double sgn = E[arg + best * m] < 0.0 ? -1.0 : 1.0;
      for (int k = 0; k < m; ++k) zs[k + j * m] = sgn * E[k + best * m] * inv;
      if (lambda_out && j == 0) *lambda_out = lam;
    }
  }
}

// r = S zs ; rt = r / scale ; scal[0] = mean . rt
__global__ void rvec_kernel(const double* __restrict__ S, int p, int m,
                            const double* __restrict__ zs,
                            const double* __restrict__ mean,
                            const double* __restrict__ scale, double* r,
                            double* rt, double* partial, unsigned* counter,
                            double* scal) {
  __shared__ double scratch[32];
  __shared__ double vals[1];
  double acc = 0.0;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p) {
    double v = 0.0;
    for (int c = 0; c < m; ++c) v = fma(S[j + (long)c * p], zs[c], v);
    const double w = v / scale[j];
    r[j] = v;
    rt[j] = w;
    acc = mean[j] * w;
  }
  const double s = block_sum(acc, scratch);
  if (threadIdx.x == 0) vals[0] = s;
  __syncthreads();
  last_block_reduce(vals, 1, partial, counter, scal);
}

// scal[1] = sum t^2, scal[2] = sum t
__global__ void tstats_kernel(const double* __restrict__ t, int n,
                              double* partial, unsigned* counter,
                              double* scal) {
  __shared__ double scratch[32];
  __shared__ double vals[2];
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    a = fma(t[i], t[i], a);
    b += t[i];
  }
  a = block_sum(a, scratch);
  b = block_sum(b, scratch);
  if (threadIdx.x == 0) {
    vals[0] = a;
    vals[1] = b;
  }
  __syncthreads();
  last_block_reduce(vals, 2, partial, counter, scal + 1);
}

// Warp-strided block reduction of `count` dot products over the block's row
// range: out[k] = sum_{j in block} col_k[j] * w[j] (w in shared memory).
__device__ inline void block_dots(const double* __restrict__ M, long ldm,
                                  int j0, int rows, const double* w, int count,
                                  double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  for (int k = warp; k < count; k += warps) {
    double acc = 0.0;
    for (int j = lane; j < rows; j += 32) acc = fma(M[j0 + j + (long)k * ldm], w[j], acc);
    acc = warp_sum(acc);
    if (lane == 0) out[k] = acc;
  }
}

// p = (praw - mean * sum t) / (scale * ||t||) ; R[:,a] = r / ||t||
// out (last block): h = V^T p (a_cur), q = S0^T R[:,a] (m)
// When `loading` is given (cached-Gram route) p = loading / ||t|| directly.
__global__ void tail1_kernel(const double* __restrict__ praw,
                             const double* __restrict__ mean,
                             const double* __restrict__ scale,
                             const double* __restrict__ scal,
                             const double* __restrict__ r,
                             const double* __restrict__ S0,
                             const double* __restrict__ V, int p, int m,
                             int a_cur, double* pvec, double* Rcol,
                             double* partial, unsigned* counter, double* hq,
                             int* flag, const double* __restrict__ loading = nullptr) {
  extern __shared__ double sm[];
  double* ps = sm;            // TB
  double* rs = sm + TB;       // TB
  double* vals = sm + 2 * TB; // a_cur + m
  const int j0 = blockIdx.x * TB;
  const int rows = min(TB, p - j0);
  const double tn = sqrt(scal[1]);
  if (!(tn > 0.0) || !isfinite(tn)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) flag_error(flag, 1);
  }
  const double inv = (tn > 0.0 && isfinite(tn)) ? 1.0 / tn : 0.0;
  const int t = threadIdx.x;
  if (t < rows) {
    const int j = j0 + t;
    const double pj = loading ? loading[j] * inv : (praw[j] - mean[j] * scal[2]) / scale[j] * inv;
    const double rj = r[j] * inv;
    pvec[j] = pj;
    Rcol[j] = rj;
    ps[t] = pj;
    rs[t] = rj;
  }
  __syncthreads();
  block_dots(V, p, j0, rows, ps, a_cur, vals);
  block_dots(S0, p, j0, rows, rs, m, vals + a_cur);
  __syncthreads();
  last_block_reduce(vals, a_cur + m, partial, counter, hq);
}

// v = p - V h ; out (last block): [v.v, S^T v (m)]
__global__ void tail2_kernel(const double* __restrict__ pvec,
                             const double* __restrict__ V,
                             const double* __restrict__ hq,
                             const double* __restrict__ S, int p, int m,
                             int a_cur, double* v, double* partial,
                             unsigned* counter, double* vr) {
  extern __shared__ double sm[];
  double* vs = sm;             // TB
  double* vals = sm + TB;      // 1 + m
  __shared__ double scratch[32];
  const int j0 = blockIdx.x * TB;
  const int rows = min(TB, p - j0);
  const int t = threadIdx.x;
  double vj = 0.0;
  if (t < rows) {
    const int j = j0 + t;
    vj = pvec[j];
    for (int k = 0; k < a_cur; ++k) vj = fma(-V[j + (long)k * p], hq[k], vj);
    v[j] = vj;
    vs[t] = vj;
  }
  __syncthreads();
  const double vv = block_sum(vj * vj, scratch);
  block_dots(S, p, j0, rows, vs, m, vals + 1);
  if (threadIdx.x == 0) vals[0] = vv;
  __syncthreads();
  last_block_reduce(vals, 1 + m, partial, counter, vr);
}

// V[:,a] = v / ||v|| ; S -= V[:,a] (row / ||v||) ; G partials of updated S
// (packed lower triangle) reduced by the last block into gpk.
// When `update` is false only the Gram of S is formed.
__global__ void tail3_kernel(const double* __restrict__ v,
                             const double* __restrict__ vr, double* S, int p,
                             int m, double* Vcol, bool update, double* partial,
                             unsigned* counter, double* gpk, int* flag) {
  extern __shared__ double sm[];
  const int jb = blockDim.x;
  double* ss = sm;                 // jb x m
  double* vals = sm + jb * m;      // m(m+1)/2
  const int j0 = blockIdx.x * jb;
  const int rows = min(jb, p - j0);
  const int t = threadIdx.x;
  double vn = 1.0;
  if (update) {
    vn = sqrt(vr[0]);
    if (!(vn > 0.0) || !isfinite(vn)) {
      if (blockIdx.x == 0 && t == 0) flag_error(flag, 1);
      vn = 0.0;
    }
  }
  const double inv = vn > 0.0 ? 1.0 / vn : 0.0;
  if (t < rows) {
    const int j = j0 + t;
    const double vj = update ? v[j] * inv : 0.0;
    if (update) Vcol[j] = vj;
    for (int c = 0; c < m; ++c) {
      double s = S[j + (long)c * p];
      if (update) {
        s = fma(-vj, vr[1 + c] * inv, s);
        S[j + (long)c * p] = s;
      }
      ss[t + c * jb] = s;
    }
  }
  __syncthreads();
  const int pairs = m * (m + 1) / 2;
  const int lane = t & 31, warp = t >> 5, warps = jb >> 5;
  for (int k = warp; k < pairs; k += warps) {
    // k -> (c, d) with d <= c, k = c(c+1)/2 + d
    int c = (int)((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
    while (c * (c + 1) / 2 > k) --c;
    while ((c + 1) * (c + 2) / 2 <= k) ++c;
    const int d = k - c * (c + 1) / 2;
    double acc = 0.0;
    for (int j = lane; j < rows; j += 32) acc = fma(ss[j + c * jb], ss[j + d * jb], acc);
    acc = warp_sum(acc);
    if (lane == 0) vals[k] = acc;
  }
  __syncthreads();
  last_block_reduce(vals, pairs, partial, counter, gpk);
}

// T[:,a] /= ||t|| ; Q[:,a] = q
__global__ void finish_component(double* Tcol, int n, const double* scal,
                                 const double* hq, int a_cur, int m,
                                 double* Qcol) {
  const double tn = sqrt(scal[1]);
  const double inv = (tn > 0.0 && isfinite(tn)) ? 1.0 / tn : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    Tcol[i] *= inv;
  if (blockIdx.x == 0)
    for (int c = threadIdx.x; c < m; c += blockDim.x) Qcol[c] = hq[a_cur + c];
}

// Rs = R / scale (p x k), roff[c] = mean . Rs[:,c]
__global__ void scaled_weights(const double* __restrict__ R, int p, int k,
                               const double* __restrict__ mean,
                               const double* __restrict__ scale, double* Rs,
                               double* roff) {
  __shared__ double scratch[32];
  const int c = blockIdx.x;
  double acc = 0.0;
  for (int j = threadIdx.x; j < p; j += blockDim.x) {
    const double w = R[j + (long)c * p] / scale[j];
    Rs[j + (long)c * p] = w;
    acc = fma(mean[j], w, acc);
  }
  acc = block_sum(acc, scratch);
  if (threadIdx.x == 0) roff[c] = acc;
}

__global__ void fill_rows_mean(double* out, int rows, int m, long ldo,
                               const double* ymean) {
  const long total = (long)rows * m;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % rows), c = (int)(idx / rows);
    out[i + (long)c * ldo] = ymean[c];
  }
}

// Gs[j, k] = (G[j, k] - n mean_j mean_k) / (scale_j scale_k): the Gram of
// the standardised predictors from the raw X^T X.
__global__ void standardize_gram(double* G, int p, int n, const double* __restrict__ mean,
                                 const double* __restrict__ scale) {
  const long total = (long)p * p;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int j = (int)(idx % p), k = (int)(idx / p);
    G[idx] = (G[idx] - (double)n * mean[j] * mean[k]) / (scale[j] * scale[k]);
  }
}

// scal[1] = r . loading (= ||X_s r||^2), scal[2] = 0 (sum t unused on this route)
__global__ void gram_tstats(const double* __restrict__ r, const double* __restrict__ loading,
                            int p, double* partial, unsigned* counter, double* scal) {
  __shared__ double scratch[32];
  __shared__ double vals[2];
  double a = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x)
    a = fma(r[j], loading[j], a);
  a = block_sum(a, scratch);
  if (threadIdx.x == 0) {
    vals[0] = a;
    vals[1] = 0.0;
  }
  __syncthreads();
  last_block_reduce(vals, 2, partial, counter, scal + 1);
}

int tail3_block(int m) { return m <= 16 ? 256 : (m <= 32 ? 128 : 64); }

}  // namespace

void Workspace::ensure(int n, int p, int m, int a, cudaStream_t s) {
  const size_t blocks_p = ceil_div(std::max(p, 1), 64) + 8;
  const size_t width = std::max<size_t>(a + m + 2, (size_t)m * (m + 1) / 2 + 2);
  block_partial.reserve(blocks_p * width + 4096, s);
  if (!counters) {
    counters.allocate(64, s);
    counters.zero(s);
  }
  for (auto& v : vec_p) v.reserve(std::max(p, 1), s);
  for (auto& v : vec_n) v.reserve(std::max(n, 1), s);
  small.reserve(64 + 2 * (size_t)kMaxResponses * kMaxResponses + 4 * (size_t)std::max(a, 1) + m, s);
  if (!flag) {
    flag.allocate(1, s);
  }
}

void raise_on_flag(Workspace& ws, cudaStream_t stream, const char* message) {
  int bad = 0;
  FPLS_CHECK(cudaMemcpyAsync(&bad, ws.flag.get(), sizeof(int),
                             cudaMemcpyDeviceToHost, stream));
  FPLS_CHECK(cudaStreamSynchronize(stream));
  if (bad) throw std::runtime_error(message);
}

template <class T>
void prepare_responses(const T* Y, const int* labels, int n, int m, double* Yc,
                       double* ymean, double* ycsum, int* flag,
                       cudaStream_t stream) {
  if (labels) center_labels<<<m, TB, 0, stream>>>(labels, n, m, Yc, ymean, ycsum, flag);
  else center_dense<T><<<m, TB, 0, stream>>>(Y, n, m, Yc, ymean, ycsum, flag);
  count_launch();
  FPLS_LAUNCH("prepare_responses");
}

__global__ void s_times_z(const double* __restrict__ S, int p, int m,
                          const double* __restrict__ zs, double* w) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int c = 0; c < m; ++c) v = fma(S[j + (long)c * p], zs[c], v);
    w[j] = v;
  }
}

void dominant_direction(const double* S, int p, int m, const double* gpk,
                        double* zs, double* w, Workspace& ws, cudaStream_t s) {
  // A, B, C, v of the dominant pair (one direction), or A, E of the Jacobi sweeps
  const size_t smem_dir = (m <= kDominantMaxOrder ? 3 * (size_t)m * m + m + 2 : 2 * (size_t)m * m) * sizeof(double);
  if (smem_dir > 48 * 1024)
    FPLS_CHECK(cudaFuncSetAttribute(direction_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_dir));
  direction_kernel<<<1, jacobi_threads(m), smem_dir, s>>>(gpk, m, zs, nullptr, ws.flag.get(), 1);
  s_times_z<<<std::min<unsigned>(ceil_div(p, TB), 4 * num_sms()), TB, 0, s>>>(S, p, m, zs, w);
  count_launch(2);
  FPLS_LAUNCH("dominant_direction");
}

template <class T>
void compute_crossprod(const T* X, int n, int p, long ld, const double* Yc,
                       const double* ycsum, int m, int scaling,
                       DeviceModel& model, double* S, Workspace& ws,
                       cudaStream_t stream) {
  model.mean.allocate(p, stream);
  model.scale.allocate(p, stream);
  model.S0.allocate((size_t)p * m, stream);
  DeviceArray<double> moments((size_t)p * (2 + m), stream);
  double* sum = moments.get();
  double* sumsq = sum + p;
  double* cross = sumsq + p;
  if (model.label_view && m <= kClassMomentsMaxClasses)
    class_moments<T>(X, n, p, ld, model.label_view, m, model.ymean.get(), sum, sumsq, cross,
                     ws.stream_partial, stream);
  else
    column_moments<T>(X, n, p, ld, Yc, m, sum, sumsq, cross, ws.stream_partial, stream);
  const unsigned gp = std::min<unsigned>(ceil_div(p, TB), 8 * num_sms());
  finish_moments<<<gp, TB, 0, stream>>>(sum, sumsq, cross, ycsum, n, p, m,
                                        scaling, model.mean.get(),
                                        model.scale.get(), S,
                                        model.S0.get(), ws.flag.get());
  count_launch();
  FPLS_LAUNCH("finish_moments");
}

void gram_of_columns(double* S, int p, int m, double* gpk, Workspace& ws,
                     cudaStream_t stream) {
  const int jb3 = tail3_block(m);
  const unsigned g3 = ceil_div(p, jb3);
  const size_t smem3 = ((size_t)jb3 * m + (size_t)m * (m + 1) / 2) * sizeof(double);
  if (smem3 > 48 * 1024)
    FPLS_CHECK(cudaFuncSetAttribute(tail3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem3));
  tail3_kernel<<<g3, jb3, smem3, stream>>>(nullptr, nullptr, S, p, m, nullptr,
                                           false, ws.block_partial.get(),
                                           ws.counters.get() + 5, gpk,
                                           ws.flag.get());
  count_launch();
  FPLS_LAUNCH("gram_of_columns");
}

template <class T>
void fit_simpls(const T* X, int n, int p, long ld, const double* Yc,
                const double* ycsum, int m, int components, int scaling,
                DeviceModel& model, Workspace& ws, cudaStream_t stream, int block,
                bool gram_route) {
  require(m >= 1 && m <= kMaxResponses, "SIMPLS supports 1..112 responses or classes");
  const int a_max = components;
  ws.ensure(n, p, m, a_max, stream);
  model.method = kSimpls;
  model.n = n;
  model.p = p;
  model.feature_p = p;
  model.m = m;
  model.scaling = scaling;
  model.R.allocate((size_t)p * a_max, stream);
  model.Q.allocate((size_t)m * a_max, stream);
  model.V.allocate((size_t)p * a_max, stream);
  model.T.allocate((size_t)n * a_max, stream);
  DeviceArray<double> S((size_t)p * m, stream);
  compute_crossprod<T>(X, n, p, ld, Yc, ycsum, m, scaling, model, S.get(), ws, stream);

  double* sm = ws.small.get();
  double* scal = sm;            // [c, sum t^2, sum t, lambda]
  double* zs = sm + 8;          // m
  double* gpk = zs + kMaxResponses;                // m(m+1)/2
  double* hq = gpk + kMaxResponses * kMaxResponses; // a + m
  double* vr = hq + a_max + m + 4;                  // 1 + m
  double* r = ws.vec_p[0].get();
  double* rt = ws.vec_p[1].get();
  double* pvec = ws.vec_p[2].get();
  double* v = ws.vec_p[3].get();
  double* praw = ws.vec_p[4].get();
  unsigned* ctr = ws.counters.get();
  double* part = ws.block_partial.get();

  const int jb3 = tail3_block(m);
  const unsigned g3 = ceil_div(p, jb3);
  const size_t smem3 = ((size_t)jb3 * m + (size_t)m * (m + 1) / 2) * sizeof(double);
  const unsigned g1 = ceil_div(p, TB);
  // A, B, C, v of the dominant pair (one direction), or A, E of the Jacobi sweeps
  const size_t smem_dir = (m <= kDominantMaxOrder ? 3 * (size_t)m * m + m + 2 : 2 * (size_t)m * m) * sizeof(double);
  if (smem3 > 48 * 1024)
    FPLS_CHECK(cudaFuncSetAttribute(tail3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem3));
  if (smem_dir > 48 * 1024)
    FPLS_CHECK(cudaFuncSetAttribute(direction_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_dir));

  // cached-Gram route (FP32 / FP64 storage): Gs = X_s^T X_s once
  gram_route = gram_route && !std::is_same<T, bf16>::value;
  DeviceArray<double> Gs, loading;
  if (gram_route) {
    Gs.allocate((size_t)p * p, stream);
    loading.allocate(p, stream);
    GemmArgs g;
    g.M = p;
    g.N = p;
    g.K = n;
    g.A = X;
    g.lda = ld;
    g.trans_a = true;
    g.a_f32 = std::is_same<T, float>::value;
    g.B = X;
    g.ldb = ld;
    g.b_f32 = std::is_same<T, float>::value;
    g.C = Gs.get();
    g.ldc = p;
    gemm_f64(g, stream);
    const long total = (long)p * p;
    standardize_gram<<<(unsigned)std::min<long>((total + 255) / 256, 8L * num_sms()), 256, 0, stream>>>(
        Gs.get(), p, n, model.mean.get(), model.scale.get());
    count_launch();
    FPLS_LAUNCH("standardize_gram");
  }

  // one direction per component: the whole loop as one persistent launch
  // (or handed to the caller's batch when it collects plans)
  if (block <= 1 && !gram_route) {
    std::unique_ptr<PersistentPlan> plan(new PersistentPlan());
    if (plan_simpls_persistent<T>(X, n, p, ld, m, a_max, model, S, gpk, ws, stream, *plan)) {
      if (std::unique_ptr<PersistentPlan>* sink = persistent_deferral()) {
        *sink = std::move(plan);
      } else {
        launch_persistent({plan.get()}, stream);
      }
      return;
    }
  }
  gram_of_columns(S.get(), p, m, gpk, ws, stream);

  // Candidate blocks (the reference's block refresh): the directions of
  // `use` consecutive components are the leading left singular vectors of S
  // at the start of the block, r_j = S_block z_j / sqrt(lambda_j), not
  // recomputed from the deflated S in between.
  block = std::max(1, std::min(block, std::min(a_max, std::min(p, m))));
  DeviceArray<double> zblk, Sblk;
  if (block > 1) {
    zblk.allocate((size_t)m * block, stream);
    Sblk.allocate((size_t)p * m, stream);
  }
  int use = 0, jb = 0;
  for (int a = 0; a < a_max; ++a) {
    if (jb == use) {
      use = std::min(block, a_max - a);
      jb = 0;
      direction_kernel<<<1, jacobi_threads(m), smem_dir, stream>>>(gpk, m, use > 1 ? zblk.get() : zs, scal + 3,
                                                    ws.flag.get(), use);
      count_launch();
      FPLS_LAUNCH("direction_kernel");
      if (use > 1)
        FPLS_CHECK(cudaMemcpyAsync(Sblk.get(), S.get(), sizeof(double) * p * m,
                                   cudaMemcpyDeviceToDevice, stream));
    }
    rvec_kernel<<<g1, TB, 0, stream>>>(use > 1 ? Sblk.get() : S.get(), p, m,
                                       use > 1 ? zblk.get() + (size_t)jb * m : zs,
                                       model.mean.get(), model.scale.get(), r, rt, part,
                                       ctr + 0, scal);
    ++jb;
    count_launch();
    FPLS_LAUNCH("rvec_kernel");
    double* tcol = model.T.get() + (size_t)a * n;
    if (gram_route) {
      // loading = Gs r (Gs symmetric: its columns dot r), ||t||^2 = r . loading
      xtv_product<double>(Gs.get(), p, p, p, r, p, 1, loading.get(), p, ws.stream_partial, stream);
      gram_tstats<<<std::min<unsigned>(ceil_div(p, TB), 2 * num_sms()), TB, 0, stream>>>(
          r, loading.get(), p, part, ctr + 1, scal);
      count_launch();
      FPLS_LAUNCH("gram_tstats");
    } else {
      xr_product<T>(X, n, p, ld, rt, p, 1, scal, tcol, n, ws.stream_partial, stream);
      tstats_kernel<<<std::min<unsigned>(ceil_div(n, TB), 2 * num_sms()), TB, 0, stream>>>(
          tcol, n, part, ctr + 1, scal);
      count_launch();
      FPLS_LAUNCH("tstats");
      xtv_product<T>(X, n, p, ld, tcol, n, 1, praw, p, ws.stream_partial, stream);
    }
    tail1_kernel<<<g1, TB, (2 * TB + a + m) * sizeof(double), stream>>>(
        praw, model.mean.get(), model.scale.get(), scal, r, model.S0.get(),
        model.V.get(), p, m, a, pvec, model.R.get() + (size_t)a * p, part,
        ctr + 2, hq, ws.flag.get(), gram_route ? loading.get() : nullptr);
    tail2_kernel<<<g1, TB, (TB + 1 + m) * sizeof(double), stream>>>(
        pvec, model.V.get(), hq, S.get(), p, m, a, v, part, ctr + 3, vr);
    tail3_kernel<<<g3, jb3, smem3, stream>>>(v, vr, S.get(), p, m,
                                             model.V.get() + (size_t)a * p,
                                             true, part, ctr + 4, gpk,
                                             ws.flag.get());
    if (!gram_route)
      finish_component<<<std::min<unsigned>(ceil_div(n, TB), 2 * num_sms()), TB, 0, stream>>>(
          tcol, n, scal, hq, a, m, model.Q.get() + (size_t)a * m);
    else
      finish_component<<<1, TB, 0, stream>>>(tcol, 0, scal, hq, a, m,
                                             model.Q.get() + (size_t)a * m);
    count_launch(4);
    FPLS_LAUNCH("simpls component");
  }
  model.a = a_max;
  if (gram_route) {
    // training scores T = X_s R (normalised: R holds r / ||t||), one pass
    project_rows<T>(model, X, n, ld, a_max, model.T.get(), n, ws, stream);
  }
}

template <class T>
void project_rows(const DeviceModel& model, const T* X, int rows, long ld,
                  int k, double* out, long ldo, Workspace& ws,
                  cudaStream_t stream) {
  require(k >= 1 && k <= model.a, "invalid projection prefix");
  const int p = model.p;
  DeviceArray<double> Rs((size_t)p * k + k, stream);
  double* roff = Rs.get() + (size_t)p * k;
  scaled_weights<<<k, TB, 0, stream>>>(model.R.get(), p, k, model.mean.get(),
                                       model.scale.get(), Rs.get(), roff);
  count_launch();
  FPLS_LAUNCH("scaled_weights");
  xr_product<T>(X, rows, p, ld, Rs.get(), p, k, roff, out, ldo,
                ws.stream_partial, stream, ws.flag.get());
}

void predict_from_scores(const DeviceModel& model, const double* scores,
                         int rows, long lds, int k, double* out, long ldo,
                         cudaStream_t stream) {
  require(k >= 1 && k <= model.a, "invalid prediction prefix");
  const int m = model.m;
  const long total = (long)rows * m;
  fill_rows_mean<<<(unsigned)std::min<long>((total + 255) / 256, 8L * num_sms()), 256, 0, stream>>>(
      out, rows, m, ldo, model.ymean.get());
  count_launch();
  FPLS_LAUNCH("fill_rows_mean");
  GemmArgs g;
  g.M = rows;
  g.N = m;
  g.K = k;
  g.A = scores;
  g.lda = lds;
  if (model.method == kPlssvd) {
    // W block for prefix k: k x m at offset (k-1) * a * m in model.W
    g.B = model.W.get() + (size_t)(k - 1) * model.a * m;
    g.ldb = k;
  } else {
    g.B = model.Q.get();
    g.ldb = m;
    g.trans_b = true;
  }
  g.C = out;
  g.ldc = ldo;
  g.beta = 1.0;
  gemm_f64(g, stream);
}

template void prepare_responses<float>(const float*, const int*, int, int, double*,
                                       double*, double*, int*, cudaStream_t);
template void prepare_responses<double>(const double*, const int*, int, int, double*,
                                        double*, double*, int*, cudaStream_t);
#define FPLS_INSTANTIATE(T)                                                    \
  template void fit_simpls<T>(const T*, int, int, long, const double*,        \
                              const double*, int, int, int, DeviceModel&,     \
                              Workspace&, cudaStream_t, int, bool);           \
  template void project_rows<T>(const DeviceModel&, const T*, int, long, int, \
                                double*, long, Workspace&, cudaStream_t);   \
  template void compute_crossprod<T>(const T*, int, int, long, const double*, \
                                     const double*, int, int, DeviceModel&,   \
                                     double*, Workspace&, cudaStream_t);
FPLS_INSTANTIATE(float)
FPLS_INSTANTIATE(double)
FPLS_INSTANTIATE(bf16)
#undef FPLS_INSTANTIATE

}  // namespace fpls
