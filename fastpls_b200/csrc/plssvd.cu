// PLS-SVD on the device (FP64 arithmetic, raw X).
//
// Reference: assemble_plssvd_model (inst/include/fastpls/core/plssvd.hpp:57-166)
// and ResidentPlssvd::fit_loaded (src/cuda_resident_plssvd.cuh:82-154):
//   S = Xs^T Yc ; S = U D V^T (rank k) ; R = U_k ; T = Xs R ; G = T^T T ;
//   per prefix j: W_j = G_j^-1 diag(d_1..d_j) V_j^T, Yhat = ymean + T_j W_j.
// The reference's randomized SVD spans the whole response space whenever
// k + oversample >= m, so the SVD here is exact: the m x m Gram S^T S is
// diagonalised by Jacobi (one block) and U = S V D^-1 is formed with one small
// GEMM. One pass over X forms S, one more forms T.
#include "kernels.cuh"
#include "model.cuh"
#include "small.cuh"

#include <algorithm>

namespace fpls {

namespace {

// Eigen-decompose the packed Gram; emit sigma (k), Vk (m x k) and
// Z = Vk D^-1 (m x k) so that U = S Z.
__global__ void small_svd_kernel(const double* __restrict__ gpk, int m, int k,
                                 double* sigma, double* Vk, double* Z,
                                 int* flag) {
  extern __shared__ double sm[];
  double* A = sm;
  double* E = sm + m * m;
  int* order = reinterpret_cast<int*>(E + m * m);
  for (int c = threadIdx.x; c < m; c += blockDim.x)
    for (int d = 0; d <= c; ++d) {
      const double v = gpk[c * (c + 1) / 2 + d];
      A[c + d * m] = v;
      A[d + c * m] = v;
    }
  __syncthreads();
  jacobi_eigen(A, E, m);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < m; ++i) order[i] = i;
    for (int i = 1; i < m; ++i) {  // insertion sort, descending eigenvalue
      const int key = order[i];
      int j = i - 1;
      while (j >= 0 && A[order[j] + order[j] * m] < A[key + key * m]) {
        order[j + 1] = order[j];
        --j;
      }
      order[j + 1] = key;
    }
    for (int c = 0; c < k; ++c) {
      const int src = order[c];
      const double lam = A[src + src * m];
      const double s = lam > 0.0 ? sqrt(lam) : 0.0;
      if (!(s > 0.0) || !isfinite(s)) flag_error(flag, 1);
      int arg = 0;
      for (int r = 1; r < m; ++r)
        if (fabs(E[r + src * m]) > fabs(E[arg + src * m])) arg = r;
      const double sgn = E[arg + src * m] < 0.0 ? -1.0 : 1.0;
      sigma[c] = s;
      for (int r = 0; r < m; ++r) {
        const double v = sgn * E[r + src * m];
        Vk[r + c * m] = v;
        Z[r + c * m] = s > 0.0 ? v / s : 0.0;
      }
    }
  }
}

// Cholesky of the score Gram once; thread j forms the prefix (j+1) weights
// W_{j+1} = G_{j+1}^-1 diag(sigma_1..j+1) V_{j+1}^T into its own block.
__global__ void plssvd_weights_kernel(const double* __restrict__ gram, int a,
                                      const double* __restrict__ sigma,
                                      const double* __restrict__ Vk, int m,
                                      double* W, double* lwork, int* flag) {
  __shared__ bool ok;
  if (threadIdx.x == 0) {
    for (int idx = 0; idx < a * a; ++idx) lwork[idx] = gram[idx];
    ok = cholesky_serial(lwork, a, 0.0);
    if (!ok) flag_error(flag, 6);
  }
  __syncthreads();
  if (!ok) return;
  for (int j = threadIdx.x; j < a; j += blockDim.x) {
    const int k = j + 1;
    double* Wk = W + (size_t)j * a * m;  // k x m, ld k
    double col[128];
    for (int c = 0; c < k; ++c) {
      // latent column c: solve L_k L_k^T x = sigma_c e_c (L_k = leading block)
      for (int i = 0; i < k; ++i) col[i] = (i == c) ? sigma[c] : 0.0;
      for (int i = 0; i < k; ++i) {
        double v = col[i];
        for (int q = 0; q < i; ++q) v -= lwork[i + q * a] * col[q];
        col[i] = v / lwork[i + i * a];
      }
      for (int i = k - 1; i >= 0; --i) {
        double v = col[i];
        for (int q = i + 1; q < k; ++q) v -= lwork[q + i * a] * col[q];
        col[i] = v / lwork[i + i * a];
      }
      // W_k[:, r] += latent[:, c] * V[r, c]
      for (int r = 0; r < m; ++r) {
        const double vr = Vk[r + c * m];
        for (int i = 0; i < k; ++i) {
          const double prev = (c == 0) ? 0.0 : Wk[i + r * k];
          Wk[i + r * k] = prev + col[i] * vr;
        }
      }
    }
  }
}

}  // namespace

template <class T>
void fit_plssvd(const T* X, int n, int p, long ld, const double* Yc,
                const double* ycsum, int m, int components, int scaling,
                DeviceModel& model, Workspace& ws, cudaStream_t stream) {
  require(m >= 1 && m <= kMaxResponses, "PLS-SVD supports 1..112 responses or classes");
  require(components <= 128, "PLS-SVD supports at most 128 components");
  const int k = components;
  require(k <= std::min(p, m), "fastPLS PLS-SVD component count exceeds cross-covariance rank");
  if (model.classification && k >= m)
    throw std::invalid_argument("classification PLS-SVD components must be below class count");
  ws.ensure(n, p, m, k, stream);
  model.method = kPlssvd;
  model.n = n;
  model.p = p;
  model.feature_p = p;
  model.m = m;
  model.scaling = scaling;
  DeviceArray<double> S((size_t)p * m, stream);
  compute_crossprod<T>(X, n, p, ld, Yc, ycsum, m, scaling, model, S.get(), ws, stream);
  double* gpk = ws.small.get() + 8 + kMaxResponses;
  gram_of_columns(S.get(), p, m, gpk, ws, stream);
  model.sigma.allocate(k, stream);
  model.Q.allocate((size_t)m * k, stream);
  DeviceArray<double> Z((size_t)m * k, stream);
  const size_t smem = 2 * (size_t)m * m * sizeof(double) + m * sizeof(int) + 16;
  if (smem > 48 * 1024)
    FPLS_CHECK(cudaFuncSetAttribute(small_svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  small_svd_kernel<<<1, jacobi_threads(m), smem, stream>>>(gpk, m, k, model.sigma.get(),
                                            model.Q.get(), Z.get(), ws.flag.get());
  count_launch();
  FPLS_LAUNCH("small_svd");
  // U = S Z  (p x k)
  model.R.allocate((size_t)p * k, stream);
  GemmArgs g;
  g.M = p;
  g.N = k;
  g.K = m;
  g.A = S.get();
  g.lda = p;
  g.B = Z.get();
  g.ldb = m;
  g.C = model.R.get();
  g.ldc = p;
  gemm_f64(g, stream);
  model.a = k;
  // T = Xs U  (n x k)
  model.T.allocate((size_t)n * k, stream);
  project_rows<T>(model, X, n, ld, k, model.T.get(), n, ws, stream);
  // G = T^T T (k x k)
  DeviceArray<double> gram((size_t)k * k, stream);
  GemmArgs h;
  h.M = k;
  h.N = k;
  h.K = n;
  h.A = model.T.get();
  h.lda = n;
  h.trans_a = true;
  h.B = model.T.get();
  h.ldb = n;
  h.splits = gemm_pick_splits(k, k, n);
  DeviceArray<double> parts((size_t)h.splits * k * k, stream);
  h.C = parts.get();
  h.ldc = k;
  h.split_stride = (long)k * k;
  gemm_f64(h, stream);
  FPLS_CHECK(cudaMemcpyAsync(gram.get(), parts.get(), sizeof(double) * k * k,
                             cudaMemcpyDeviceToDevice, stream));
  model.W.allocate((size_t)k * k * m, stream);
  DeviceArray<double> lwork((size_t)k * k, stream);
  plssvd_weights_kernel<<<1, 128, 0, stream>>>(gram.get(), k, model.sigma.get(),
                                               model.Q.get(), m, model.W.get(),
                                               lwork.get(), ws.flag.get());
  count_launch();
  FPLS_LAUNCH("plssvd_weights");
}

template void fit_plssvd<float>(const float*, int, int, long, const double*,
                                const double*, int, int, int, DeviceModel&,
                                Workspace&, cudaStream_t);
template void fit_plssvd<double>(const double*, int, int, long, const double*,
                                 const double*, int, int, int, DeviceModel&,
                                 Workspace&, cudaStream_t);
template void fit_plssvd<bf16>(const bf16*, int, int, long, const double*,
                               const double*, int, int, int, DeviceModel&,
                               Workspace&, cudaStream_t);

}  // namespace fpls
