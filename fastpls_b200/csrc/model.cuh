// Resident model state and fitting entry points (host declarations).
#pragma once

#include "common.cuh"

#include <algorithm>
#include <type_traits>

namespace fpls {

// m x m direction eigenproblem in one block: 2 m^2 doubles of shared memory
// (200 KB at 112) and m <= 128 for the block Jacobi
constexpr int kMaxResponses = 112;

enum Method { kPlssvd = 1, kSimpls = 3, kOpls = 4, kKernelPls = 5 };

// Scratch reused across the kernels of one fit / prediction.
struct Workspace {
  DeviceArray<double> stream_partial;  // xr / xtv per-chunk partials
  DeviceArray<double> block_partial;   // last-block reductions
  DeviceArray<unsigned> counters;      // tickets of last-block reductions
  DeviceArray<double> vec_p[5];        // p-length vectors
  DeviceArray<double> vec_n[2];        // n-length vectors
  DeviceArray<double> small;           // small scalars / m x m blocks
  DeviceArray<int> flag;               // device error flag
  void ensure(int n, int p, int m, int a, cudaStream_t s);
};

// A fitted model resident on the device. Every matrix is FP64 and
// column-major. Linear methods predict Yhat = ymean + Xs R_k Q_k^T with
// Xs = (X - mean) / scale; PLS-SVD uses per-prefix weights instead of Q.
struct DeviceModel {
  int method = kSimpls;
  int n = 0, p = 0, m = 0, a = 0;  // rows, input columns, responses, components
  int feature_p = 0;               // rows of R (p; n for kernel PLS)
  int scaling = 1;
  bool classification = false;
  DeviceArray<double> mean, scale, ymean;  // p, p, m
  DeviceArray<double> R, Q, V, T;          // p x a, m x a, p x a, n x a
  DeviceArray<double> S0;                  // p x m centred cross-product
  DeviceArray<double> sigma;               // PLS-SVD singular values (a)
  DeviceArray<double> W;                   // PLS-SVD per-prefix weights (a x m x a)
  DeviceArray<int> labels;                 // training labels (classification)
  const int* label_view = nullptr;         // labels of the rows being fitted
                                           // (one-based, not owned): the
                                           // class-sum cross-product pass
  std::vector<int> class_counts;           // host copy (classification)
  // kernel PLS: input standardisation (in_p columns), standardised training
  // rows, their squared norms, training kernel column means (+ grand mean)
  int in_p = 0, kernel_kind = 0, degree = 0;
  double gamma = 0.0, coef0 = 0.0;
  DeviceArray<double> in_mean, in_scale, reference, ref_norms, kcol_means;
};

// Centre responses (dense Y, or one-hot minus prior for one-based labels).
// Yc: n x m FP64; ymean: m; ycsum: column sums of Yc (rounding residue).
template <class T>
void prepare_responses(const T* Y, const int* labels, int n, int m,
                       double* Yc, double* ymean, double* ycsum, int* flag,
                       cudaStream_t stream);

// SIMPLS fit on raw X (n x p, ld) with centred responses Yc (n x m).
// Fills model.{mean, scale, ymean (caller), R, Q, V, T, S0, a}.
// gram_route: loadings from the cached p x p Gram of the standardised
// predictors instead of two passes over X per component (simpls_gram_route).
template <class T>
void fit_simpls(const T* X, int n, int p, long ld, const double* Yc,
                const double* ycsum, int m, int components, int scaling,
                DeviceModel& model, Workspace& ws, cudaStream_t stream,
                int block = 1, bool gram_route = false);

// The reference's cached predictor cross-product route
// (src/cuda_resident_simpls.cuh:135, step_crossprod in
// src/cuda_resident_component.cuh:131-167): classification fits with at
// least 8 components and n >= 8 p form X_s^T X_s once and take each
// component's loadings from it; the scores are X_s R at the end. FP32 and
// FP64 storage.
inline bool simpls_gram_route(int n, int p, int components, bool classification) {
  return classification && components >= 8 && (long)n >= 8L * p;
}

// Candidate block size of a SIMPLS fit (src/cuda_resident_simpls.cuh:144-153):
// a classification fit with q <= 2048 classes, at least 4 components and
// n p q >= 5e8 takes min(64, components, p, q) directions from one
// decomposition; an FP32 regression fit whose p x q cross-covariance exceeds
// 512 MiB in FP32 and has at least 4 components takes min(8, components, p, q);
// every other fit refreshes the direction once per component.
inline int simpls_block_size(int n, int p, int q, int components,
                             bool classification, bool fp32) {
  const double work = (double)n * (double)p * (double)q;
  const int cap = std::min(components, std::min(p, q));
  if (classification && q <= 2048 && components >= 4 && work >= 5.0e8)
    return std::max(1, std::min(64, cap));
  if (!classification && fp32 && components >= 4 &&
      (double)p * (double)q * 4.0 > 512.0 * 1024.0 * 1024.0)
    return std::max(1, std::min(8, cap));
  return 1;
}

// PLS-SVD fit (exact SVD of the m-column cross-product).
template <class T>
void fit_plssvd(const T* X, int n, int p, long ld, const double* Yc,
                const double* ycsum, int m, int components, int scaling,
                DeviceModel& model, Workspace& ws, cudaStream_t stream);

// Column centre/scale (model.mean, model.scale) and the scaled centred
// cross-product S = Xs^T Yc (written to S and model.S0), one pass over X.
template <class T>
void compute_crossprod(const T* X, int n, int p, long ld, const double* Yc,
                       const double* ycsum, int m, int scaling,
                       DeviceModel& model, double* S, Workspace& ws,
                       cudaStream_t stream);

// Packed lower triangle of S^T S (m x m) for S p x m, into gpk.
void gram_of_columns(double* S, int p, int m, double* gpk, Workspace& ws,
                     cudaStream_t stream);

// Unit dominant left singular vector w (p) of S (p x m) from its packed Gram
// (gpk, from gram_of_columns); zs receives z / sqrt(lambda).
void dominant_direction(const double* S, int p, int m, const double* gpk,
                        double* zs, double* w, Workspace& ws, cudaStream_t s);

// OPLS (north orthogonal filters + SIMPLS on the filtered predictors);
// `design` keeps the filtered standardised predictors (FP64 n x p).
template <class T>
void fit_opls(const T* X, int n, int p, long ld, const double* Yc,
              const double* ycsum, int m, int components, int scaling,
              int north, DeviceModel& model, Workspace& ws,
              DeviceArray<double>& design, cudaStream_t s);

// Nonlinear kernel PLS (kind 2 = RBF, 3 = polynomial); `design` keeps the
// centred n x n training kernel.
template <class T>
void fit_kernelpls(const T* X, int n, int p, long ld, const double* Yc,
                   const double* ycsum, int m, int components, int scaling,
                   int kind, double gamma, int degree, double coef0,
                   DeviceModel& model, Workspace& ws, DeviceArray<double>& design,
                   cudaStream_t s);

// Kernel PLS scores of new rows (rows x k).
template <class T>
void kernel_scores(const DeviceModel& model, const T* X, int rows, long ld, int k,
                   double* out, long ldo, Workspace& ws, cudaStream_t s);

// Latent scores of new rows: out (rows x k) = Xs R[:, :k] (FP64).
template <class T>
void project_rows(const DeviceModel& model, const T* X, int rows, long ld,
                  int k, double* out, long ldo, Workspace& ws,
                  cudaStream_t stream);

// Responses for prefix k from scores (rows x >= k): out = ymean + T_k B_k.
void predict_from_scores(const DeviceModel& model, const double* scores,
                         int rows, long lds, int k, double* out, long ldo,
                         cudaStream_t stream);

// Throws when the device error flag was raised (synchronises the stream).
void raise_on_flag(Workspace& ws, cudaStream_t stream, const char* message);

}  // namespace fpls
