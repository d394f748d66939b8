// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// C-callable harness around the reference's own header-only FP64 numerics
// (fastPLS inst/include/fastpls/core/*.hpp, compiled unchanged from the
// reference tree by oracle/Makefile into oracle/_ref/libfastpls_ref.so).
// It plays the role of the reference's CPU path
// (src/r_api.cpp: pls_matrix_core_cpp 5316-5375, regression_cv_result
// 1702-1760, classification_cv_result 1603-1660), which itself cannot be
// built here because it includes R headers.
//
// The linear-algebra backend below is written for this project. It mirrors
// the reference's CPU adapter (src/core_cpu_backend.cpp:441-526 gemm,
// src/core_cpu_lapack.cpp:49-205 dgeqrf+dorgqr / dsyevd('V','L') /
// dgesvd('S','N') / dgesdd('S')) over the LP64 OpenBLAS that scipy ships.
// The solver controls restate src/r_api.cpp:1149-1190 (simpls_controls).
#include <fastpls/core.hpp>
#include <fastpls/core/cross_validation.hpp>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

extern "C" {
void scipy_cblas_dgemm(int order, int transa, int transb, int m, int n, int k,
                       double alpha, const double* a, int lda, const double* b,
                       int ldb, double beta, double* c, int ldc);
void scipy_dgeqrf_(const int* m, const int* n, double* a, const int* lda,
                   double* tau, double* work, const int* lwork, int* info);
void scipy_dorgqr_(const int* m, const int* n, const int* k, double* a,
                   const int* lda, const double* tau, double* work,
                   const int* lwork, int* info);
void scipy_dsyevd_(const char* jobz, const char* uplo, const int* n, double* a,
                   const int* lda, double* w, double* work, const int* lwork,
                   int* iwork, const int* liwork, int* info, size_t, size_t);
void scipy_dgesvd_(const char* jobu, const char* jobvt, const int* m,
                   const int* n, double* a, const int* lda, double* s,
                   double* u, const int* ldu, double* vt, const int* ldvt,
                   double* work, const int* lwork, int* info, size_t, size_t);
void scipy_dgesdd_(const char* jobz, const int* m, const int* n, double* a,
                   const int* lda, double* s, double* u, const int* ldu,
                   double* vt, const int* ldvt, double* work, const int* lwork,
                   int* iwork, int* info, size_t);
void scipy_openblas_set_num_threads(int);
}

namespace {

using fastpls::core::ConstMatrixView;
using fastpls::core::Matrix;
using fastpls::core::MatrixView;

constexpr int kColMajor = 102, kNoTrans = 111, kTrans = 112;

int as_int(std::size_t value) {
  if (value > static_cast<std::size_t>(0x7fffffff))
    throw std::invalid_argument("oracle dimension exceeds LP64 LAPACK");
  return static_cast<int>(value);
}

Matrix<double> dense_copy(ConstMatrixView<double> input) {
  Matrix<double> out(input.rows(), input.columns());
  for (std::size_t c = 0; c < input.columns(); ++c)
    for (std::size_t r = 0; r < input.rows(); ++r) out(r, c) = input(r, c);
  return out;
}

int query_size(double q) {
  if (!(q >= 1.0)) return 1;
  return static_cast<int>(q);
}

// Backend concept of fastpls::core (core/README.md): gemm, qr_economy,
// symmetric_eigen, svd_economy.
class BlasBackend {
 public:
  void gemm(ConstMatrixView<double> left, ConstMatrixView<double> right,
            bool tl, bool tr, MatrixView<double> out) {
    const std::size_t m = out.rows(), n = out.columns();
    const std::size_t k = tl ? left.rows() : left.columns();
    if (m == 0 || n == 0) return;
    if (k == 0) {
      for (std::size_t c = 0; c < n; ++c)
        for (std::size_t r = 0; r < m; ++r) out(r, c) = 0.0;
      return;
    }
    scipy_cblas_dgemm(kColMajor, tl ? kTrans : kNoTrans, tr ? kTrans : kNoTrans,
                      as_int(m), as_int(n), as_int(k), 1.0, left.data(),
                      std::max(1, as_int(left.leading_dimension())),
                      right.data(),
                      std::max(1, as_int(right.leading_dimension())), 0.0,
                      out.data(), std::max(1, as_int(out.leading_dimension())));
  }

  bool qr_economy(ConstMatrixView<double> input, Matrix<double>& q) {
    const int m = as_int(input.rows()), n = as_int(input.columns());
    const int rank = std::min(m, n);
    if (rank == 0) {
      q.resize(input.rows(), 0);
      return true;
    }
    Matrix<double> factor = dense_copy(input);
    const int lda = std::max(1, m);
    std::vector<double> tau(rank);
    int info = 0, lwork = -1;
    double wq = 0.0;
    scipy_dgeqrf_(&m, &n, factor.data(), &lda, tau.data(), &wq, &lwork, &info);
    if (info) return false;
    lwork = query_size(wq);
    std::vector<double> work(lwork);
    scipy_dgeqrf_(&m, &n, factor.data(), &lda, tau.data(), work.data(), &lwork,
                  &info);
    if (info) return false;
    q.resize(input.rows(), rank);
    std::memcpy(q.data(), factor.data(), sizeof(double) * m * rank);
    lwork = -1;
    scipy_dorgqr_(&m, &rank, &rank, q.data(), &lda, tau.data(), &wq, &lwork,
                  &info);
    if (info) return false;
    lwork = query_size(wq);
    work.assign(lwork, 0.0);
    scipy_dorgqr_(&m, &rank, &rank, q.data(), &lda, tau.data(), work.data(),
                  &lwork, &info);
    return info == 0;
  }

  bool symmetric_eigen(Matrix<double>& a, std::vector<double>& values) {
    if (a.rows() != a.columns())
      throw std::invalid_argument("oracle eigen needs a square matrix");
    const int n = as_int(a.rows());
    values.resize(n);
    if (n == 0) return true;
    const int lda = std::max(1, n);
    int info = 0, lwork = -1, liwork = -1, iq = 0;
    double wq = 0.0;
    scipy_dsyevd_("V", "L", &n, a.data(), &lda, values.data(), &wq, &lwork,
                  &iq, &liwork, &info, 1, 1);
    if (info) return false;
    lwork = query_size(wq);
    liwork = std::max(1, iq);
    std::vector<double> work(lwork);
    std::vector<int> iwork(liwork);
    scipy_dsyevd_("V", "L", &n, a.data(), &lda, values.data(), work.data(),
                  &lwork, iwork.data(), &liwork, &info, 1, 1);
    return info == 0;
  }

  bool svd_economy(ConstMatrixView<double> input, bool left_only,
                   Matrix<double>& u, std::vector<double>& s,
                   Matrix<double>& vt) {
    const int m = as_int(input.rows()), n = as_int(input.columns());
    const int rank = std::min(m, n);
    if (rank == 0) {
      u.resize(input.rows(), 0);
      s.clear();
      vt.resize(0, input.columns());
      return true;
    }
    Matrix<double> factor = dense_copy(input);
    const int lda = std::max(1, m), ldu = std::max(1, m);
    u.resize(input.rows(), rank);
    s.resize(rank);
    int info = 0, lwork = -1;
    double wq = 0.0;
    if (left_only) {
      const int ldvt = 1;
      double dummy = 0.0;
      scipy_dgesvd_("S", "N", &m, &n, factor.data(), &lda, s.data(), u.data(),
                    &ldu, &dummy, &ldvt, &wq, &lwork, &info, 1, 1);
      if (info) return false;
      lwork = query_size(wq);
      std::vector<double> work(lwork);
      scipy_dgesvd_("S", "N", &m, &n, factor.data(), &lda, s.data(), u.data(),
                    &ldu, &dummy, &ldvt, work.data(), &lwork, &info, 1, 1);
      vt.resize(0, input.columns());
      return info == 0;
    }
    const int ldvt = std::max(1, rank);
    vt.resize(rank, input.columns());
    std::vector<int> iwork(8 * rank);
    scipy_dgesdd_("S", &m, &n, factor.data(), &lda, s.data(), u.data(), &ldu,
                  vt.data(), &ldvt, &wq, &lwork, iwork.data(), &info, 1);
    if (info) return false;
    lwork = query_size(wq);
    std::vector<double> work(lwork);
    scipy_dgesdd_("S", &m, &n, factor.data(), &lda, s.data(), u.data(), &ldu,
                  vt.data(), &ldvt, work.data(), &lwork, iwork.data(), &info,
                  1);
    return info == 0;
  }
};

// Restatement of src/r_api.cpp:1149-1190 (environment knobs at defaults:
// FAST_CROSSPROD_MAX_P 512, MIN_NCOMP 20, MIN_N_TO_P_RATIO 8).
fastpls::core::SimplsControls simpls_controls(
    std::size_t n, std::size_t p, std::size_t m, std::size_t components,
    bool classification, int oversample, int power, unsigned seed) {
  fastpls::core::SimplsControls c;
  c.components = components;
  c.maximum_block = fastpls::core::simpls_candidate_block_size(
      components, p, m, classification, n, 64);
  c.cache_predictor_crossprod = components >= 20 && p <= n && n >= p * 8 &&
                                p <= 512;
  c.batch_candidate_geometry = c.maximum_block > 1 &&
                               !c.cache_predictor_crossprod;
  c.reorthogonalize = false;
  c.store_scores = true;
  c.use_right_gram = true;
  c.rsvd.oversample = oversample;
  c.rsvd.power = power;
  c.rsvd.seed = seed;
  return c;
}

void put_error(char* out, std::size_t cap, const char* message) {
  if (out && cap) std::snprintf(out, cap, "%s", message);
}

Matrix<double> load(const double* data, std::size_t rows, std::size_t cols) {
  Matrix<double> out(rows, cols);
  std::memcpy(out.data(), data, sizeof(double) * rows * cols);
  return out;
}

void store(const Matrix<double>& m, double* out) {
  if (out && m.rows() * m.columns())
    std::memcpy(out, m.data(), sizeof(double) * m.rows() * m.columns());
}

}  // namespace

extern "C" {

void ref_set_threads(int threads) {
  scipy_openblas_set_num_threads(threads < 1 ? 1 : threads);
}

// One SIMPLS fit as the reference CPU path runs it: in-place scaling and the
// centred cross-product (supervised.hpp:27-124 / classification.hpp:88-186),
// then fit_simpls_preprocessed<double> (simpls.hpp:479-763).
// labels: one-based class labels (or NULL for dense responses y, n x m).
// Outputs are column-major; any output pointer may be NULL.
int ref_simpls_fit(const double* x, const double* y, const int* labels, int n,
                   int p, int m, int ncomp, int scaling, int oversample,
                   int power, unsigned seed, double* weights,
                   double* response_loadings, double* deflation_basis,
                   double* scores, double* predictor_center,
                   double* predictor_scale, double* response_mean,
                   int* completed, double* seconds, char* error,
                   std::size_t capacity) {
  put_error(error, capacity, "");
  try {
    BlasBackend backend;
    Matrix<double> predictors = load(x, n, p);
    const auto scale = static_cast<fastpls::core::PredictorScaling>(scaling);
    std::vector<double> centre, spread, ymean;
    Matrix<double> crossprod;
    if (labels) {
      std::vector<std::size_t> zero_based(n);
      for (int i = 0; i < n; ++i) zero_based[i] = std::size_t(labels[i] - 1);
      auto prepared = fastpls::core::prepare_scaled_label_crossprod(
          predictors.view(), zero_based.data(), std::size_t(n), std::size_t(m),
          scale, backend);
      crossprod = std::move(prepared.crossprod);
      centre = prepared.predictor_center;
      spread = prepared.predictor_scale;
      ymean = prepared.response_mean;
    } else {
      Matrix<double> responses = load(y, n, m);
      auto prepared = fastpls::core::prepare_scaled_dense_crossprod(
          predictors.view(), ConstMatrixView<double>(responses.view()), scale,
          backend);
      crossprod = std::move(prepared.crossprod);
      centre = prepared.predictor_center;
      spread = prepared.predictor_scale;
      ymean = prepared.response_mean;
    }
    const std::size_t capped = std::min<std::size_t>(
        {std::size_t(ncomp), std::size_t(p),
         std::max<std::size_t>(std::size_t(n) - 1, 1)});
    auto controls = simpls_controls(n, p, m, capped, labels != nullptr,
                                    oversample, power, seed);
    controls.phase_timing = true;
    fastpls::core::SimplsWorkspace<double> workspace;
    auto model = fastpls::core::fit_simpls_preprocessed<double>(
        ConstMatrixView<double>(predictors.view()),
        ConstMatrixView<double>(crossprod.view()), controls, backend,
        workspace);
    store(model.weights, weights);
    store(model.response_loadings, response_loadings);
    store(model.deflation_basis, deflation_basis);
    store(model.scores, scores);
    if (predictor_center) std::copy(centre.begin(), centre.end(), predictor_center);
    if (predictor_scale) std::copy(spread.begin(), spread.end(), predictor_scale);
    if (response_mean) std::copy(ymean.begin(), ymean.end(), response_mean);
    if (completed) *completed = int(model.completed_components);
    if (seconds) *seconds = model.timing.total;
    return 0;
  } catch (const std::exception& e) {
    put_error(error, capacity, e.what());
    return 1;
  }
}

// One PLS-SVD fit (plssvd.hpp:57-166 via fit_plssvd_preprocessed 196-223).
// prediction_weights receives, for each prefix j, a prefixes[j] x m block
// (concatenated, column-major), i.e. the matrix W with Yhat = mean + T_j W.
int ref_plssvd_fit(const double* x, const double* y, const int* labels, int n,
                   int p, int m, const int* prefixes, int prefix_count,
                   int scaling, int oversample, int power, unsigned seed,
                   double* weights, double* response_loadings, double* scores,
                   double* singular_values, double* prediction_weights,
                   double* predictor_center, double* predictor_scale,
                   double* response_mean, char* error, std::size_t capacity) {
  put_error(error, capacity, "");
  try {
    BlasBackend backend;
    Matrix<double> predictors = load(x, n, p);
    const auto scale = static_cast<fastpls::core::PredictorScaling>(scaling);
    std::vector<double> centre, spread, ymean;
    Matrix<double> crossprod;
    if (labels) {
      std::vector<std::size_t> zero_based(n);
      for (int i = 0; i < n; ++i) zero_based[i] = std::size_t(labels[i] - 1);
      auto prepared = fastpls::core::prepare_scaled_label_crossprod(
          predictors.view(), zero_based.data(), std::size_t(n), std::size_t(m),
          scale, backend);
      crossprod = std::move(prepared.crossprod);
      centre = prepared.predictor_center;
      spread = prepared.predictor_scale;
      ymean = prepared.response_mean;
    } else {
      Matrix<double> responses = load(y, n, m);
      auto prepared = fastpls::core::prepare_scaled_dense_crossprod(
          predictors.view(), ConstMatrixView<double>(responses.view()), scale,
          backend);
      crossprod = std::move(prepared.crossprod);
      centre = prepared.predictor_center;
      spread = prepared.predictor_scale;
      ymean = prepared.response_mean;
    }
    fastpls::core::PlssvdControls controls;
    controls.rsvd.oversample = oversample;
    controls.rsvd.power = power;
    controls.rsvd.seed = seed;
    auto model = fastpls::core::fit_plssvd_preprocessed<double>(
        ConstMatrixView<double>(predictors.view()),
        ConstMatrixView<double>(crossprod.view()), prefixes,
        std::size_t(prefix_count), controls, backend);
    store(model.weights, weights);
    store(model.response_loadings, response_loadings);
    store(model.scores, scores);
    if (singular_values)
      std::copy(model.singular_values.begin(), model.singular_values.end(),
                singular_values);
    if (prediction_weights) {
      double* cursor = prediction_weights;
      for (const auto& w : model.prediction_weights) {
        store(w, cursor);
        cursor += w.rows() * w.columns();
      }
    }
    if (predictor_center) std::copy(centre.begin(), centre.end(), predictor_center);
    if (predictor_scale) std::copy(spread.begin(), spread.end(), predictor_scale);
    if (response_mean) std::copy(ymean.begin(), ymean.end(), response_mean);
    return 0;
  } catch (const std::exception& e) {
    put_error(error, capacity, e.what());
    return 1;
  }
}

// Regression cross-validation (cross_validation.hpp:1790-2173), driven as
// src/r_api.cpp:1702-1760 drives it. family: 1 = PLS-SVD, 3 = SIMPLS.
// predictions (optional): prefix_count blocks of n x m.
int ref_cv_regression(const double* x, const double* y, const int* folds,
                      int n, int p, int m, const int* prefixes,
                      int prefix_count, int scaling, int family, int metric,
                      int oversample, int power, unsigned seed,
                      double* predictions, int* status, double* metrics,
                      double* q2, double* rmsd, double* observed_r2,
                      char* error, std::size_t capacity) {
  put_error(error, capacity, "");
  try {
    BlasBackend backend;
    Matrix<double> predictors = load(x, n, p);
    Matrix<double> responses = load(y, n, m);
    fastpls::core::PlssvdControls plssvd;
    plssvd.rsvd.oversample = oversample;
    plssvd.rsvd.power = power;
    plssvd.rsvd.seed = seed;
    const int maximum = *std::max_element(prefixes, prefixes + prefix_count);
    const auto simpls = simpls_controls(n, p, m, std::size_t(maximum), false,
                                        oversample, power, seed);
    auto result = fastpls::core::cross_validate_regression<double>(
        ConstMatrixView<double>(predictors.view()),
        ConstMatrixView<double>(responses.view()), folds, prefixes,
        std::size_t(prefix_count),
        static_cast<fastpls::core::PredictorScaling>(scaling),
        static_cast<fastpls::core::LinearPlsFamily>(family),
        static_cast<fastpls::core::RegressionMetric>(metric), plssvd, simpls,
        backend, predictions != nullptr);
    for (std::size_t f = 0; f < result.status.size(); ++f)
      if (status) status[f] = result.status[f];
    for (int j = 0; j < prefix_count; ++j) {
      if (metrics) metrics[j] = result.metrics[j];
      if (q2) q2[j] = result.q2[j];
      if (rmsd) rmsd[j] = result.rmsd[j];
      if (observed_r2) observed_r2[j] = result.observed_r2[j];
      if (predictions)
        store(result.predictions[j], predictions + std::size_t(j) * n * m);
    }
    return 0;
  } catch (const std::exception& e) {
    put_error(error, capacity, e.what());
    return 1;
  }
}

// Classification cross-validation (cross_validation.hpp:1360-1788), driven as
// src/r_api.cpp:1603-1660 drives it. head: 0 = argmax, 1 = LDA.
// predictions (optional): n x prefix_count one-based labels.
int ref_cv_classification(const double* x, const int* labels, const int* folds,
                          int n, int p, int classes, const int* prefixes,
                          int prefix_count, int scaling, int family, int head,
                          int oversample, int power, unsigned seed,
                          int* predictions, int* status, double* metrics,
                          char* error, std::size_t capacity) {
  put_error(error, capacity, "");
  try {
    BlasBackend backend;
    Matrix<double> predictors = load(x, n, p);
    fastpls::core::PlssvdControls plssvd;
    plssvd.rsvd.oversample = oversample;
    plssvd.rsvd.power = power;
    plssvd.rsvd.seed = seed;
    const int maximum = *std::max_element(prefixes, prefixes + prefix_count);
    const auto simpls = simpls_controls(n, p, classes, std::size_t(maximum),
                                        true, oversample, power, seed);
    auto result = fastpls::core::cross_validate_classification<double>(
        ConstMatrixView<double>(predictors.view()), labels,
        std::size_t(classes), folds, prefixes, std::size_t(prefix_count),
        static_cast<fastpls::core::PredictorScaling>(scaling),
        static_cast<fastpls::core::LinearPlsFamily>(family),
        static_cast<fastpls::core::ClassificationHead>(head), plssvd, simpls,
        backend, predictions != nullptr, false);
    for (std::size_t f = 0; f < result.status.size(); ++f)
      if (status) status[f] = result.status[f];
    for (int j = 0; j < prefix_count; ++j) {
      if (metrics) metrics[j] = result.metrics[j];
    }
    if (predictions)
      std::memcpy(predictions, result.predictions.data(),
                  sizeof(int) * std::size_t(n) * prefix_count);
    return 0;
  } catch (const std::exception& e) {
    put_error(error, capacity, e.what());
    return 1;
  }
}

// OPLS + SIMPLS (oplspls.hpp:30-74 fit, 86-101 predict) with the exact
// leading-direction filter (opls.hpp:57-115, randomized_filter = false).
// predictions: rows x m for `ncomp` components of the predictive model.
int ref_opls_predict(const double* x, const double* y, int n, int p, int m,
                     int ncomp, int north, int scaling, const double* xtest,
                     int rows, double* predictions, char* error,
                     std::size_t capacity) {
  put_error(error, capacity, "");
  try {
    BlasBackend backend;
    fastpls::core::OplsControls c;
    c.orthogonal_components = std::size_t(north);
    c.scaling = static_cast<fastpls::core::PredictorScaling>(scaling);
    c.randomized_filter = false;
    c.simpls = simpls_controls(n, p, m, std::size_t(ncomp), false, 32, 5, 1);
    Matrix<double> responses = load(y, n, m);
    auto model = fastpls::core::fit_opls<double>(
        load(x, n, p), ConstMatrixView<double>(responses.view()), c, backend);
    auto pred = fastpls::core::predict_opls<double>(model, load(xtest, rows, p),
                                                    std::size_t(ncomp), backend);
    store(pred, predictions);
    return 0;
  } catch (const std::exception& e) {
    put_error(error, capacity, e.what());
    return 1;
  }
}

// Kernel PLS (kernelpls.hpp:85-196): kind 2 = RBF, 3 = polynomial.
int ref_kernelpls_predict(const double* x, const double* y, int n, int p,
                          int m, int ncomp, int scaling, int kind,
                          double gamma, int degree, double coef0,
                          const double* xtest, int rows, double* predictions,
                          char* error, std::size_t capacity) {
  put_error(error, capacity, "");
  try {
    BlasBackend backend;
    fastpls::core::KernelPlsControls c;
    c.kernel = static_cast<fastpls::core::KernelType>(kind);
    c.gamma = gamma;
    c.degree = degree;
    c.offset = coef0;
    c.scaling = static_cast<fastpls::core::PredictorScaling>(scaling);
    c.simpls = simpls_controls(n, n, m, std::size_t(ncomp), false, 32, 5, 1);
    Matrix<double> responses = load(y, n, m);
    auto model = fastpls::core::fit_kernelpls<double>(
        load(x, n, p), ConstMatrixView<double>(responses.view()), c, backend);
    auto pred = fastpls::core::predict_kernelpls<double>(model, load(xtest, rows, p),
                                                         std::size_t(ncomp), backend);
    store(pred, predictions);
    return 0;
  } catch (const std::exception& e) {
    put_error(error, capacity, e.what());
    return 1;
  }
}

// LDA on latent scores (lda.hpp:156-223 train, 284-318 predict).
// discriminants (optional): prefix_count blocks of rows x classes;
// predicted: rows x prefix_count one-based labels.
int ref_lda(const double* train_scores, const int* labels, int n, int a,
            int classes, const int* prefixes, int prefix_count,
            const double* test_scores, int rows, double* discriminants,
            int* predicted, char* error, std::size_t capacity) {
  put_error(error, capacity, "");
  try {
    Matrix<double> scores = load(train_scores, n, a);
    Matrix<double> test = load(test_scores, rows, a);
    auto models = fastpls::core::train_lda_prefixes<double>(
        ConstMatrixView<double>(scores.view()), labels, std::size_t(n),
        std::size_t(classes), prefixes, std::size_t(prefix_count));
    for (int j = 0; j < prefix_count; ++j) {
      const std::size_t k = std::size_t(prefixes[j]);
      ConstMatrixView<double> prefix_view(test.data(), rows, k, rows);
      auto d = fastpls::core::lda_scores<double>(prefix_view, models[j]);
      if (discriminants) store(d, discriminants + std::size_t(j) * rows * classes);
      if (predicted) {
        for (int r = 0; r < rows; ++r)
          predicted[std::size_t(j) * rows + r] =
              int(fastpls::core::row_argmax(ConstMatrixView<double>(d.view()),
                                            std::size_t(r)) + 1);
      }
    }
    return 0;
  } catch (const std::exception& e) {
    put_error(error, capacity, e.what());
    return 1;
  }
}

}  // extern "C"
