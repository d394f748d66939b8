// The C ABI of the library (declared in include/fastpls_b200.h).
//
// The first twenty entry points keep the names, signatures, argument meaning
// and error behaviour of the reference's CUDA ABI (src/cuda_resident_api.h
// and the extern "C" shims of src/cuda_resident_api.cuh:1026-1353): return
// 0 / non-null on success, 1 / NULL on error with a NUL-terminated message
// in the caller's buffer; nothing throws across the boundary.
#include "upload.cuh"
#include "../../include/fastpls_b200.h"

#include "batched.cuh"
#include "ozaki.cuh"
#include "cv.cuh"
#include "handle.cuh"
#include "persistent.cuh"

#include <atomic>
#include <cstdio>
#include <cstring>

namespace fpls {

static std::atomic<unsigned long long> g_launches{0};
void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launch(unsigned long long n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
void keep_pool_memory() {
  static thread_local int configured_device = -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (dev == configured_device) return;
  cudaMemPool_t pool;
  size_t free_b = 0, total_b = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
      cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
    unsigned long long threshold = total_b / 2;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  cudaGetLastError();
  configured_device = dev;
}

cudaStream_t& caller_stream() {
  static cudaStream_t s = nullptr;
  return s;
}

namespace {

void write_error(char* out, size_t cap, const char* message) noexcept {
  if (out && cap) std::snprintf(out, cap, "%s", message);
}

template <class F>
int guarded(char* error, size_t cap, const char* fallback, F&& body) noexcept {
  write_error(error, cap, "");
  try {
    body();
    return 0;
  } catch (const std::exception& e) {
    write_error(error, cap, e.what());
    return 1;
  } catch (...) {
    write_error(error, cap, fallback);
    return 1;
  }
}

template <class F>
void* guarded_create(char* error, size_t cap, const char* fallback, F&& body) noexcept {
  write_error(error, cap, "");
  try {
    return body();
  } catch (const std::exception& e) {
    write_error(error, cap, e.what());
    return nullptr;
  } catch (...) {
    write_error(error, cap, fallback);
    return nullptr;
  }
}

template <class T>
void host_gemm(const T* left, const T* right, int rows, int inner, int columns,
               T* output) {
  cudaStream_t s = nullptr;
  FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct Guard {
    cudaStream_t s;
    ~Guard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } guard{s};
  DeviceArray<T> a((size_t)rows * inner, s), b((size_t)inner * columns, s);
  DeviceArray<double> c((size_t)rows * columns, s);
  FPLS_CHECK(cudaMemcpyAsync(a.get(), left, sizeof(T) * rows * inner, cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(b.get(), right, sizeof(T) * inner * columns, cudaMemcpyHostToDevice, s));
  GemmArgs g;
  g.M = rows;
  g.N = columns;
  g.K = inner;
  g.A = a.get();
  g.lda = rows;
  g.a_f32 = std::is_same<T, float>::value;
  g.B = b.get();
  g.ldb = inner;
  g.b_f32 = g.a_f32;
  g.C = c.get();
  g.ldc = rows;
  gemm_f64(g, s);
  std::vector<double> host((size_t)rows * columns);
  FPLS_CHECK(cudaMemcpyAsync(host.data(), c.get(), sizeof(double) * host.size(), cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaStreamSynchronize(s));
  for (size_t k = 0; k < host.size(); ++k) output[k] = static_cast<T>(host[k]);
}

FitRequest request(int method, const void* x, const void* y, const int* labels,
                   int n, int p, int q, int components, int scaling,
                   int oversample, int power, int retain, unsigned long long seed) {
  FitRequest r;
  r.method = method;
  r.x = x;
  r.y = y;
  r.labels = labels;
  r.n = n;
  r.p = p;
  r.q = q;
  r.components = components;
  r.scaling = scaling;
  r.oversample = oversample;
  r.power = power;
  r.retain_scores = retain == 1;
  r.seed = seed;
  return r;
}

template <class T>
void cv_permutation(const void* predictors, const void* responses,
                    const int* folds, const int* permutations,
                    int permutation_count, int n, int p, int q,
                    const int* prefixes, int prefix_count, int scaling,
                    int metric, double* metrics, double* q2, double* rmsd,
                    double* observed_r2, int* status, bool device_inputs) {
  if (!predictors || !responses || !folds || !prefixes || !metrics || n < 2 ||
      p < 1 || q < 1 || prefix_count < 1 || scaling < 1 || scaling > 3 ||
      metric < 2 || metric > 4 || permutation_count < 0 ||
      (permutation_count > 0 && !permutations))
    throw std::invalid_argument("invalid batched CUDA CV permutation input");
  cudaStream_t s = caller_stream();
  const bool own = s == nullptr;
  if (own) FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct Guard {
    cudaStream_t s;
    bool own;
    ~Guard() {
      cudaStreamSynchronize(s);
      if (own) cudaStreamDestroy(s);
    }
  } guard{s, own};
  {
    DeviceArray<T> X, Y;
    DeviceArray<int> P;
    std::vector<int> host_folds;
    const T* xd = static_cast<const T*>(predictors);
    const T* yd = static_cast<const T*>(responses);
    const int* pd = permutations;
    const int* fh = folds;
    if (!device_inputs) {
      X.allocate((size_t)n * p, s);
      Y.allocate((size_t)n * q, s);
      upload_h2d(X.get(), predictors, sizeof(T) * n * p, s);
      FPLS_CHECK(cudaMemcpyAsync(Y.get(), responses, sizeof(T) * n * q, cudaMemcpyHostToDevice, s));
      if (permutation_count > 0) {
        P.allocate((size_t)permutation_count * n, s);
        FPLS_CHECK(cudaMemcpyAsync(P.get(), permutations, sizeof(int) * permutation_count * n,
                                   cudaMemcpyHostToDevice, s));
      }
      xd = X.get();
      yd = Y.get();
      pd = P.get();
    } else {
      host_folds.resize(n);
      FPLS_CHECK(cudaMemcpyAsync(host_folds.data(), folds, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
      FPLS_CHECK(cudaStreamSynchronize(s));
      fh = host_folds.data();
    }
    BatchedCv<T> engine;
    engine.run(xd, n, p, yd, q, fh, pd, permutation_count, prefixes, prefix_count, scaling, s);
    engine.metrics(metric, metrics, q2, rmsd, observed_r2);
    if (status)
      for (size_t f = 0; f < engine.status.size(); ++f) status[f] = engine.status[f];
  }
}

// Classification CV x permutations on the batched engine: one-hot
// indicators of the (permuted) labels as responses, the argmax head over the
// classes present in each training fold (src/cuda_resident_api.cuh:620-745,
// without LDA), accuracy per permutation and prefix. Training folds must hold
// at least two classes and stay below the candidate-block threshold of
// classification SIMPLS (n_train p classes < 5e8 or fewer than 4 components),
// since the engine refreshes the direction every component.
template <class T>
void cv_permutation_classification(const T* predictors, const int* labels, const int* folds,
                                   const int* permutations, int permutation_count, int n, int p,
                                   int classes, const int* prefixes, int prefix_count,
                                   int scaling, double* accuracy, int* status, bool lda = false) {
  if (!predictors || !labels || !folds || !prefixes || !accuracy || n < 2 || p < 1 ||
      classes < 2 || classes > kBatchMaxResponses || prefix_count < 1 || scaling < 1 ||
      scaling > 3 || permutation_count < 0 || (permutation_count > 0 && !permutations))
    throw std::invalid_argument("invalid batched CUDA classification CV input");
  int folds_n = 0;
  for (int i = 0; i < n; ++i) {
    if (labels[i] < 1 || labels[i] > classes || folds[i] < 1)
      throw std::invalid_argument("invalid batched CUDA classification CV input");
    folds_n = std::max(folds_n, folds[i]);
  }
  const int kmax = prefixes[prefix_count - 1];
  const int B = permutation_count + 1;
  std::vector<int> count((size_t)classes);
  // instances whose training rows hold one class predict that class for every
  // held-out row (the reference's status 4 fold, cross_validation.hpp:
  // 1360-1788); they are counted here and not fitted
  std::vector<unsigned char> single((size_t)B * folds_n, 0);
  std::vector<int> blocks((size_t)B * folds_n, 1);
  std::vector<double> single_hits((size_t)B * folds_n, 0.0);
  for (int b = 0; b < B; ++b)
    for (int f = 1; f <= folds_n; ++f) {
      std::fill(count.begin(), count.end(), 0);
      int ntrain = 0, nheld = 0;
      for (int r = 0; r < n; ++r) {
        if (folds[r] == f) {
          ++nheld;
          continue;
        }
        const int src = b == 0 ? r : permutations[(size_t)(b - 1) * n + r];
        if (src < 0 || src >= n) throw std::invalid_argument("invalid batched CUDA classification CV input");
        ++count[labels[src] - 1];
        ++ntrain;
      }
      if (nheld == 0) continue;
      int active = 0, only = 0;
      for (int c = 0; c < classes; ++c)
        if (count[c] > 0) {
          ++active;
          only = c + 1;
        }
      if (active < 2) {
        const int predicted = active == 1 ? only : 1;
        double hits = 0.0;
        for (int r = 0; r < n; ++r) {
          if (folds[r] != f) continue;
          const int src = b == 0 ? r : permutations[(size_t)(b - 1) * n + r];
          hits += labels[src] == predicted ? 1.0 : 0.0;
        }
        single[(size_t)b * folds_n + f - 1] = 1;
        single_hits[(size_t)b * folds_n + f - 1] = hits;
        continue;
      }
      // the reference's candidate blocks (classification: n_train p classes
      // >= 5e8 and 4+ components) on this instance's training rows and its
      // active classes (src/cuda_resident_simpls.cuh:144-153)
      blocks[(size_t)b * folds_n + f - 1] = simpls_block_size(ntrain, p, active, kmax, true, false);
    }
  std::vector<T> onehot((size_t)n * classes, T(0));
  std::vector<int> zero_based(n);
  for (int i = 0; i < n; ++i) {
    onehot[(size_t)(labels[i] - 1) * n + i] = T(1);
    zero_based[i] = labels[i] - 1;
  }
  cudaStream_t s = caller_stream();
  const bool own = s == nullptr;
  if (own) FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct Guard {
    cudaStream_t s;
    bool own;
    ~Guard() {
      cudaStreamSynchronize(s);
      if (own) cudaStreamDestroy(s);
    }
  } guard{s, own};
  {
    DeviceArray<T> X((size_t)n * p, s), Y((size_t)n * classes, s);
    DeviceArray<int> P, L(n, s);
    upload_h2d(X.get(), predictors, sizeof(T) * n * p, s);
    FPLS_CHECK(cudaMemcpyAsync(Y.get(), onehot.data(), sizeof(T) * n * classes, cudaMemcpyHostToDevice, s));
    FPLS_CHECK(cudaMemcpyAsync(L.get(), zero_based.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    if (permutation_count > 0) {
      P.allocate((size_t)permutation_count * n, s);
      FPLS_CHECK(cudaMemcpyAsync(P.get(), permutations, sizeof(int) * permutation_count * n,
                                 cudaMemcpyHostToDevice, s));
    }
    BatchedCv<T> engine;
    engine.class_labels = L.get();
    engine.lda_head = lda;
    engine.skip = single;
    engine.blocks = blocks;
    engine.run(X.get(), n, p, Y.get(), classes, folds, P.get(), permutation_count, prefixes,
               prefix_count, scaling, s);
    for (int b = 0; b < B; ++b)
      for (int f = 0; f < folds_n; ++f)
        if (single[(size_t)b * folds_n + f])
          for (int j = 0; j < prefix_count; ++j)
            engine.inst_sse[((size_t)b * folds_n + f) * prefix_count + j] =
                single_hits[(size_t)b * folds_n + f];
    for (int f = 0; f < folds_n; ++f)
      if (single[f] && engine.status[f] == 1) engine.status[f] = 4;
    engine.accuracy(accuracy);
    if (status)
      for (size_t f = 0; f < engine.status.size(); ++f) status[f] = engine.status[f];
  }
}

}  // namespace
}  // namespace fpls

using namespace fpls;

extern "C" {

int fastpls_cuda_gemm(const void* left, const void* right, int precision,
                      int rows, int inner, int columns, void* output,
                      char* error, size_t error_capacity) {
  return guarded(error, error_capacity, "unknown CUDA matrix multiplication error", [&] {
    if (!left || !right || !output || (precision != 32 && precision != 64) ||
        rows < 1 || inner < 1 || columns < 1)
      throw std::invalid_argument("invalid CUDA matrix multiplication input");
    if (precision == 32)
      host_gemm(static_cast<const float*>(left), static_cast<const float*>(right), rows, inner, columns,
                static_cast<float*>(output));
    else
      host_gemm(static_cast<const double*>(left), static_cast<const double*>(right), rows, inner, columns,
                static_cast<double*>(output));
  });
}

int fastpls_resident_simpls_cv_classification(
    const void* predictors, const int* labels, const int* folds, int precision,
    int n, int p, int classes, const int* prefixes, int prefix_count,
    int scaling, int lda, int oversample, int power, unsigned long long seed,
    int store_predictions, int store_scores, int* predictions, void* scores,
    int* status, double* metrics, char* error, size_t error_capacity) {
  (void)oversample;
  (void)power;
  (void)seed;
  return guarded(error, error_capacity, "unknown resident CUDA CV error", [&] {
    if ((precision != 32 && precision != 64) || (lda != 0 && lda != 1) ||
        (store_predictions != 0 && store_predictions != 1) ||
        (store_scores != 0 && store_scores != 1))
      throw std::invalid_argument("invalid resident CUDA CV controls");
    if (precision == 32)
      cv_classification<float>(kSimpls, static_cast<const float*>(predictors), labels, folds, n, p, classes,
                               prefixes, prefix_count, scaling, lda == 1, store_predictions == 1,
                               store_scores == 1, predictions, static_cast<float*>(scores), status, metrics);
    else
      cv_classification<double>(kSimpls, static_cast<const double*>(predictors), labels, folds, n, p, classes,
                                prefixes, prefix_count, scaling, lda == 1, store_predictions == 1,
                                store_scores == 1, predictions, static_cast<double*>(scores), status, metrics);
  });
}

int fastpls_resident_simpls_cv_regression(
    const void* predictors, const void* responses, const int* folds,
    int precision, int n, int p, int q, const int* prefixes, int prefix_count,
    int scaling, int metric, int oversample, int power, unsigned long long seed,
    int store_predictions, double* predictions, int* status, double* metrics,
    double* q2, double* rmsd, double* observed_r2, char* error,
    size_t error_capacity) {
  (void)oversample;
  (void)power;
  (void)seed;
  return guarded(error, error_capacity, "unknown resident CUDA regression CV error", [&] {
    if ((precision != 32 && precision != 64) || !q2 || !rmsd || !observed_r2 ||
        (store_predictions != 0 && store_predictions != 1))
      throw std::invalid_argument("invalid resident CUDA regression CV controls");
    if (precision == 32)
      cv_regression<float>(kSimpls, static_cast<const float*>(predictors), static_cast<const float*>(responses),
                           folds, n, p, q, prefixes, prefix_count, scaling, metric, store_predictions == 1,
                           predictions, status, metrics, q2, rmsd, observed_r2);
    else
      cv_regression<double>(kSimpls, static_cast<const double*>(predictors), static_cast<const double*>(responses),
                            folds, n, p, q, prefixes, prefix_count, scaling, metric, store_predictions == 1,
                            predictions, status, metrics, q2, rmsd, observed_r2);
  });
}

int fastpls_resident_plssvd_cv_classification(
    const void* predictors, const int* labels, const int* folds, int precision,
    int n, int p, int classes, const int* prefixes, int prefix_count,
    int scaling, int lda, int oversample, int power, unsigned long long seed,
    int store_predictions, int store_scores, int* predictions, void* scores,
    int* status, double* metrics, char* error, size_t error_capacity) {
  (void)oversample;
  (void)power;
  (void)seed;
  return guarded(error, error_capacity, "unknown resident CUDA PLS-SVD CV error", [&] {
    if ((precision != 32 && precision != 64) || (lda != 0 && lda != 1) ||
        (store_predictions != 0 && store_predictions != 1) ||
        (store_scores != 0 && store_scores != 1))
      throw std::invalid_argument("invalid resident CUDA PLS-SVD CV controls");
    if (precision == 32)
      cv_classification<float>(kPlssvd, static_cast<const float*>(predictors), labels, folds, n, p, classes,
                               prefixes, prefix_count, scaling, lda == 1, store_predictions == 1,
                               store_scores == 1, predictions, static_cast<float*>(scores), status, metrics);
    else
      cv_classification<double>(kPlssvd, static_cast<const double*>(predictors), labels, folds, n, p, classes,
                                prefixes, prefix_count, scaling, lda == 1, store_predictions == 1,
                                store_scores == 1, predictions, static_cast<double*>(scores), status, metrics);
  });
}

int fastpls_resident_plssvd_cv_regression(
    const void* predictors, const void* responses, const int* folds,
    int precision, int n, int p, int q, const int* prefixes, int prefix_count,
    int scaling, int metric, int oversample, int power, unsigned long long seed,
    int store_predictions, double* predictions, int* status, double* metrics,
    double* q2, double* rmsd, double* observed_r2, char* error,
    size_t error_capacity) {
  (void)oversample;
  (void)power;
  (void)seed;
  return guarded(error, error_capacity, "unknown resident CUDA PLS-SVD regression CV error", [&] {
    if ((precision != 32 && precision != 64) || !q2 || !rmsd || !observed_r2 ||
        (store_predictions != 0 && store_predictions != 1))
      throw std::invalid_argument("invalid resident CUDA PLS-SVD regression CV controls");
    if (precision == 32)
      cv_regression<float>(kPlssvd, static_cast<const float*>(predictors), static_cast<const float*>(responses),
                           folds, n, p, q, prefixes, prefix_count, scaling, metric, store_predictions == 1,
                           predictions, status, metrics, q2, rmsd, observed_r2);
    else
      cv_regression<double>(kPlssvd, static_cast<const double*>(predictors), static_cast<const double*>(responses),
                            folds, n, p, q, prefixes, prefix_count, scaling, metric, store_predictions == 1,
                            predictions, status, metrics, q2, rmsd, observed_r2);
  });
}

void* fastpls_resident_simpls_create(const void* x, const void* y, const int* labels,
                                     int precision, int n, int p, int q, int components,
                                     int scaling, int oversample, int power, int retain_scores,
                                     unsigned long long seed, char* error, size_t error_capacity) {
  return guarded_create(error, error_capacity, "unknown resident CUDA fitting error", [&]() -> void* {
    if (!x || (precision != 32 && precision != 64 && precision != 16))
      throw std::invalid_argument("invalid resident matrix or precision");
    if (retain_scores != 0 && retain_scores != 1)
      throw std::invalid_argument("invalid resident score-retention request");
    return make_handle(precision, request(kSimpls, x, y, labels, n, p, q, components, scaling,
                                          oversample, power, retain_scores, seed));
  });
}

void* fastpls_b200_model_import(int method, int precision, int n, int p, int q, int components,
                                int scaling, int classification, const double* weights,
                                const double* response_loadings, const double* scores,
                                const double* mean_x, const double* scale_x, const double* mean_y,
                                const int* labels, char* error, size_t error_capacity) {
  return guarded_create(error, error_capacity, "unknown resident CUDA import error", [&]() -> void* {
    if (precision != 32 && precision != 64 && precision != 16)
      throw std::invalid_argument("invalid resident matrix or precision");
    fpls::ImportRequest im;
    im.method = method;
    im.n = n;
    im.p = p;
    im.q = q;
    im.components = components;
    im.scaling = scaling;
    im.classification = classification != 0;
    im.R = weights;
    im.Q = response_loadings;
    im.T = scores;
    im.mean = mean_x;
    im.scale = scale_x;
    im.ymean = mean_y;
    im.labels = labels;
    return fpls::import_handle(precision, im);
  });
}

void* fastpls_resident_plssvd_create(const void* x, const void* y, const int* labels,
                                     int precision, int n, int p, int q, int components,
                                     int scaling, int oversample, int power, int retain_scores,
                                     unsigned long long seed, char* error, size_t error_capacity) {
  return guarded_create(error, error_capacity, "unknown resident CUDA PLS-SVD fitting error", [&]() -> void* {
    if (!x || (precision != 32 && precision != 64 && precision != 16))
      throw std::invalid_argument("invalid resident matrix or precision");
    if (retain_scores != 0 && retain_scores != 1)
      throw std::invalid_argument("invalid resident score-retention request");
    return make_handle(precision, request(kPlssvd, x, y, labels, n, p, q, components, scaling,
                                          oversample, power, retain_scores, seed));
  });
}

void* fastpls_resident_opls_create(const void* x, const void* y, const int* labels,
                                   int precision, int n, int p, int q, int components,
                                   int scaling, int oversample, int power, int retain_scores,
                                   unsigned long long seed, int north, char* error,
                                   size_t error_capacity) {
  return guarded_create(error, error_capacity, "unknown resident CUDA OPLS fitting error", [&]() -> void* {
    if (!x || (precision != 32 && precision != 64 && precision != 16) || north < 0)
      throw std::invalid_argument("invalid resident CUDA OPLS input");
    FitRequest r = request(kOpls, x, y, labels, n, p, q, components, scaling, oversample, power,
                           retain_scores, seed);
    r.north = north;
    return make_handle(precision, r);
  });
}

void* fastpls_resident_kernelpls_create(const void* x, const void* y, const int* labels,
                                        int precision, int n, int p, int q, int components,
                                        int scaling, int oversample, int power, int retain_scores,
                                        unsigned long long seed, int kernel, double gamma,
                                        int degree, double coef0, char* error,
                                        size_t error_capacity) {
  return guarded_create(error, error_capacity, "unknown resident CUDA nonlinear kernel PLS fitting error",
                        [&]() -> void* {
    if (!x || (precision != 32 && precision != 64 && precision != 16) || (kernel != 2 && kernel != 3))
      throw std::invalid_argument("invalid resident CUDA nonlinear kernel PLS input");
    FitRequest r = request(kKernelPls, x, y, labels, n, p, q, components, scaling, oversample, power,
                           retain_scores, seed);
    r.kernel = kernel;
    r.gamma = gamma;
    r.degree = degree;
    r.coef0 = coef0;
    return make_handle(precision, r);
  });
}

int fastpls_resident_predict_path(void* model, const void* x, int rows, const int* prefixes,
                                  int prefix_count, int lda, void* predictions, char* error,
                                  size_t error_capacity) {
  return guarded(error, error_capacity, "unknown resident prediction-path error", [&] {
    if (!model || (lda != 0 && lda != 1))
      throw std::invalid_argument("invalid resident prediction-path model");
    static_cast<ResidentHandle*>(model)->predict_path(x, rows, prefixes, prefix_count, lda == 1, predictions);
  });
}

void fastpls_resident_simpls_destroy(void* model) {
  delete static_cast<ResidentHandle*>(model);
}

int fastpls_resident_export(void* model, int field, void* out, size_t elements, char* error,
                            size_t error_capacity) {
  return guarded(error, error_capacity, "unknown resident export error", [&] {
    if (!model) throw std::invalid_argument("null resident model");
    static_cast<ResidentHandle*>(model)->export_field(field, out, elements);
  });
}

int fastpls_resident_classify_path(void* model, const void* x, int rows, const int* prefixes,
                                   int prefix_count, int lda, int top, int* labels, char* error,
                                   size_t error_capacity) {
  return guarded(error, error_capacity, "unknown resident classification-path error", [&] {
    if (!model || (lda != 0 && lda != 1))
      throw std::invalid_argument("invalid resident classification-path model");
    static_cast<ResidentHandle*>(model)->classify_path(x, rows, prefixes, prefix_count, lda == 1, top,
                                                       labels, nullptr);
  });
}

int fastpls_resident_classify_response_path(void* model, const void* x, int rows,
                                            const int* prefixes, int prefix_count, int lda, int top,
                                            int* labels, void* predictions, char* error,
                                            size_t error_capacity) {
  return guarded(error, error_capacity, "unknown resident classification-response path error", [&] {
    if (!model) throw std::invalid_argument("null resident model");
    if (!predictions)
      throw std::invalid_argument("invalid resident classification-response path request");
    static_cast<ResidentHandle*>(model)->classify_path(x, rows, prefixes, prefix_count, lda != 0, top,
                                                       labels, predictions);
  });
}

int fastpls_resident_response_sums(void* model, const void* x, const void* y, const int* labels,
                                   int rows, int prefix, void* out, char* error,
                                   size_t error_capacity) {
  return guarded(error, error_capacity, "unknown resident metric error", [&] {
    if (!model) throw std::invalid_argument("null resident model");
    static_cast<ResidentHandle*>(model)->response_sums(x, y, labels, rows, prefix, out);
  });
}

int fastpls_resident_project(void* model, const void* x, int rows, int prefix, void* out,
                             char* error, size_t error_capacity) {
  return guarded(error, error_capacity, "unknown resident projection error", [&] {
    if (!model) throw std::invalid_argument("null resident model");
    static_cast<ResidentHandle*>(model)->project(x, rows, prefix, out);
  });
}

int fastpls_resident_controls(void* model, int* oversample, int* power, int* block,
                              int* block_limit, int* implicit_operator,
                              int* predictor_crossprod_cache, char* error,
                              size_t error_capacity) {
  return guarded(error, error_capacity, "unknown resident control error", [&] {
    if (!model) throw std::invalid_argument("null resident model");
    static_cast<ResidentHandle*>(model)->controls(oversample, power, block, block_limit,
                                                  implicit_operator, predictor_crossprod_cache);
  });
}

int fastpls_resident_compact(void* model, int prepare_lda, char* error, size_t error_capacity) {
  return guarded(error, error_capacity, "unknown resident compaction error", [&] {
    if (!model || (prepare_lda != 0 && prepare_lda != 1))
      throw std::invalid_argument("invalid resident compaction request");
    static_cast<ResidentHandle*>(model)->compact(prepare_lda == 1);
  });
}

// ------------------------------------------------------------------ additions
int fastpls_b200_resident_vip(void* model, double* out, size_t size, char* error,
                              size_t error_capacity) {
  return guarded(error, error_capacity, "unknown VIP calculation error", [&] {
    if (!model) throw std::invalid_argument("VIP requires a fitted fastPLS model");
    static_cast<ResidentHandle*>(model)->vip(out, size);
  });
}

int fastpls_b200_device_count(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return count;
}

unsigned long long fastpls_b200_launch_count(void) { return launch_count(); }

void fastpls_b200_set_stream(void* stream) {
  caller_stream() = static_cast<cudaStream_t>(stream);
}

void fastpls_b200_profile_gemm(int enable) { gemm_profile_enable(enable != 0); }

int fastpls_b200_fp64_peak(double* tflops, char* error, size_t error_capacity) {
  return guarded(error, error_capacity, "unknown probe error", [&] {
    if (!tflops) throw std::invalid_argument("null output");
    *tflops = fp64_fma_tflops();
  });
}

void fastpls_b200_profile_gemm_read(double* milliseconds, double* flops,
                                    unsigned long long* launches) {
  gemm_profile_read(milliseconds, flops, launches);
}

void fastpls_b200_set_product_digits(int digits) {
  ozaki_slices() = std::max(0, std::min(digits, kOzakiMaxSlices));
}

int fastpls_b200_product_digits(void) { return ozaki_slices(); }

void fastpls_b200_set_batch_lanes(int lanes) { batch_lanes() = std::max(1, std::min(lanes, 4)); }

int fastpls_b200_batch_lanes(void) { return batch_lanes(); }

void fastpls_b200_set_argmax_guard(double margin) {
  argmax_guard() = (margin > 0.0 && std::isfinite(margin)) ? margin : 0.0;
}

double fastpls_b200_argmax_guard(void) { return argmax_guard(); }

int fastpls_b200_guard_refits(void) { return last_guard_refits(); }

void fastpls_b200_last_fit_times(double* copy_ms, double* fit_ms) {
  read_last_fit_times(copy_ms, fit_ms);
}

void fastpls_b200_set_persistent(int enable) { persistent_enabled() = enable ? 1 : 0; }

int fastpls_b200_persistent(void) { return persistent_enabled(); }

void fastpls_b200_int8_wait_test(int skip_last_stage, long long wait_cycles) {
  ozaki_wait_test().skip_last = skip_last_stage ? 1 : 0;
  ozaki_wait_test().cycles = wait_cycles;
}

void fastpls_b200_persistent_wait_test(int absent_cta, long long wait_cycles) {
  persistent_wait_test().absent = absent_cta ? 1 : 0;
  persistent_wait_test().cycles = wait_cycles;
}

void fastpls_b200_set_autotune(int enable) { batch_autotune() = enable ? 1 : 0; }

int fastpls_b200_autotune(void) { return batch_autotune(); }

void fastpls_b200_batched_stats(int* groups, int* graph_replays, int* graph_captures, int* tuned,
                                int* lanes, int* tile_n) {
  const BatchedStats& s = last_batched_stats();
  if (groups) *groups = s.groups;
  if (graph_replays) *graph_replays = s.graph_replays;
  if (graph_captures) *graph_captures = s.graph_captures;
  if (tuned) *tuned = s.tuned;
  if (lanes) *lanes = s.lanes;
  if (tile_n) *tile_n = s.tile_n;
}

void fastpls_b200_release_workspace(void) { release_batched_workspace(); }

void fastpls_b200_profile_int8(int enable) { ozaki_profile_enable(enable != 0); }

void fastpls_b200_profile_int8_read(double* milliseconds, double* int8_ops,
                                    unsigned long long* launches) {
  ozaki_profile_read(milliseconds, int8_ops, launches);
}

int fastpls_b200_int8_crossprod(const double* a, int lda, const double* b, int ldb, int m,
                                int n, int k, int digits, int symmetric, int tile_n, int pair,
                                double* c, int ldc, char* error, size_t error_capacity) {
  return guarded(error, error_capacity, "unknown int8 split product error", [&] {
    if (!a || !b || !c || m < 1 || n < 1 || k < 0 || lda < std::max(k, 1) ||
        ldb < std::max(k, 1) || ldc < m || digits < 1 || digits > kOzakiMaxSlices ||
        (tile_n != 0 && tile_n != 128 && tile_n != 192 && tile_n != 256) ||
        (symmetric && tile_n != 0 && tile_n != 128) || pair < -1 || pair > 1 ||
        (pair == 1 && (symmetric || tile_n == 128)))
      throw std::invalid_argument("invalid int8 split product input");
    if (symmetric && (a != b || m != n || lda != ldb))
      throw std::invalid_argument("symmetric int8 split product needs one operand");
    if (k == 0) {
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) c[i + (size_t)j * ldc] = 0.0;
      return;
    }
    cudaStream_t s = nullptr;
    FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct Guard {
      cudaStream_t s;
      ~Guard() {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    } guard{s};
    DeviceArray<double> da((size_t)lda * m, s), db, dc((size_t)m * n, s);
    DeviceArray<int> flag(1, s);
    flag.zero(s);
    FPLS_CHECK(cudaMemcpyAsync(da.get(), a, sizeof(double) * lda * m, cudaMemcpyHostToDevice, s));
    OzakiOperand oa, ob;
    ozaki_split_rows(da.get(), lda, m, k, digits, oa, flag.get(), s);
    if (symmetric) {
      ozaki_gemm(oa, oa, dc.get(), m, true, flag.get(), s);
    } else {
      db.allocate((size_t)ldb * n, s);
      FPLS_CHECK(cudaMemcpyAsync(db.get(), b, sizeof(double) * ldb * n, cudaMemcpyHostToDevice, s));
      ozaki_split_rows(db.get(), ldb, n, k, digits, ob, flag.get(), s);
      ozaki_gemm(oa, ob, dc.get(), m, false, flag.get(), s, tile_n, pair);
    }
    int bad = 0;
    FPLS_CHECK(cudaMemcpyAsync(&bad, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    FPLS_CHECK(cudaMemcpy2DAsync(c, sizeof(double) * ldc, dc.get(), sizeof(double) * m,
                                 sizeof(double) * m, n, cudaMemcpyDeviceToHost, s));
    FPLS_CHECK(cudaStreamSynchronize(s));
    if (bad == 4) throw std::runtime_error("int8 split product: tensor-core pipeline wait timed out");
    if (bad) throw std::runtime_error("int8 split product: non-finite input");
  });
}

int fastpls_b200_simpls_cv_permutation(
    const void* predictors, const void* responses, const int* folds,
    const int* permutations, int permutation_count, int precision, int n,
    int p, int q, const int* prefixes, int prefix_count, int scaling,
    int metric, double* metrics, double* q2, double* rmsd, double* observed_r2,
    int* status, char* error, size_t error_capacity) {
  return guarded(error, error_capacity, "unknown batched CUDA CV error", [&] {
    if (precision != 32 && precision != 64)
      throw std::invalid_argument("invalid batched CUDA CV precision");
    if (precision == 32)
      cv_permutation<float>(predictors, responses, folds, permutations, permutation_count, n, p, q,
                            prefixes, prefix_count, scaling, metric, metrics, q2, rmsd, observed_r2,
                            status, false);
    else
      cv_permutation<double>(predictors, responses, folds, permutations, permutation_count, n, p, q,
                             prefixes, prefix_count, scaling, metric, metrics, q2, rmsd, observed_r2,
                             status, false);
  });
}

int fastpls_b200_simpls_cv_permutation_classification(
    const void* predictors, const int* labels, const int* folds, const int* permutations,
    int permutation_count, int precision, int n, int p, int classes, const int* prefixes,
    int prefix_count, int scaling, double* accuracy, int* status, char* error,
    size_t error_capacity) {
  return guarded(error, error_capacity, "unknown batched CUDA CV error", [&] {
    if (precision != 32 && precision != 64)
      throw std::invalid_argument("invalid batched CUDA CV precision");
    if (precision == 32)
      cv_permutation_classification<float>(static_cast<const float*>(predictors), labels, folds,
                                           permutations, permutation_count, n, p, classes, prefixes,
                                           prefix_count, scaling, accuracy, status);
    else
      cv_permutation_classification<double>(static_cast<const double*>(predictors), labels, folds,
                                            permutations, permutation_count, n, p, classes,
                                            prefixes, prefix_count, scaling, accuracy, status);
  });
}

int fastpls_b200_simpls_cv_permutation_classification_head(
    const void* predictors, const int* labels, const int* folds, const int* permutations,
    int permutation_count, int precision, int n, int p, int classes, const int* prefixes,
    int prefix_count, int scaling, int lda, double* accuracy, int* status, char* error,
    size_t error_capacity) {
  return guarded(error, error_capacity, "unknown batched CUDA CV error", [&] {
    if (precision != 32 && precision != 64)
      throw std::invalid_argument("invalid batched CUDA CV precision");
    if (lda != 0 && lda != 1) throw std::invalid_argument("invalid batched CUDA CV head");
    if (precision == 32)
      cv_permutation_classification<float>(static_cast<const float*>(predictors), labels, folds,
                                           permutations, permutation_count, n, p, classes, prefixes,
                                           prefix_count, scaling, accuracy, status, lda != 0);
    else
      cv_permutation_classification<double>(static_cast<const double*>(predictors), labels, folds,
                                            permutations, permutation_count, n, p, classes,
                                            prefixes, prefix_count, scaling, accuracy, status,
                                            lda != 0);
  });
}

int fastpls_b200_simpls_cv_permutation_device(
    const void* predictors, const void* responses, const int* folds,
    const int* permutations, int permutation_count, int precision, int n,
    int p, int q, const int* prefixes, int prefix_count, int scaling,
    int metric, double* metrics, double* q2, double* rmsd, double* observed_r2,
    int* status, char* error, size_t error_capacity) {
  return guarded(error, error_capacity, "unknown batched CUDA CV error", [&] {
    if (precision != 32 && precision != 64)
      throw std::invalid_argument("invalid batched CUDA CV precision");
    if (precision == 32)
      cv_permutation<float>(predictors, responses, folds, permutations, permutation_count, n, p, q,
                            prefixes, prefix_count, scaling, metric, metrics, q2, rmsd, observed_r2,
                            status, true);
    else
      cv_permutation<double>(predictors, responses, folds, permutations, permutation_count, n, p, q,
                             prefixes, prefix_count, scaling, metric, metrics, q2, rmsd, observed_r2,
                             status, true);
  });
}

}  // extern "C"
