// Cross-validation drivers behind the reference's CV entry points
// (fastpls_resident_{simpls,plssvd}_cv_{regression,classification}).
//
// Behavioural contract: src/cuda_resident_api.cuh:538-1023 of the reference
// (validation and messages, fold status codes 1/2/4, metric assembly in long
// double, prediction and score output layouts). X and Y are uploaded once;
// each fold's training and held-out rows are gathered on the device and the
// fold model is fitted by the resident engine (fit.cu / plssvd.cu).
// Folds run one after another here; the many-fold / many-permutation batched
// engine lives in batched.cu.
#include "upload.cuh"
#include "cv.cuh"
#include "handle.cuh"
#include "lda.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

namespace fpls {

namespace {

__global__ void fold_sums_kernel(const double* __restrict__ pred,
                                 const double* __restrict__ y,
                                 const double* __restrict__ ymean, int n,
                                 int q, double* out) {
  __shared__ double scratch[32];
  const int c = blockIdx.x;
  double sse = 0.0, st = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = y[i + (long)c * n];
    const double e = v - pred[i + (long)c * n], d = v - ymean[c];
    sse = fma(e, e, sse);
    st = fma(d, d, st);
  }
  sse = block_sum(sse, scratch);
  st = block_sum(st, scratch);
  if (threadIdx.x == 0) {
    out[2 * c] = sse;
    out[2 * c + 1] = st;
  }
}

template <class T>
__global__ void to_f64_kernel(const T* __restrict__ in, long count, double* out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x)
    out[i] = as_f64(in[i]);
}

struct Folds {
  int count = 0;
  std::vector<std::vector<int>> test;
  int max_test = 0, max_train = 0;
};

Folds partition(const int* folds, int n) {
  Folds f;
  for (int i = 0; i < n; ++i) f.count = std::max(f.count, folds[i]);
  f.test.assign(f.count, {});
  for (int i = 0; i < n; ++i) f.test[folds[i] - 1].push_back(i);
  for (const auto& t : f.test) {
    f.max_test = std::max(f.max_test, (int)t.size());
    f.max_train = std::max(f.max_train, n - (int)t.size());
  }
  return f;
}

template <class T>
void fit_method(int method, const T* X, int n, int p, const double* Yc,
                const double* ycsum, int m, int a, int scaling,
                DeviceModel& model, Workspace& ws, cudaStream_t s) {
  if (method == kPlssvd) fit_plssvd<T>(X, n, p, n, Yc, ycsum, m, a, scaling, model, ws, s);
  else fit_simpls<T>(X, n, p, n, Yc, ycsum, m, a, scaling, model, ws, s,
                     simpls_block_size(n, p, m, a, model.classification, std::is_same<T, float>::value),
                     simpls_gram_route(n, p, a, model.classification));
}

}  // namespace

template <class T>
void cv_regression(int method, const T* predictors, const T* responses,
                   const int* folds, int n, int p, int q, const int* prefixes,
                   int prefix_count, int scaling, int metric,
                   bool store_predictions, double* prediction_output,
                   int* status, double* metrics, double* q2_values,
                   double* rmsd_values, double* observed_r2_values) {
  if (!predictors || !responses || !folds || !prefixes || !status || !metrics ||
      n < 2 || p < 1 || q < 1 || prefix_count < 1 || scaling < 1 ||
      scaling > 3 || metric < 2 || metric > 4)
    throw std::invalid_argument("invalid resident CUDA regression CV input");
  int maximum_prefix = 0;
  for (int j = 0; j < prefix_count; ++j) {
    if (prefixes[j] <= maximum_prefix)
      throw std::invalid_argument("CUDA CV component path must be strictly increasing");
    maximum_prefix = prefixes[j];
  }
  for (int i = 0; i < n; ++i)
    if (folds[i] < 1) throw std::invalid_argument("invalid CUDA CV fold");
  if (maximum_prefix > std::min(n - 1, p) || (store_predictions && !prediction_output))
    throw std::invalid_argument("invalid CUDA regression CV output or rank");
  Folds fp = partition(folds, n);
  if (fp.max_test < 1 || fp.max_train < 2)
    throw std::invalid_argument("CUDA CV contains an empty train or test fold");

  long double total_ss = 0.0L;
  for (int c = 0; c < q; ++c) {
    long double s = 0.0L, ss = 0.0L;
    for (int i = 0; i < n; ++i) {
      const long double v = responses[(size_t)c * n + i];
      s += v;
      ss += v * v;
    }
    total_ss += ss - s * s / n;
  }

  cudaStream_t s = nullptr;
  FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    }
  } guard{s};
  {
    DeviceArray<T> X((size_t)n * p, s), Y((size_t)n * q, s);
    upload_h2d(X.get(), predictors, sizeof(T) * n * p, s);
    FPLS_CHECK(cudaMemcpyAsync(Y.get(), responses, sizeof(T) * n * q, cudaMemcpyHostToDevice, s));
    DeviceArray<double> Y64((size_t)n * q, s);
    to_f64_kernel<T><<<std::min<unsigned>(ceil_div((size_t)n * q, 256), 4 * num_sms()), 256, 0, s>>>(Y.get(), (long)n * q, Y64.get());
    count_launch();
    DeviceArray<T> Xtr((size_t)fp.max_train * p, s), Xte((size_t)fp.max_test * p, s);
    DeviceArray<T> Ytr((size_t)fp.max_train * q, s);
    DeviceArray<double> Yte((size_t)fp.max_test * q, s);
    DeviceArray<int> idx_tr(fp.max_train, s), idx_te(fp.max_test, s);
    DeviceArray<double> Yc((size_t)fp.max_train * q, s), ycsum(q, s);
    DeviceArray<double> scores((size_t)fp.max_test * maximum_prefix, s);
    DeviceArray<double> pred((size_t)fp.max_test * q, s);
    DeviceArray<double> sums((size_t)2 * q * prefix_count, s);
    Workspace ws;
    ws.ensure(fp.max_train, p, q, maximum_prefix, s);

    std::fill(metrics, metrics + prefix_count, 0.0);
    std::vector<double> counts(prefix_count, 0.0), fold_ss(prefix_count, 0.0);
    std::vector<double> host_sums((size_t)2 * q * prefix_count);
    std::vector<double> host_pred;
    std::vector<int> train;
    for (int f = 0; f < fp.count; ++f) {
      const auto& held = fp.test[f];
      if (held.empty()) {
        status[f] = 2;
        continue;
      }
      std::vector<char> flag(n, 0);
      for (int r : held) flag[r] = 1;
      train.clear();
      for (int i = 0; i < n; ++i)
        if (!flag[i]) train.push_back(i);
      const int ntr = (int)train.size(), nte = (int)held.size();
      if (maximum_prefix > std::min(ntr - 1, p))
        throw std::invalid_argument("CUDA CV component count exceeds a fold rank");
      FPLS_CHECK(cudaMemcpyAsync(idx_tr.get(), train.data(), sizeof(int) * ntr, cudaMemcpyHostToDevice, s));
      FPLS_CHECK(cudaMemcpyAsync(idx_te.get(), held.data(), sizeof(int) * nte, cudaMemcpyHostToDevice, s));
      gather_rows<T>(X.get(), n, p, idx_tr.get(), ntr, Xtr.get(), ntr, s);
      gather_rows<T>(X.get(), n, p, idx_te.get(), nte, Xte.get(), nte, s);
      gather_rows<T>(Y.get(), n, q, idx_tr.get(), ntr, Ytr.get(), ntr, s);
      gather_rows<double>(Y64.get(), n, q, idx_te.get(), nte, Yte.get(), nte, s);
      FPLS_CHECK(cudaMemsetAsync(ws.flag.get(), 0, sizeof(int), s));
      DeviceModel model;
      model.ymean.allocate(q, s);
      prepare_responses<T>(Ytr.get(), nullptr, ntr, q, Yc.get(), model.ymean.get(), ycsum.get(), ws.flag.get(), s);
      fit_method<T>(method, Xtr.get(), ntr, p, Yc.get(), ycsum.get(), q, maximum_prefix, scaling, model, ws, s);
      project_rows<T>(model, Xte.get(), nte, nte, maximum_prefix, scores.get(), nte, ws, s);
      if (store_predictions) host_pred.resize((size_t)nte * q * prefix_count);
      for (int j = 0; j < prefix_count; ++j) {
        predict_from_scores(model, scores.get(), nte, nte, prefixes[j], pred.get(), nte, s);
        if (store_predictions)
          FPLS_CHECK(cudaMemcpyAsync(host_pred.data() + (size_t)j * nte * q, pred.get(),
                                     sizeof(double) * nte * q, cudaMemcpyDeviceToHost, s));
        fold_sums_kernel<<<q, 256, 0, s>>>(pred.get(), Yte.get(), model.ymean.get(), nte, q,
                                           sums.get() + (size_t)2 * q * j);
        count_launch();
        FPLS_LAUNCH("fold_sums");
      }
      FPLS_CHECK(cudaMemcpyAsync(host_sums.data(), sums.get(), sizeof(double) * 2 * q * prefix_count,
                                 cudaMemcpyDeviceToHost, s));
      raise_on_flag(ws, s, method == kPlssvd
          ? "resident PLS-SVD failed: invalid labels, decomposition or score Gram"
          : "resident SIMPLS failed: invalid labels, decomposition or component norm");
      for (int j = 0; j < prefix_count; ++j) {
        long double sse = 0.0L, tss = 0.0L;
        for (int c = 0; c < q; ++c) {
          sse += host_sums[(size_t)2 * q * j + 2 * c];
          tss += host_sums[(size_t)2 * q * j + 2 * c + 1];
        }
        metrics[j] += (double)sse;
        fold_ss[j] += (double)tss;
        counts[j] += (double)nte * q;
        if (store_predictions)
          for (int c = 0; c < q; ++c)
            for (int i = 0; i < nte; ++i)
              prediction_output[(size_t)j * n * q + (size_t)c * n + held[i]] =
                  host_pred[(size_t)j * nte * q + (size_t)c * nte + i];
      }
      status[f] = 1;
    }
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (int j = 0; j < prefix_count; ++j) {
      const double sse = metrics[j];
      const double rmsd = counts[j] > 0.0 ? std::sqrt(sse / counts[j]) : nan;
      const double q2 = fold_ss[j] > 0.0 ? 1.0 - sse / fold_ss[j] : nan;
      const double r2 = total_ss > 0.0L ? 1.0 - sse / (double)total_ss : nan;
      if (rmsd_values) rmsd_values[j] = rmsd;
      if (q2_values) q2_values[j] = q2;
      if (observed_r2_values) observed_r2_values[j] = r2;
      metrics[j] = metric == 4 ? rmsd : metric == 3 ? q2 : r2;
    }
    FPLS_CHECK(cudaStreamSynchronize(s));
  }
}

template <class T>
void cv_classification(int method, const T* predictors, const int* labels,
                       const int* folds, int n, int p, int classes,
                       const int* prefixes, int prefix_count, int scaling,
                       bool use_lda, bool store_predictions, bool store_scores,
                       int* prediction_output, T* score_output, int* status,
                       double* metrics) {
  if (!predictors || !labels || !folds || !prefixes || !status || !metrics ||
      n < 2 || p < 1 || classes < 2 || prefix_count < 1 || scaling < 1 || scaling > 3)
    throw std::invalid_argument("invalid resident CUDA CV input");
  int maximum_prefix = 0;
  for (int j = 0; j < prefix_count; ++j) {
    if (prefixes[j] <= maximum_prefix)
      throw std::invalid_argument("CUDA CV component path must be strictly increasing");
    maximum_prefix = prefixes[j];
  }
  for (int i = 0; i < n; ++i)
    if (labels[i] < 1 || labels[i] > classes || folds[i] < 1)
      throw std::invalid_argument("invalid CUDA CV label or fold");
  if (maximum_prefix > std::min(n - 1, p))
    throw std::invalid_argument("CUDA CV component count exceeds rank");
  if (store_predictions && !prediction_output)
    throw std::invalid_argument("null CUDA CV prediction output");
  if (store_scores && !score_output)
    throw std::invalid_argument("null CUDA CV score output");
  Folds fp = partition(folds, n);
  if (fp.max_test < 1 || fp.max_train < 2)
    throw std::invalid_argument("CUDA CV contains an empty train or test fold");

  cudaStream_t s = nullptr;
  FPLS_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    }
  } guard{s};
  {
    DeviceArray<T> X((size_t)n * p, s);
    upload_h2d(X.get(), predictors, sizeof(T) * n * p, s);
    DeviceArray<T> Xtr((size_t)fp.max_train * p, s), Xte((size_t)fp.max_test * p, s);
    DeviceArray<int> idx_tr(fp.max_train, s), idx_te(fp.max_test, s);
    DeviceArray<int> lab_tr(fp.max_train, s), top(fp.max_test, s);
    DeviceArray<double> Yc((size_t)fp.max_train * classes, s), ycsum(classes, s);
    DeviceArray<double> scores((size_t)fp.max_test * maximum_prefix, s);
    DeviceArray<double> pred((size_t)fp.max_test * classes, s), disc((size_t)fp.max_test * classes, s);
    Workspace ws;
    ws.ensure(fp.max_train, p, classes, maximum_prefix, s);
    std::fill(metrics, metrics + prefix_count, 0.0);
    std::vector<double> counts(prefix_count, 0.0);
    if (store_scores) std::fill(score_output, score_output + (size_t)n * classes * prefix_count, T(0));
    std::vector<int> train, host_labels;
    std::vector<double> host_scores;
    for (int f = 0; f < fp.count; ++f) {
      const auto& held = fp.test[f];
      if (held.empty()) {
        status[f] = 2;
        continue;
      }
      std::vector<char> flag(n, 0);
      for (int r : held) flag[r] = 1;
      train.clear();
      std::vector<int> cnt(classes, 0);
      for (int i = 0; i < n; ++i)
        if (!flag[i]) {
          train.push_back(i);
          ++cnt[labels[i] - 1];
        }
      std::vector<int> active, active_map(classes, -1);
      for (int c = 0; c < classes; ++c)
        if (cnt[c] > 0) {
          active_map[c] = (int)active.size();
          active.push_back(c + 1);
        }
      if (active.size() <= 1) {
        const int fallback = active.empty() ? 1 : active.front();
        for (int j = 0; j < prefix_count; ++j)
          for (int r : held) {
            if (store_predictions) prediction_output[(size_t)j * n + r] = fallback;
            metrics[j] += labels[r] == fallback ? 1.0 : 0.0;
            counts[j] += 1.0;
          }
        status[f] = 4;
        continue;
      }
      const int ntr = (int)train.size(), nte = (int)held.size();
      const int c = (int)active.size();
      if (maximum_prefix > std::min(ntr - 1, p))
        throw std::invalid_argument("CUDA CV component count exceeds a fold rank");
      std::vector<int> compact(ntr);
      std::vector<int> ccount(c, 0);
      for (int i = 0; i < ntr; ++i) {
        compact[i] = active_map[labels[train[i]] - 1] + 1;
        ++ccount[compact[i] - 1];
      }
      FPLS_CHECK(cudaMemcpyAsync(idx_tr.get(), train.data(), sizeof(int) * ntr, cudaMemcpyHostToDevice, s));
      FPLS_CHECK(cudaMemcpyAsync(idx_te.get(), held.data(), sizeof(int) * nte, cudaMemcpyHostToDevice, s));
      FPLS_CHECK(cudaMemcpyAsync(lab_tr.get(), compact.data(), sizeof(int) * ntr, cudaMemcpyHostToDevice, s));
      gather_rows<T>(X.get(), n, p, idx_tr.get(), ntr, Xtr.get(), ntr, s);
      gather_rows<T>(X.get(), n, p, idx_te.get(), nte, Xte.get(), nte, s);
      FPLS_CHECK(cudaMemsetAsync(ws.flag.get(), 0, sizeof(int), s));
      DeviceModel model;
      model.classification = true;
      model.label_view = lab_tr.get();
      model.ymean.allocate(c, s);
      prepare_responses<T>(nullptr, lab_tr.get(), ntr, c, Yc.get(), model.ymean.get(), ycsum.get(), ws.flag.get(), s);
      fit_method<T>(method, Xtr.get(), ntr, p, Yc.get(), ycsum.get(), c, maximum_prefix, scaling, model, ws, s);
      project_rows<T>(model, Xte.get(), nte, nte, maximum_prefix, scores.get(), nte, ws, s);
      std::unique_ptr<LdaState> lda;
      if (use_lda) {
        lda.reset(new LdaState());
        lda->train(model.T.get(), ntr, ntr, maximum_prefix, lab_tr.get(), c, ccount, ws.flag.get(), s);
      }
      host_labels.resize((size_t)nte * prefix_count);
      if (store_scores) host_scores.resize((size_t)nte * c * prefix_count);
      for (int j = 0; j < prefix_count; ++j) {
        predict_from_scores(model, scores.get(), nte, nte, prefixes[j], pred.get(), nte, s);
        if (store_scores)
          FPLS_CHECK(cudaMemcpyAsync(host_scores.data() + (size_t)j * nte * c, pred.get(),
                                     sizeof(double) * nte * c, cudaMemcpyDeviceToHost, s));
        const double* decoded = pred.get();
        if (use_lda) {
          lda->discriminants(scores.get(), nte, nte, prefixes[j], disc.get(), nte, s);
          decoded = disc.get();
        }
        topk_rows(decoded, nte, c, 1, top.get(), nte, s);
        FPLS_CHECK(cudaMemcpyAsync(host_labels.data() + (size_t)j * nte, top.get(),
                                   sizeof(int) * nte, cudaMemcpyDeviceToHost, s));
      }
      raise_on_flag(ws, s, method == kPlssvd
          ? "resident PLS-SVD failed: invalid labels, decomposition or score Gram"
          : "resident SIMPLS failed: invalid labels, decomposition or component norm");
      for (int j = 0; j < prefix_count; ++j) {
        for (int i = 0; i < nte; ++i) {
          const int predicted = active[host_labels[(size_t)j * nte + i] - 1];
          const int row = held[i];
          if (store_predictions) prediction_output[(size_t)j * n + row] = predicted;
          metrics[j] += predicted == labels[row] ? 1.0 : 0.0;
          counts[j] += 1.0;
        }
        if (store_scores)
          for (int ai = 0; ai < c; ++ai) {
            const int dest = active[ai] - 1;
            for (int i = 0; i < nte; ++i)
              score_output[(size_t)j * n * classes + (size_t)dest * n + held[i]] =
                  static_cast<T>(host_scores[(size_t)j * nte * c + (size_t)ai * nte + i]);
          }
      }
      status[f] = 1;
    }
    for (int j = 0; j < prefix_count; ++j)
      metrics[j] = counts[j] > 0.0 ? metrics[j] / counts[j]
                                   : std::numeric_limits<double>::quiet_NaN();
    FPLS_CHECK(cudaStreamSynchronize(s));
  }
}

#define FPLS_INSTANTIATE(T)                                                     \
  template void cv_regression<T>(int, const T*, const T*, const int*, int, int, \
                                 int, const int*, int, int, int, bool, double*, \
                                 int*, double*, double*, double*, double*);     \
  template void cv_classification<T>(int, const T*, const int*, const int*,     \
                                     int, int, int, const int*, int, int, bool, \
                                     bool, bool, int*, T*, int*, double*);
FPLS_INSTANTIATE(float)
FPLS_INSTANTIATE(double)
#undef FPLS_INSTANTIATE

}  // namespace fpls
