// Resident model handle (host orchestration of the fitting and prediction
// kernels). Behavioural contract: src/cuda_resident_api.cuh:69-479 of the
// reference (validation order, error strings, field sizes, synchronous
// calls on a per-handle non-blocking stream).
#include "upload.cuh"
#include "handle.cuh"
#include "persistent.cuh"
#include "lda.cuh"
#include "reduce.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace fpls {

namespace {

template <class T>
__global__ void convert_kernel(const double* __restrict__ in, long count,
                               T* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count;
       i += (long)gridDim.x * blockDim.x)
    out[i] = static_cast<T>(in[i]);
}

template <class T>
void convert(const double* in, long count, T* out, cudaStream_t s) {
  if (count <= 0) return;
  convert_kernel<T><<<(unsigned)std::min<long>((count + 255) / 256, 8L * num_sms()), 256, 0, s>>>(in, count, out);
  count_launch();
  FPLS_LAUNCH("convert");
}

// SSE, SS about the training mean, SS about the observed mean, per response
// (response_sums, src/cuda_resident_metrics.cuh:9-43), FP64.
template <class T>
__global__ void response_sums_kernel(const double* __restrict__ pred,
                                     const T* __restrict__ y,
                                     const int* __restrict__ labels,
                                     const double* __restrict__ ymean, int n,
                                     int q, double* out, int* flag) {
  __shared__ double scratch[32];
  const int c = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (labels && (labels[i] < 1 || labels[i] > q)) flag_error(flag, 4);
    const double v = labels ? (labels[i] == c + 1 ? 1.0 : 0.0)
                            : as_f64(y[i + (long)c * n]);
    if (!isfinite(v)) flag_error(flag, 4);
    s += v;
  }
  const double mu = block_sum(s, scratch) / n;
  double sse = 0.0, st = 0.0, so = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = labels ? (labels[i] == c + 1 ? 1.0 : 0.0)
                            : as_f64(y[i + (long)c * n]);
    const double f = pred[i + (long)c * n];
    if (!isfinite(f)) flag_error(flag, 4);
    const double e = v - f, d = v - ymean[c], o = v - mu;
    sse = fma(e, e, sse);
    st = fma(d, d, st);
    so = fma(o, o, so);
  }
  sse = block_sum(sse, scratch);
  st = block_sum(st, scratch);
  so = block_sum(so, scratch);
  if (threadIdx.x == 0) {
    out[3 * c] = sse;
    out[3 * c + 1] = st;
    out[3 * c + 2] = so;
  }
}

// Loadings P and sequential residual loadings (variance_loadings,
// src/cuda_resident_variance.cuh:10-24), FP64, one thread per predictor.
__global__ void variance_loadings_kernel(const double* __restrict__ cross,
                                         const double* __restrict__ gram,
                                         int p, int a, double* loadings,
                                         double* sequential) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < p;
       f += gridDim.x * blockDim.x) {
    for (int j = 0; j < a; ++j) {
      const double den = gram[j + (long)j * a];
      const bool ok = isfinite(den) && den > 0.0;
      double v = cross[f + (long)j * p];
      loadings[f + (long)j * p] = ok ? v / den : 0.0;
      for (int i = 0; i < j; ++i) v -= sequential[f + (long)i * p] * gram[i + (long)j * a];
      sequential[f + (long)j * p] = ok ? v / den : 0.0;
    }
  }
}

// cross = (X^T T - mean * colsum(T)) / scale  (in place)
__global__ void standardize_cross(double* cross, int p, int a,
                                  const double* __restrict__ mean,
                                  const double* __restrict__ scale,
                                  const double* __restrict__ tsum) {
  const long total = (long)p * a;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int j = (int)(idx % p), k = (int)(idx / p);
    cross[idx] = (cross[idx] - mean[j] * tsum[k]) / scale[j];
  }
}

__global__ void column_sums_kernel(const double* __restrict__ M, int rows,
                                   long ld, double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) s += M[i + (long)blockIdx.x * ld];
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__global__ void column_sumsq_kernel(const double* __restrict__ M, int rows,
                                    long ld, double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const double v = M[i + (long)blockIdx.x * ld];
    s = fma(v, v, s);
  }
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// Variable importance in projection per response and component prefix
// (vip_values, src/r_api.cpp:3973-4025): with SS_c = q_rc^2 ||t_c||^2,
// vip[r][c, j] = sqrt(fp * sum_{c' <= c} (w_jc'^2 / ||w_c'||^2) SS_c' /
// sum_{c' <= c} SS_c'); NaN while the denominator is zero. out holds, per
// response r, an a x fp column-major block at offset r a fp.
__global__ void vip_kernel(const double* __restrict__ R, int fp, const double* __restrict__ Q,
                           int m, const double* __restrict__ tss,
                           const double* __restrict__ wss, int a, double* __restrict__ out) {
  const long total = (long)m * fp;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int r = (int)(idx / fp), j = (int)(idx % fp);
    double num = 0.0, den = 0.0;
    double* o = out + (long)r * a * fp + (long)j * a;
    for (int c = 0; c < a; ++c) {
      const double q = Q[r + (long)c * m];
      const double explained = q * q * tss[c];
      den += explained;
      if (wss[c] > 0.0) {
        const double w = R[j + (long)c * fp];
        num += w * w * explained / wss[c];
      }
      o[c] = den > 0.0 ? sqrt(fp * num / den) : nan("");
    }
  }
}

// result[j] = ||sequential_j||^2 * gram_jj ; result[a] = sum_j column SS of Xs
__global__ void variance_finish_kernel(const double* __restrict__ sequential,
                                       const double* __restrict__ gram,
                                       const double* __restrict__ sum,
                                       const double* __restrict__ sumsq,
                                       const double* __restrict__ mean,
                                       const double* __restrict__ scale,
                                       int n, int p, int a, double* result) {
  __shared__ double scratch[32];
  for (int j = blockIdx.x; j <= a; j += gridDim.x) {
    double acc = 0.0;
    if (j < a) {
      for (int f = threadIdx.x; f < p; f += blockDim.x) {
        const double v = sequential[f + (long)j * p];
        acc = fma(v, v, acc);
      }
    } else {
      for (int f = threadIdx.x; f < p; f += blockDim.x) {
        const double mu = mean[f], sd = scale[f];
        const double ss = sumsq[f] - 2.0 * mu * sum[f] + (double)n * mu * mu;
        acc += fmax(ss, 0.0) / (sd * sd);
      }
    }
    acc = block_sum(acc, scratch);
    if (threadIdx.x == 0) {
      if (j < a) {
        const double g = acc * gram[j + (long)j * a];
        result[j] = (isfinite(g) && g > 0.0) ? g : 0.0;
      } else {
        result[a] = acc;
      }
    }
  }
}

void check_path(const int* prefixes, int count, int a) {
  require(prefixes != nullptr && count >= 1, "invalid resident prediction-path request");
  int previous = 0;
  for (int j = 0; j < count; ++j) {
    if (prefixes[j] <= previous || prefixes[j] > a)
      throw std::invalid_argument("component path must be strictly increasing");
    previous = prefixes[j];
  }
}

}  // namespace

// T: storage type of the predictors (float, double, or bf16 for precision
// 16); TO: type of responses and of every result written back (T, or float
// for bf16 predictors).
// Device time of the calling thread's last fit: input copies, then the fit
// proper (CUDA events on the handle's stream, read once the fit finished).
struct FitTimes {
  double copy_ms = 0.0, fit_ms = 0.0;
};
FitTimes& last_fit_times() {
  thread_local FitTimes t;
  return t;
}

class FitTimer {
 public:
  explicit FitTimer(cudaStream_t s) : s_(s) {
    for (cudaEvent_t& e : ev_) FPLS_CHECK(cudaEventCreate(&e));
    FPLS_CHECK(cudaEventRecord(ev_[0], s_));
  }
  ~FitTimer() {
    for (cudaEvent_t e : ev_) cudaEventDestroy(e);
  }
  FitTimer(const FitTimer&) = delete;
  FitTimer& operator=(const FitTimer&) = delete;
  void mark() { FPLS_CHECK(cudaEventRecord(ev_[++marks_], s_)); }
  // after the stream has finished the fit
  void finish() {
    if (marks_ != 2) return;
    float a = 0.f, b = 0.f;
    FPLS_CHECK(cudaEventSynchronize(ev_[2]));
    FPLS_CHECK(cudaEventElapsedTime(&a, ev_[0], ev_[1]));
    FPLS_CHECK(cudaEventElapsedTime(&b, ev_[1], ev_[2]));
    last_fit_times() = {a, b};
  }

 private:
  cudaStream_t s_;
  cudaEvent_t ev_[3] = {};
  int marks_ = 0;
};

template <class T>
class TypedHandle final : public ResidentHandle {
  using TO = typename io_type<T>::type;

 public:
  // defer: a SIMPLS fit that plans a persistent launch leaves it pending
  // (pending_plan()); the caller launches the plans of several handles
  // together, orders this handle's stream after that launch and calls
  // complete_fit().
  explicit TypedHandle(const FitRequest& rq, bool defer = false) : rq_(rq) {
    try {
      FPLS_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
      if (defer && rq_.method == kSimpls) {
        struct Sink {
          explicit Sink(std::unique_ptr<PersistentPlan>* s) { persistent_deferral() = s; }
          ~Sink() { persistent_deferral() = nullptr; }
        } sink(&pending_);
        fit_begin();
      } else {
        fit_begin();
      }
      if (!pending_) fit_end();
    } catch (...) {
      release();
      throw;
    }
  }
  explicit TypedHandle(const ImportRequest& im) {
    try {
      FPLS_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
      load(im);
    } catch (...) {
      release();
      throw;
    }
  }
  ~TypedHandle() override { release(); }

  PersistentPlan* pending_plan() override { return pending_.get(); }
  cudaStream_t stream() const override { return stream_; }
  void complete_fit() override {
    if (!pending_) return;
    fit_end();
    pending_.reset();
  }

  void predict_path(const void* x, int rows, const int* prefixes, int count,
                    bool lda, void* out) override {
    if (!x || !out || rows < 1 || count < 1)
      throw std::invalid_argument("invalid resident prediction-path request");
    check_path(prefixes, count, model_.a);
    if (lda && !model_.classification)
      throw std::invalid_argument("LDA requires class labels");
    const int kmax = prefixes[count - 1];
    upload_rows(x, rows);
    score_rows(rows, kmax);
    const int q = model_.m;
    pred_.reserve((size_t)rows * q, stream_);
    conv_.reserve((size_t)rows * q, stream_);
    TO* dst = static_cast<TO*>(out);
    for (int j = 0; j < count; ++j) {
      const int k = prefixes[j];
      if (lda) lda_state().discriminants(scores_.get(), rows, rows, k, pred_.get(), rows, stream_);
      else predict_from_scores(model_, scores_.get(), rows, rows, k, pred_.get(), rows, stream_);
      download(pred_.get(), (long)rows * q, dst + (size_t)j * rows * q);
    }
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  void classify_path(const void* x, int rows, const int* prefixes, int count,
                     bool lda, int top, int* out, void* response_out) override {
    const int q = model_.m;
    if (!model_.classification || !x || !out || count < 1 || top < 1 || top > q || rows < 1)
      throw std::invalid_argument(response_out
          ? "invalid resident classification-response path request"
          : "invalid resident classification-path request");
    check_path(prefixes, count, model_.a);
    const int kmax = prefixes[count - 1];
    upload_rows(x, rows);
    score_rows(rows, kmax);
    pred_.reserve((size_t)rows * q, stream_);
    disc_.reserve((size_t)rows * q, stream_);
    conv_.reserve((size_t)rows * q, stream_);
    top_.reserve((size_t)rows * top, stream_);
    TO* resp = static_cast<TO*>(response_out);
    for (int j = 0; j < count; ++j) {
      const int k = prefixes[j];
      const double* decoded = pred_.get();
      if (!lda || resp) {
        predict_from_scores(model_, scores_.get(), rows, rows, k, pred_.get(), rows, stream_);
        if (resp) download(pred_.get(), (long)rows * q, resp + (size_t)j * rows * q);
      }
      if (lda) {
        lda_state().discriminants(scores_.get(), rows, rows, k, disc_.get(), rows, stream_);
        decoded = disc_.get();
      }
      topk_rows(decoded, rows, q, top, top_.get(), rows, stream_);
      FPLS_CHECK(cudaMemcpyAsync(out + (size_t)j * rows * top, top_.get(),
                                 sizeof(int) * rows * top,
                                 cudaMemcpyDeviceToHost, stream_));
    }
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  void project(const void* x, int rows, int prefix, void* out) override {
    if (!x || !out || rows < 1 || prefix < 1 || prefix > model_.a)
      throw std::invalid_argument("invalid resident score request");
    upload_rows(x, rows);
    score_rows(rows, prefix);
    conv_.reserve((size_t)rows * prefix, stream_);
    download(scores_.get(), (long)rows * prefix, static_cast<TO*>(out));
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  void response_sums(const void* x, const void* y, const int* labels, int rows,
                     int prefix, void* out) override {
    if (!out || (!y && !labels) || (y && labels) ||
        (model_.classification != (labels != nullptr)))
      throw std::invalid_argument("invalid resident response representation");
    if (!x || rows < 1 || prefix < 1 || prefix > model_.a)
      throw std::invalid_argument("invalid resident prediction input");
    const int q = model_.m;
    upload_rows(x, rows);
    score_rows(rows, prefix);
    pred_.reserve((size_t)rows * q, stream_);
    predict_from_scores(model_, scores_.get(), rows, rows, prefix, pred_.get(), rows, stream_);
    DeviceArray<TO> yd;
    DeviceArray<int> ld;
    if (labels) {
      ld.allocate(rows, stream_);
      FPLS_CHECK(cudaMemcpyAsync(ld.get(), labels, sizeof(int) * rows, cudaMemcpyHostToDevice, stream_));
    } else {
      yd.allocate((size_t)rows * q, stream_);
      FPLS_CHECK(cudaMemcpyAsync(yd.get(), y, sizeof(TO) * rows * q, cudaMemcpyHostToDevice, stream_));
    }
    DeviceArray<double> sums((size_t)3 * q, stream_);
    FPLS_CHECK(cudaMemsetAsync(ws_.flag.get(), 0, sizeof(int), stream_));
    response_sums_kernel<TO><<<q, 256, 0, stream_>>>(pred_.get(), yd.get(), ld.get(),
                                                    model_.ymean.get(), rows, q,
                                                    sums.get(), ws_.flag.get());
    count_launch();
    FPLS_LAUNCH("response_sums");
    conv_.reserve((size_t)3 * q, stream_);
    download(sums.get(), 3L * q, static_cast<TO*>(out));
    raise_on_flag(ws_, stream_, "nonfinite response/prediction or invalid class label in resident metrics");
  }

  void export_field(int field, void* out, std::size_t size) override {
    const std::size_t a = model_.a, q = model_.m, p = rq_.p, fp = model_.feature_p;
    const std::size_t counts[] = {fp * a, q * a, (size_t)model_.n * a, p, p, q, fp * a, a + 1};
    if (field < 0 || field > 7 || !out || size != counts[field])
      throw std::invalid_argument("invalid resident field output size");
    const double* src = nullptr;
    switch (field) {
      case 0: src = model_.R.get(); break;
      case 1: src = q_export(); break;
      case 2: src = model_.T.get(); break;
      case 3: src = model_.method == kKernelPls ? model_.in_mean.get() : model_.mean.get(); break;
      case 4: src = model_.method == kKernelPls ? model_.in_scale.get() : model_.scale.get(); break;
      case 5: src = model_.ymean.get(); break;
      default: ensure_variance(); src = field == 6 ? loadings_.get() : var_ss_.get(); break;
    }
    if (!src) throw std::invalid_argument("resident field is not available after compaction");
    conv_.reserve(size, stream_);
    download(src, (long)size, static_cast<TO*>(out));
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  void vip(double* out, std::size_t size) override {
    const int a = model_.a, m = model_.m, fp = model_.feature_p;
    if (!out || size != (std::size_t)m * a * fp)
      throw std::invalid_argument("invalid resident VIP output size");
    if (model_.method == kPlssvd && !model_.Q)
      throw std::invalid_argument("VIP requires response loadings");
    if (!model_.T) throw std::invalid_argument("VIP requires a model fitted with fit = TRUE");
    DeviceArray<double> tss(a, stream_), wss(a, stream_), res(size, stream_);
    column_sumsq_kernel<<<a, 256, 0, stream_>>>(model_.T.get(), model_.n, model_.n, tss.get());
    column_sumsq_kernel<<<a, 256, 0, stream_>>>(model_.R.get(), fp, fp, wss.get());
    vip_kernel<<<(unsigned)std::min<long>(((long)m * fp + 255) / 256, 8L * num_sms()), 256, 0, stream_>>>(
        model_.R.get(), fp, q_export(), m, tss.get(), wss.get(), a, res.get());
    count_launch(3);
    FPLS_LAUNCH("vip");
    FPLS_CHECK(cudaMemcpyAsync(out, res.get(), sizeof(double) * size, cudaMemcpyDeviceToHost, stream_));
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  void controls(int* oversample, int* power, int* block, int* block_limit,
                int* implicit_operator, int* crossprod_cache) override {
    if (!oversample || !power || !block || !block_limit || !implicit_operator || !crossprod_cache)
      throw std::invalid_argument("null resident control output");
    // the requested sketch controls (directions are exact here), the
    // candidate block and the cached-Gram route this fit took; the
    // cross-covariance is always explicit (no implicit operator)
    *oversample = rq_.oversample;
    *power = rq_.power;
    *block = used_block_;
    *block_limit = 0;
    *implicit_operator = 0;
    *crossprod_cache = used_gram_ ? 1 : 0;
  }

  void compact(bool prepare_lda) override {
    if (prepare_lda) {
      if (!model_.classification)
        throw std::invalid_argument("LDA compaction requires classification labels");
      lda_state();
    }
    FPLS_CHECK(cudaStreamSynchronize(stream_));
    xtrain_.release();
    design_.release();
    model_.V.release();
    ws_.stream_partial.release();
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

 private:
  void fit_begin() {
    const int n = rq_.n, p = rq_.p, q = rq_.q, a = rq_.components;
    const bool cls = rq_.labels != nullptr;
    if (!rq_.x) throw std::invalid_argument("invalid resident matrix or precision");
    if ((rq_.y == nullptr) == (rq_.labels == nullptr))
      throw std::invalid_argument("provide responses or labels, not both");
    if (rq_.method == kKernelPls && (n < 2 || p < 1 || q < 1 || a < 1 || a > n - 1))
      throw std::invalid_argument("invalid resident CUDA nonlinear kernel PLS dimensions or controls");
    if (rq_.method == kOpls && (n < 2 || p < 1 || q < 1 || a < 1 || a > std::min(n - 1, p)))
      throw std::invalid_argument("invalid resident CUDA OPLS dimensions");
    if (rq_.method != kKernelPls &&
        (n < 2 || p < 1 || q < 1 || a < 1 || a > std::min(n - 1, p) || rq_.scaling < 1 || rq_.scaling > 3))
      throw std::invalid_argument(rq_.method == kPlssvd ? "invalid resident PLS-SVD dimensions"
                                                        : "invalid resident SIMPLS dimensions");
    if (cls && q < 2) throw std::invalid_argument("classification requires at least two classes");
    timer_.reset(new FitTimer(stream_));
    FitTimer& timer = *timer_;
    xtrain_.allocate((size_t)n * p, stream_);
    upload_h2d(xtrain_.get(), rq_.x, sizeof(T) * n * p, stream_);
    DeviceArray<TO> y;
    if (cls) {
      model_.labels.allocate(n, stream_);
      FPLS_CHECK(cudaMemcpyAsync(model_.labels.get(), rq_.labels, sizeof(int) * n, cudaMemcpyHostToDevice, stream_));
      model_.class_counts.assign(q, 0);
      for (int i = 0; i < n; ++i)
        if (rq_.labels[i] >= 1 && rq_.labels[i] <= q) ++model_.class_counts[rq_.labels[i] - 1];
      model_.label_view = model_.labels.get();
    } else {
      y.allocate((size_t)n * q, stream_);
      FPLS_CHECK(cudaMemcpyAsync(y.get(), rq_.y, sizeof(TO) * n * q, cudaMemcpyHostToDevice, stream_));
    }
    model_.classification = cls;
    timer.mark();  // inputs on the device: the fit proper starts here
    ws_.ensure(n, p, q, a, stream_);
    FPLS_CHECK(cudaMemsetAsync(ws_.flag.get(), 0, sizeof(int), stream_));
    DeviceArray<double> yc((size_t)n * q, stream_);
    DeviceArray<double> ycsum(q, stream_);
    model_.ymean.allocate(q, stream_);
    prepare_responses<TO>(y.get(), model_.labels.get(), n, q, yc.get(),
                         model_.ymean.get(), ycsum.get(), ws_.flag.get(), stream_);
    if (rq_.method == kPlssvd)
      fit_plssvd<T>(xtrain_.get(), n, p, n, yc.get(), ycsum.get(), q, a, rq_.scaling, model_, ws_, stream_);
    else if (rq_.method == kOpls)
      fit_opls<T>(xtrain_.get(), n, p, n, yc.get(), ycsum.get(), q, a, rq_.scaling, rq_.north, model_, ws_,
                  design_, stream_);
    else if (rq_.method == kKernelPls)
      fit_kernelpls<T>(xtrain_.get(), n, p, n, yc.get(), ycsum.get(), q, a, rq_.scaling, rq_.kernel,
                       rq_.gamma, rq_.degree, rq_.coef0, model_, ws_, design_, stream_);
    else
    {
      used_block_ = simpls_block_size(n, p, q, a, cls, std::is_same<T, float>::value);
      used_gram_ = simpls_gram_route(n, p, a, cls) && !std::is_same<T, bf16>::value;
      fit_simpls<T>(xtrain_.get(), n, p, n, yc.get(), ycsum.get(), q, a, rq_.scaling, model_, ws_, stream_,
                    used_block_, used_gram_);
    }
  }

  // after the fit's kernels (or its pending persistent launch) are enqueued
  void fit_end() {
    timer_->mark();
    raise_on_flag(ws_, stream_, rq_.method == kPlssvd
        ? "resident PLS-SVD failed: invalid labels, decomposition or score Gram"
        : rq_.method == kOpls ? "resident CUDA OPLS filtering failed"
        : "resident SIMPLS failed: invalid labels, decomposition or component norm");
    timer_->finish();
    timer_.reset();
  }

  void load(const ImportRequest& im) {
    const int n = im.n, p = im.p, q = im.q, a = im.components;
    if (im.method != kSimpls && im.method != kOpls)
      throw std::invalid_argument("model import supports SIMPLS and OPLS models");
    if (p < 1 || q < 1 || a < 1 || a > p || !im.R || !im.Q || !im.mean || !im.scale || !im.ymean ||
        im.scaling < 1 || im.scaling > 3)
      throw std::invalid_argument("invalid imported model fields");
    if (im.labels && (!im.T || !im.classification || n < 2))
      throw std::invalid_argument("imported labels need the training scores of a classification model");
    if (im.T && n < 1) throw std::invalid_argument("invalid imported model fields");
    if (im.classification && q < 2)
      throw std::invalid_argument("classification requires at least two classes");
    for (int j = 0; j < p; ++j)
      if (!std::isfinite(im.mean[j]) || !std::isfinite(im.scale[j]) || im.scale[j] == 0.0)
        throw std::invalid_argument("invalid imported model fields");
    rq_.method = im.method;
    rq_.n = im.T ? n : 0;
    rq_.p = p;
    rq_.q = q;
    rq_.components = a;
    rq_.scaling = im.scaling;
    model_.method = im.method;
    model_.n = rq_.n;
    model_.p = p;
    model_.feature_p = p;
    model_.m = q;
    model_.a = a;
    model_.scaling = im.scaling;
    model_.classification = im.classification;
    auto up = [&](DeviceArray<double>& dst, const double* src, size_t count) {
      dst.allocate(count, stream_);
      FPLS_CHECK(cudaMemcpyAsync(dst.get(), src, sizeof(double) * count, cudaMemcpyHostToDevice, stream_));
    };
    up(model_.R, im.R, (size_t)p * a);
    up(model_.Q, im.Q, (size_t)q * a);
    up(model_.mean, im.mean, p);
    up(model_.scale, im.scale, p);
    up(model_.ymean, im.ymean, q);
    if (im.T) up(model_.T, im.T, (size_t)n * a);
    if (im.labels) {
      model_.class_counts.assign(q, 0);
      for (int i = 0; i < n; ++i) {
        if (im.labels[i] < 1 || im.labels[i] > q) throw std::invalid_argument("invalid imported labels");
        ++model_.class_counts[im.labels[i] - 1];
      }
      model_.labels.allocate(n, stream_);
      FPLS_CHECK(cudaMemcpyAsync(model_.labels.get(), im.labels, sizeof(int) * n, cudaMemcpyHostToDevice,
                                 stream_));
    }
    ws_.ensure(std::max(rq_.n, 1), p, q, a, stream_);
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  const double* q_export() { return model_.Q.get(); }

  double* scores(int rows, int k) {
    scores_.reserve((size_t)rows * k, stream_);
    return scores_.get();
  }

  // latent scores of the uploaded rows (xbuf_) into scores_ (rows x k)
  void score_rows(int rows, int k) {
    if (model_.method == kKernelPls)
      kernel_scores<T>(model_, xbuf_.get(), rows, rows, k, scores(rows, k), rows, ws_, stream_);
    else
      project_rows<T>(model_, xbuf_.get(), rows, rows, k, scores(rows, k), rows, ws_, stream_);
  }

  void upload_rows(const void* x, int rows) {
    xbuf_.reserve((size_t)rows * rq_.p, stream_);
    upload_h2d(xbuf_.get(), x, sizeof(T) * rows * rq_.p, stream_);
  }

  void download(const double* src, long count, TO* dst) {
    const TO* from = nullptr;
    if (std::is_same<TO, double>::value) {
      from = reinterpret_cast<const TO*>(src);
    } else {
      convert<TO>(src, count, conv_.get(), stream_);
      from = conv_.get();
    }
    FPLS_CHECK(cudaMemcpyAsync(dst, from, sizeof(TO) * count, cudaMemcpyDeviceToHost, stream_));
    if (!std::is_same<TO, double>::value) FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  LdaState& lda_state() {
    if (!lda_) {
      if (!model_.classification) throw std::invalid_argument("LDA requires class labels");
      if (!model_.T || !model_.labels)
        throw std::invalid_argument("LDA requires the training scores and labels of the model");
      auto next = std::make_unique<LdaState>();
      next->train(model_.T.get(), model_.n, model_.n, model_.a, model_.labels.get(),
                  model_.m, model_.class_counts, ws_.flag.get(), stream_);
      lda_ = std::move(next);
    }
    return *lda_;
  }

  void ensure_variance() {
    if (loadings_) return;
    if (design_) {
      const int fp = model_.feature_p;
      DeviceArray<double> zero(fp, stream_), one(fp, stream_);
      zero.zero(stream_);
      fill_ones(one.get(), fp);
      variance_from<double>(design_.get(), fp, zero.get(), one.get());
      return;
    }
    if (!xtrain_) throw std::invalid_argument("resident variance requires the training predictors (call before compaction)");
    variance_from<T>(xtrain_.get(), model_.p, model_.mean.get(), model_.scale.get());
  }

  void fill_ones(double* ptr, int count) {
    std::vector<double> ones(count, 1.0);
    FPLS_CHECK(cudaMemcpyAsync(ptr, ones.data(), sizeof(double) * count, cudaMemcpyHostToDevice, stream_));
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  // loadings P and per-component SS from predictors X (n x p, standardised by
  // mean/scale) and the training scores (variance_loadings/variance_finish,
  // src/cuda_resident_variance.cuh:10-94)
  template <class TX>
  void variance_from(const TX* X, int p, const double* mean, const double* scale) {
    const int n = model_.n, a = model_.a;
    DeviceArray<double> cross((size_t)p * a, stream_), seq((size_t)p * a, stream_);
    DeviceArray<double> gram((size_t)a * a, stream_), tsum(a, stream_);
    DeviceArray<double> mom((size_t)2 * p, stream_);
    loadings_.allocate((size_t)p * a, stream_);
    var_ss_.allocate(a + 1, stream_);
    xtv_product<TX>(X, n, p, n, model_.T.get(), n, a, cross.get(), p, ws_.stream_partial, stream_);
    column_moments<TX>(X, n, p, n, nullptr, 0, mom.get(), mom.get() + p, nullptr, ws_.stream_partial, stream_);
    column_sums_kernel<<<a, 256, 0, stream_>>>(model_.T.get(), n, n, tsum.get());
    count_launch();
    standardize_cross<<<std::min<unsigned>(ceil_div((size_t)p * a, 256), 8 * num_sms()), 256, 0, stream_>>>(
        cross.get(), p, a, mean, scale, tsum.get());
    count_launch();
    GemmArgs g;
    g.M = a; g.N = a; g.K = n;
    g.A = model_.T.get(); g.lda = n; g.trans_a = true;
    g.B = model_.T.get(); g.ldb = n;
    g.C = gram.get(); g.ldc = a;
    gemm_f64(g, stream_);
    variance_loadings_kernel<<<std::min<unsigned>(ceil_div(p, 256), 8 * num_sms()), 256, 0, stream_>>>(
        cross.get(), gram.get(), p, a, loadings_.get(), seq.get());
    count_launch();
    variance_finish_kernel<<<std::min(a + 1, 4 * num_sms()), 256, 0, stream_>>>(
        seq.get(), gram.get(), mom.get(), mom.get() + p, mean, scale, n, p, a, var_ss_.get());
    count_launch();
    FPLS_LAUNCH("variance");
    FPLS_CHECK(cudaStreamSynchronize(stream_));
  }

  void release() noexcept {
    if (stream_) cudaStreamSynchronize(stream_);
    pending_.reset();
    timer_.reset();
    lda_.reset();
    model_ = DeviceModel();
    ws_ = Workspace();
    xtrain_.release();
    design_.release();
    xbuf_.release();
    scores_.release();
    pred_.release();
    disc_.release();
    conv_.release();
    top_.release();
    loadings_.release();
    var_ss_.release();
    if (stream_) {
      cudaStreamSynchronize(stream_);
      cudaStreamDestroy(stream_);
    }
    stream_ = nullptr;
  }

  FitRequest rq_;
  cudaStream_t stream_ = nullptr;
  DeviceModel model_;
  Workspace ws_;
  DeviceArray<T> xtrain_, xbuf_;
  DeviceArray<TO> conv_;
  DeviceArray<double> scores_, pred_, disc_, loadings_, var_ss_, design_;
  DeviceArray<int> top_;
  std::unique_ptr<LdaState> lda_;
  std::unique_ptr<PersistentPlan> pending_;
  std::unique_ptr<FitTimer> timer_;
  int used_block_ = 1;
  bool used_gram_ = false;
};

ResidentHandle* import_handle(int precision, const ImportRequest& im) {
  if (precision == 32) return new TypedHandle<float>(im);
  if (precision == 64) return new TypedHandle<double>(im);
  if (precision == 16) return new TypedHandle<bf16>(im);
  throw std::invalid_argument("invalid resident matrix or precision");
}

void read_last_fit_times(double* copy_ms, double* fit_ms) {
  const FitTimes& t = last_fit_times();
  if (copy_ms) *copy_ms = t.copy_ms;
  if (fit_ms) *fit_ms = t.fit_ms;
}

ResidentHandle* make_handle(int precision, const FitRequest& rq, bool defer) {
  if (precision == 32) return new TypedHandle<float>(rq, defer);
  if (precision == 64) return new TypedHandle<double>(rq, defer);
  if (precision == 16) return new TypedHandle<bf16>(rq, defer);
  throw std::invalid_argument("invalid resident matrix or precision");
}

}  // namespace fpls
