// Serving loop: fit and predict requests with continuous admission.
//
// Requests (fits of any method and size, predictions against resident
// models, model releases) enter one queue. Worker threads -- one CUDA stream
// each through the resident handles -- take the oldest request whose HBM
// footprint fits the remaining budget, so later small requests overtake a
// large one that is waiting for memory, and requests that arrive while
// others are running start as soon as a worker and memory free up; their
// work overlaps on the device across streams. Predictions queued against the
// same model are merged into one projection (rows concatenated) and split
// back per request. Fitted models stay resident (their training predictors
// are released after the fit) and keep their footprint charged until they
// are released. Every computation is deterministic, so a request's result is
// identical whether it runs alone or in a mix.
//
// There is no counterpart in the reference (it fits one model per call).
#include "../../include/fastpls_b200.h"
#include "handle.cuh"
#include "persistent.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace fpls {

namespace {

using Clock = std::chrono::steady_clock;

enum RequestKind { kFit = 1, kPredict = 2 };

struct Request {
  unsigned long long ticket = 0;
  int kind = kFit;
  int precision = 64;
  FitRequest fit;
  std::vector<unsigned char> x, y;
  std::vector<int> labels;
  // borrowed inputs (the server's borrow mode): the caller's buffers, valid
  // until the request has finished; null when the request owns copies
  const unsigned char* bx = nullptr;
  const unsigned char* by = nullptr;
  const int* blabels = nullptr;
  const unsigned char* xdata() const { return bx ? bx : x.data(); }
  const void* ydata() const { return by ? static_cast<const void*>(by) : (y.empty() ? nullptr : y.data()); }
  const int* labdata() const { return blabels ? blabels : (labels.empty() ? nullptr : labels.data()); }
  // prediction
  unsigned long long model = 0;
  int rows = 0;
  std::vector<int> prefixes;
  int lda = 0;
  bool deferred = false;  // submitted before its model existed (fit still queued or running)
  // results
  bool done = false;
  int status = 0;  // 0 ok, 1 error
  std::string error;
  std::vector<unsigned char> out;
  size_t footprint = 0;
  Clock::time_point submitted, started, finished;
};

struct Model {
  std::unique_ptr<ResidentHandle> handle;
  int precision = 64, q = 0, p = 0, ncomp = 0;
  size_t footprint = 0;
  int busy = 0;
};

size_t elem(int precision) { return precision == 32 ? 4 : 8; }

size_t fit_footprint(const Request& r) {
  const double n = r.fit.n, p = r.fit.p, q = r.fit.q, a = r.fit.components;
  double bytes = n * p * elem(r.precision);                 // X
  bytes += 8.0 * (p * (2 * a + 3 * q + 8) + n * (a + 2 * q + 4));
  if (r.fit.method == kOpls) bytes += 8.0 * n * p;          // FP64 filtered copy
  if (r.fit.method == kKernelPls) bytes += 8.0 * (2 * n * n + n * p);
  bytes += 64.0 * 1024 * 1024;                               // partials / scratch
  return (size_t)bytes;
}

size_t resident_footprint(const Request& r) {
  const double n = r.fit.n, p = r.fit.p, q = r.fit.q, a = r.fit.components;
  double bytes = 8.0 * (p * (2 * a + q + 2) + n * a + q * a);
  if (r.fit.method == kKernelPls) bytes += 8.0 * (n * p + n * a + 2 * n);
  return (size_t)bytes;
}

// A SIMPLS fit that runs as one persistent launch (one direction per
// component, within the launch's co-resident CTAs) and can share that launch
// with other such fits of the same storage type.
bool batchable_fit(const Request& r) {
  const FitRequest& f = r.fit;
  if (r.kind != kFit || f.method != kSimpls || !persistent_enabled()) return false;
  if (f.n < 2 || f.p < 1 || f.components < 1 || f.components > std::min(f.n - 1, f.p)) return false;
  if (!persistent_supported(f.q, f.components)) return false;
  if ((long)f.n * f.p > kPersistMaxElements) return false;
  if (simpls_block_size(f.n, f.p, f.q, f.components, !r.labels.empty(), r.precision == 32) != 1)
    return false;
  const int elem = r.precision == 16 ? 2 : r.precision == 32 ? 4 : 8;
  const int cap = persistent_capacity(elem);
  const int ctas = persistent_ctas(f.n, f.p);
  return cap > 0 && ctas > 0 && ctas <= cap;
}

size_t predict_footprint(int rows, const Model& m) {
  return (size_t)rows * m.p * elem(m.precision) + (size_t)rows * (m.ncomp + 2 * m.q) * 8 +
         16u * 1024 * 1024;
}

}  // namespace

class Server {
 public:
  Server(size_t budget, int workers) : budget_(budget) {
    FPLS_CHECK(cudaGetDevice(&device_));
    for (int w = 0; w < workers; ++w) threads_.emplace_back([this] { worker(); });
  }
  ~Server() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : threads_) t.join();
  }

  unsigned long long submit(std::unique_ptr<Request> r) {
    std::lock_guard<std::mutex> lock(mu_);
    r->ticket = next_ticket_++;
    r->submitted = Clock::now();
    if (r->kind == kPredict) {
      auto it = models_.find(r->model);
      if (it != models_.end()) {
        if (it->second.p != r->fit.p || it->second.precision != r->precision)
          throw std::invalid_argument("prediction rows do not match the model's columns or precision");
        r->footprint = predict_footprint(r->rows, it->second);
      } else {
        // a prediction may be queued behind the fit of its model: it is
        // admitted once that fit has produced the model
        auto ft = all_.find(r->model);
        if (ft == all_.end() || ft->second->kind != kFit ||
            (ft->second->done && ft->second->status == 0))
          throw std::invalid_argument("unknown model ticket");
        if (ft->second->fit.p != r->fit.p || ft->second->precision != r->precision)
          throw std::invalid_argument("prediction rows do not match the model's columns or precision");
        if (ft->second->done) {
          // the fit has already failed (and is not yet collected): the
          // prediction completes at once with that error
          r->status = 1;
          r->error = "the model's fit failed: " + ft->second->error;
          r->started = r->finished = Clock::now();
          r->done = true;
          const unsigned long long t = r->ticket;
          all_[t] = std::move(r);
          cv_done_.notify_all();
          return t;
        }
        r->deferred = true;
      }
    } else {
      r->footprint = fit_footprint(*r);
      if (r->footprint + resident_footprint(*r) > budget_)
        throw std::invalid_argument("request exceeds the server's HBM budget");
    }
    const unsigned long long t = r->ticket;
    pending_.push_back(r.get());
    all_[t] = std::move(r);
    cv_work_.notify_all();
    return t;
  }

  // Blocks until the request is done or `timeout` seconds pass.
  Request* wait(unsigned long long ticket, double timeout) {
    std::unique_lock<std::mutex> lock(mu_);
    auto it = all_.find(ticket);
    if (it == all_.end()) throw std::invalid_argument("unknown request ticket");
    Request* r = it->second.get();
    const auto deadline = Clock::now() + std::chrono::duration<double>(timeout);
    while (!r->done) {
      if (cv_done_.wait_until(lock, deadline) == std::cv_status::timeout && !r->done)
        throw std::runtime_error("timed out waiting for the request");
    }
    return r;
  }

  void forget(unsigned long long ticket) {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = all_.find(ticket);
    if (it != all_.end() && it->second->done) all_.erase(it);
  }

  void release_model(unsigned long long ticket) {
    std::unique_ptr<ResidentHandle> h;
    {
      std::unique_lock<std::mutex> lock(mu_);
      auto it = models_.find(ticket);
      if (it == models_.end()) throw std::invalid_argument("unknown model ticket");
      cv_done_.wait(lock, [&] { return it->second.busy == 0; });
      h = std::move(it->second.handle);
      in_use_ -= it->second.footprint;
      models_.erase(it);
    }
    h.reset();
    cv_work_.notify_all();
  }

  void stats(size_t* in_use, size_t* queued, size_t* models) {
    std::lock_guard<std::mutex> lock(mu_);
    if (in_use) *in_use = in_use_;
    if (queued) *queued = pending_.size();
    if (models) *models = models_.size();
  }

  void batch_stats(size_t* launches, size_t* fits) {
    std::lock_guard<std::mutex> lock(mu_);
    if (launches) *launches = batched_launches_;
    if (fits) *fits = batched_fits_;
  }

 private:
  // Oldest admissible request; predictions for the same model queued behind
  // it join its batch. Called with mu_ held.
  std::vector<Request*> take() {
    for (auto it = pending_.begin(); it != pending_.end();) {
      Request* r = *it;
      Model* model = nullptr;
      if (r->kind == kPredict) {
        auto mit = models_.find(r->model);
        if (mit == models_.end()) {
          auto ft = all_.find(r->model);
          if (ft != all_.end() && ft->second->kind == kFit && !ft->second->done) {
            ++it;  // its fit is still queued or running
            continue;
          }
          // the fit failed, or the model was released while this waited
          r->status = 1;
          r->error = ft != all_.end() && ft->second->status != 0
                         ? "the model's fit failed: " + ft->second->error
                         : "unknown model ticket";
          r->started = r->finished = Clock::now();
          r->done = true;
          it = pending_.erase(it);
          cv_done_.notify_all();
          continue;
        }
        model = &mit->second;
        if (r->deferred) {
          r->footprint = predict_footprint(r->rows, *model);
          r->deferred = false;
        }
        // one batch per model at a time: requests arriving meanwhile queue
        // up and join the next batch
        if (model->busy > 0) {
          ++it;
          continue;
        }
      }
      if (in_use_ + r->footprint > budget_) {
        ++it;
        continue;
      }
      std::vector<Request*> batch{r};
      size_t fp = r->footprint;
      pending_.erase(it);
      if (r->kind == kFit && batchable_fit(*r)) {
        // later compatible fits that fit the budget share its persistent
        // launch, up to the launch's co-resident CTAs
        const int elem = r->precision == 16 ? 2 : r->precision == 32 ? 4 : 8;
        const int cap = persistent_capacity(elem);
        int ctas = persistent_ctas(r->fit.n, r->fit.p);
        for (auto jt = pending_.begin(); jt != pending_.end() && (int)batch.size() < kFitBatchMax;) {
          Request* o = *jt;
          if (o->kind == kFit && o->precision == r->precision && batchable_fit(*o) &&
              ctas + persistent_ctas(o->fit.n, o->fit.p) <= cap &&
              in_use_ + fp + o->footprint <= budget_) {
            ctas += persistent_ctas(o->fit.n, o->fit.p);
            batch.push_back(o);
            fp += o->footprint;
            jt = pending_.erase(jt);
          } else {
            ++jt;
          }
        }
      }
      if (model) {
        for (auto jt = pending_.begin(); jt != pending_.end();) {
          Request* o = *jt;
          if (o->kind == kPredict && o->model == r->model && o->deferred) {
            o->footprint = predict_footprint(o->rows, *model);
            o->deferred = false;
          }
          if (o->kind == kPredict && o->model == r->model && o->lda == r->lda &&
              o->prefixes == r->prefixes && in_use_ + fp + o->footprint <= budget_) {
            batch.push_back(o);
            fp += o->footprint;
            jt = pending_.erase(jt);
          } else {
            ++jt;
          }
        }
        model->busy += 1;
      }
      in_use_ += fp;
      return batch;
    }
    return {};
  }

  void worker() {
    cudaSetDevice(device_);
    // this worker's stream for the persistent launches of fit batches
    cudaStream_t launch_stream = nullptr;
    if (cudaStreamCreateWithFlags(&launch_stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      launch_stream = nullptr;
    }
    struct StreamGuard {
      cudaStream_t s;
      ~StreamGuard() {
        if (s) {
          cudaStreamSynchronize(s);
          cudaStreamDestroy(s);
        }
      }
    } guard{launch_stream};
    for (;;) {
      std::vector<Request*> batch;
      {
        std::unique_lock<std::mutex> lock(mu_);
        cv_work_.wait(lock, [&] {
          if (stop_) return true;
          batch = take();
          return !batch.empty();
        });
        if (batch.empty()) return;
      }
      const auto start = Clock::now();
      for (auto* r : batch) r->started = start;
      size_t charged = 0;
      for (auto* r : batch) charged += r->footprint;
      if (batch[0]->kind == kFit && batch.size() > 1 && launch_stream)
        run_fit_batch(batch, launch_stream);
      else if (batch[0]->kind == kFit && batch.size() > 1)
        for (auto* r : batch) run_fit(r, r->footprint);
      else if (batch[0]->kind == kFit) run_fit(batch[0], charged);
      else run_predict(batch, charged);
    }
  }

  void finish(const std::vector<Request*>& batch, size_t release, Model* model_busy) {
    std::lock_guard<std::mutex> lock(mu_);
    in_use_ -= release;
    if (model_busy) model_busy->busy -= 1;
    const auto end = Clock::now();
    for (auto* r : batch) {
      r->finished = end;
      r->done = true;
    }
    cv_done_.notify_all();
    cv_work_.notify_all();
  }

  void run_fit(Request* r, size_t charged) {
    size_t keep = 0;
    try {
      r->fit.x = r->xdata();
      r->fit.y = r->ydata();
      r->fit.labels = r->labdata();
      std::unique_ptr<ResidentHandle> h(make_handle(r->precision, r->fit));
      h->compact(false);  // training predictors are not needed for serving
      Model m;
      m.handle = std::move(h);
      m.precision = r->precision;
      m.q = r->fit.q;
      m.p = r->fit.p;
      m.ncomp = r->fit.components;
      m.footprint = resident_footprint(*r);
      keep = m.footprint;
      std::lock_guard<std::mutex> lock(mu_);
      models_.emplace(r->ticket, std::move(m));
      in_use_ += keep;
    } catch (const std::exception& e) {
      r->status = 1;
      r->error = e.what();
    }
    r->x.clear();
    r->x.shrink_to_fit();
    r->y.clear();
    r->y.shrink_to_fit();
    finish({r}, charged, nullptr);
  }

  // Several SIMPLS fits in one persistent launch: each fit's inputs, moments
  // and cross-product are prepared on its own handle's stream, one
  // cooperative launch (on this worker's stream, after all of them) runs the
  // component loops of every fit, and each handle then finishes on its own
  // stream. A fit keeps the CTA count and chunking it has alone, so its
  // result is bit-identical alone or in a batch.
  void run_fit_batch(const std::vector<Request*>& batch, cudaStream_t batch_stream_) {
    std::vector<std::unique_ptr<ResidentHandle>> handles(batch.size());
    std::vector<PersistentPlan*> plans;
    std::vector<size_t> pending_idx;
    for (size_t i = 0; i < batch.size(); ++i) {
      Request* r = batch[i];
      try {
        r->fit.x = r->xdata();
        r->fit.y = r->ydata();
        r->fit.labels = r->labdata();
        handles[i].reset(make_handle(r->precision, r->fit, true));
        if (PersistentPlan* pl = handles[i]->pending_plan()) {
          plans.push_back(pl);
          pending_idx.push_back(i);
        }
      } catch (const std::exception& e) {
        r->status = 1;
        r->error = e.what();
        handles[i].reset();
      }
    }
    if (!plans.empty()) {
      std::vector<cudaEvent_t> evs;
      try {
        for (size_t i : pending_idx) {
          cudaEvent_t e = nullptr;
          FPLS_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
          evs.push_back(e);
          FPLS_CHECK(cudaEventRecord(e, handles[i]->stream()));
          FPLS_CHECK(cudaStreamWaitEvent(batch_stream_, e, 0));
        }
        launch_persistent(plans, batch_stream_);
        cudaEvent_t done = nullptr;
        FPLS_CHECK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        evs.push_back(done);
        FPLS_CHECK(cudaEventRecord(done, batch_stream_));
        for (size_t i : pending_idx) FPLS_CHECK(cudaStreamWaitEvent(handles[i]->stream(), done, 0));
      } catch (const std::exception& e) {
        cudaStreamSynchronize(batch_stream_);
        for (size_t i : pending_idx) {
          batch[i]->status = 1;
          batch[i]->error = e.what();
          handles[i].reset();
        }
      }
      for (cudaEvent_t e : evs) cudaEventDestroy(e);
    }
    for (size_t i = 0; i < batch.size(); ++i) {
      Request* r = batch[i];
      size_t keep = 0;
      if (handles[i]) {
        try {
          handles[i]->complete_fit();
          handles[i]->compact(false);  // training predictors are not needed for serving
          Model m;
          m.handle = std::move(handles[i]);
          m.precision = r->precision;
          m.q = r->fit.q;
          m.p = r->fit.p;
          m.ncomp = r->fit.components;
          m.footprint = resident_footprint(*r);
          keep = m.footprint;
          std::lock_guard<std::mutex> lock(mu_);
          models_.emplace(r->ticket, std::move(m));
          in_use_ += keep;
        } catch (const std::exception& e) {
          r->status = 1;
          r->error = e.what();
          handles[i].reset();
        }
      }
      r->x.clear();
      r->x.shrink_to_fit();
      r->y.clear();
      r->y.shrink_to_fit();
      finish({r}, r->footprint, nullptr);
    }
    {
      std::lock_guard<std::mutex> lock(mu_);
      ++batched_launches_;
      batched_fits_ += plans.size();
    }
  }

  void run_predict(const std::vector<Request*>& batch, size_t charged) {
    Model* model = nullptr;
    {
      std::lock_guard<std::mutex> lock(mu_);
      model = &models_.at(batch[0]->model);
    }
    try {
      const size_t es = elem(model->precision);
      const int p = model->p, q = model->q;
      const int count = (int)batch[0]->prefixes.size();
      int rows = 0;
      for (auto* r : batch) rows += r->rows;
      // merge the row blocks (column-major: one column at a time)
      std::vector<unsigned char> x((size_t)rows * p * es);
      int off = 0;
      for (auto* r : batch) {
        for (int j = 0; j < p; ++j)
          std::memcpy(x.data() + ((size_t)j * rows + off) * es,
                      r->xdata() + (size_t)j * r->rows * es, (size_t)r->rows * es);
        off += r->rows;
      }
      std::vector<unsigned char> out((size_t)rows * q * count * es);
      model->handle->predict_path(x.data(), rows, batch[0]->prefixes.data(), count,
                                  batch[0]->lda != 0, out.data());
      off = 0;
      for (auto* r : batch) {
        r->out.resize((size_t)r->rows * q * count * es);
        for (int k = 0; k < count; ++k)
          for (int c = 0; c < q; ++c)
            std::memcpy(r->out.data() + (((size_t)k * q + c) * r->rows) * es,
                        out.data() + (((size_t)k * q + c) * rows + off) * es,
                        (size_t)r->rows * es);
        off += r->rows;
        r->x.clear();
        r->x.shrink_to_fit();
      }
    } catch (const std::exception& e) {
      for (auto* r : batch) {
        r->status = 1;
        r->error = e.what();
      }
    }
    finish(batch, charged, model);
  }

  static constexpr int kFitBatchMax = 32;
 public:
  // borrow mode: submitted inputs are read in place (no host copy)
  bool borrow = false;

 private:
  size_t batched_launches_ = 0, batched_fits_ = 0;
  size_t budget_, in_use_ = 0;
  int device_ = 0;
  bool stop_ = false;
  unsigned long long next_ticket_ = 1;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<Request*> pending_;
  std::unordered_map<unsigned long long, std::unique_ptr<Request>> all_;
  std::unordered_map<unsigned long long, Model> models_;
  std::vector<std::thread> threads_;
};

}  // namespace fpls

using fpls::Request;
using fpls::Server;

namespace {

void put_error(char* out, size_t cap, const char* m) {
  if (out && cap) std::snprintf(out, cap, "%s", m);
}

template <class F>
int guard(char* err, size_t cap, F&& f) {
  put_error(err, cap, "");
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    put_error(err, cap, e.what());
    return 1;
  }
}

}  // namespace

extern "C" {

FASTPLS_B200_API void* fastpls_b200_server_create(size_t budget_bytes, int workers,
                                                  char* error, size_t error_capacity) {
  put_error(error, error_capacity, "");
  try {
    if (workers < 1 || workers > 64 || budget_bytes == 0)
      throw std::invalid_argument("invalid server budget or worker count");
    return new Server(budget_bytes, workers);
  } catch (const std::exception& e) {
    put_error(error, error_capacity, e.what());
    return nullptr;
  }
}

FASTPLS_B200_API void fastpls_b200_server_destroy(void* server) {
  delete static_cast<Server*>(server);
}

FASTPLS_B200_API int fastpls_b200_server_submit_fit(
    void* server, int method, const void* x, const void* y, const int* labels,
    int precision, int n, int p, int q, int components, int scaling, int north,
    int kernel, double gamma, int degree, double coef0,
    unsigned long long* ticket, char* error, size_t error_capacity) {
  return guard(error, error_capacity, [&] {
    if (!server || !x || !ticket || (precision != 32 && precision != 64) || n < 2 || p < 1 ||
        q < 1 || ((y == nullptr) == (labels == nullptr)) ||
        (method != 1 && method != 3 && method != 4 && method != 5))
      throw std::invalid_argument("invalid fit request");
    auto r = std::make_unique<Request>();
    r->kind = fpls::kFit;
    r->precision = precision;
    const size_t es = precision == 32 ? 4 : 8;
    if (static_cast<Server*>(server)->borrow) {
      r->bx = static_cast<const unsigned char*>(x);
      r->by = static_cast<const unsigned char*>(y);
      r->blabels = labels;
    } else {
      r->x.assign(static_cast<const unsigned char*>(x), static_cast<const unsigned char*>(x) + (size_t)n * p * es);
      if (y) r->y.assign(static_cast<const unsigned char*>(y), static_cast<const unsigned char*>(y) + (size_t)n * q * es);
      if (labels) r->labels.assign(labels, labels + n);
    }
    auto& f = r->fit;
    f.method = method;
    f.n = n;
    f.p = p;
    f.q = q;
    f.components = components;
    f.scaling = scaling;
    f.north = north;
    f.kernel = kernel;
    f.gamma = gamma;
    f.degree = degree;
    f.coef0 = coef0;
    *ticket = static_cast<Server*>(server)->submit(std::move(r));
  });
}

FASTPLS_B200_API int fastpls_b200_server_submit_predict(
    void* server, unsigned long long model, const void* x, int rows, int p,
    int precision, const int* prefixes, int prefix_count, int lda,
    unsigned long long* ticket, char* error, size_t error_capacity) {
  return guard(error, error_capacity, [&] {
    if (!server || !x || !ticket || rows < 1 || p < 1 || !prefixes || prefix_count < 1 ||
        (precision != 32 && precision != 64))
      throw std::invalid_argument("invalid prediction request");
    auto r = std::make_unique<Request>();
    r->kind = fpls::kPredict;
    r->precision = precision;
    r->model = model;
    r->rows = rows;
    r->fit.p = p;
    r->lda = lda;
    r->prefixes.assign(prefixes, prefixes + prefix_count);
    const size_t es = precision == 32 ? 4 : 8;
    if (static_cast<Server*>(server)->borrow)
      r->bx = static_cast<const unsigned char*>(x);
    else
      r->x.assign(static_cast<const unsigned char*>(x), static_cast<const unsigned char*>(x) + (size_t)rows * p * es);
    *ticket = static_cast<Server*>(server)->submit(std::move(r));
  });
}

// Wait for a request. For predictions `out` receives rows x q x prefixes
// values in the request's precision (`capacity_bytes` must be large enough);
// fits produce no output (their ticket is the model id). queue_ms and
// service_ms report the time from submission to start and start to finish.
FASTPLS_B200_API int fastpls_b200_server_wait(
    void* server, unsigned long long ticket, double timeout_seconds, void* out,
    size_t capacity_bytes, double* queue_ms, double* service_ms, char* error,
    size_t error_capacity) {
  return guard(error, error_capacity, [&] {
    if (!server) throw std::invalid_argument("null server");
    Server* s = static_cast<Server*>(server);
    Request* r = s->wait(ticket, timeout_seconds);
    if (queue_ms)
      *queue_ms = std::chrono::duration<double, std::milli>(r->started - r->submitted).count();
    if (service_ms)
      *service_ms = std::chrono::duration<double, std::milli>(r->finished - r->started).count();
    if (r->status != 0) {
      const std::string msg = r->error;
      s->forget(ticket);
      throw std::runtime_error(msg);
    }
    if (r->kind == fpls::kPredict) {
      if (!out || capacity_bytes < r->out.size())
        throw std::invalid_argument("prediction output buffer too small");
      std::memcpy(out, r->out.data(), r->out.size());
    }
    s->forget(ticket);
  });
}

FASTPLS_B200_API int fastpls_b200_server_release(void* server, unsigned long long model,
                                                 char* error, size_t error_capacity) {
  return guard(error, error_capacity, [&] {
    if (!server) throw std::invalid_argument("null server");
    static_cast<Server*>(server)->release_model(model);
  });
}

FASTPLS_B200_API int fastpls_b200_server_stats(void* server, size_t* bytes_in_use,
                                               size_t* queued, size_t* resident_models) {
  if (!server) return 1;
  static_cast<Server*>(server)->stats(bytes_in_use, queued, resident_models);
  return 0;
}

FASTPLS_B200_API int fastpls_b200_server_batch_stats(void* server, size_t* launches,
                                                     size_t* fits) {
  if (!server) return 1;
  static_cast<Server*>(server)->batch_stats(launches, fits);
  return 0;
}

FASTPLS_B200_API int fastpls_b200_server_set_borrow(void* server, int on) {
  if (!server) return 1;
  static_cast<Server*>(server)->borrow = on != 0;
  return 0;
}

}  // extern "C"
