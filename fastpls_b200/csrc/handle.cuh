// Resident model handle behind the C ABI (host code).
//
// Mirrors the contract of the reference's TypedResidentHandle
// (src/cuda_resident_api.cuh:69-479): one non-blocking stream per handle,
// every call synchronous, host buffers borrowed only for the call, outputs in
// the caller's precision (32 or 64), errors as exceptions turned into
// strings at the ABI.
#pragma once

#include "kernels.cuh"
#include "model.cuh"

#include <memory>

namespace fpls {

struct LdaState;        // lda.cu
struct PersistentPlan;  // persistent.cuh

class ResidentHandle {
 public:
  virtual ~ResidentHandle() = default;
  virtual void predict_path(const void* x, int rows, const int* prefixes,
                            int count, bool lda, void* out) = 0;
  virtual void classify_path(const void* x, int rows, const int* prefixes,
                             int count, bool lda, int top, int* out,
                             void* response_out) = 0;
  virtual void project(const void* x, int rows, int prefix, void* out) = 0;
  virtual void response_sums(const void* x, const void* y, const int* labels,
                             int rows, int prefix, void* out) = 0;
  virtual void export_field(int field, void* out, std::size_t size) = 0;
  virtual void controls(int* oversample, int* power, int* block,
                        int* block_limit, int* implicit_operator,
                        int* crossprod_cache) = 0;
  virtual void compact(bool prepare_lda) = 0;
  virtual void vip(double* out, std::size_t size) = 0;
  // A fit made with make_handle(..., defer = true) may leave its persistent
  // launch pending: the plan to launch (with others), the handle's stream
  // (to order after that launch), and the step that finishes the fit.
  virtual PersistentPlan* pending_plan() { return nullptr; }
  virtual cudaStream_t stream() const { return nullptr; }
  virtual void complete_fit() {}
};

struct FitRequest {
  int method = kSimpls;
  const void* x = nullptr;
  const void* y = nullptr;
  const int* labels = nullptr;
  int n = 0, p = 0, q = 0, components = 0, scaling = 1;
  int oversample = 32, power = 5;
  bool retain_scores = true;
  unsigned long long seed = 1;
  int north = 0, kernel = 0, degree = 3;
  double gamma = 0.0, coef0 = 1.0;
};

ResidentHandle* make_handle(int precision, const FitRequest& request, bool defer = false);

// A fitted SIMPLS or OPLS model rebuilt from its exported fields (R, Q, the
// predictor means and scales, the response means; optionally the training
// scores T and labels for LDA), so a model saved by the host survives without
// refitting. FP64 host arrays; `precision` is that of later prediction rows.
struct ImportRequest {
  int method = kSimpls;
  int n = 0, p = 0, q = 0, components = 0, scaling = 1;
  bool classification = false;
  const double* R = nullptr;      // p x a
  const double* Q = nullptr;      // q x a
  const double* T = nullptr;      // n x a (optional)
  const double* mean = nullptr;   // p
  const double* scale = nullptr;  // p
  const double* ymean = nullptr;  // q
  const int* labels = nullptr;    // n, one-based (optional, needs T)
};

ResidentHandle* import_handle(int precision, const ImportRequest& request);

// Device time of the calling thread's last resident fit (CUDA events on the
// handle's stream): the input copies and the fit proper, in milliseconds.
struct FitTimes;
FitTimes& last_fit_times();
void read_last_fit_times(double* copy_ms, double* fit_ms);

}  // namespace fpls
