// Batched SIMPLS over CV folds x response permutations x component path
// (host interface; see batched.cu).
#pragma once

#include "kernels.cuh"
#include "ozaki.cuh"

#include <vector>

namespace fpls {

constexpr int kBatchMaxResponses = 32;
// Instance groups run as up to batch_lanes() interleaved stream lanes of at
// least kLaneMinInstances instances each (process-wide setting, 1..4).
constexpr int kLaneMinInstances = 32;
int& batch_lanes();

template <class T>
struct BatchedCv {
  // Runs every (fold, permutation) instance. X, Y and perms are device
  // pointers (X n x p, Y n x q column-major; perms P x n zero-based source
  // rows, instance 0 uses the observed order); folds and prefixes are host.
  void run(const T* X, int n, int p, const T* Y, int q, const int* folds,
           const int* perms, int perm_count, const int* prefixes,
           int prefix_count, int scaling, cudaStream_t stream);
  // Metrics per (permutation + 1) x prefix, row-major by instance group:
  // index b * prefix_count + j, b = 0 the observed responses.
  void metrics(int metric, double* metric_out, double* q2, double* rmsd,
               double* r2) const;
  // Classification (class_labels set before run): held-out accuracy of the
  // argmax head per (permutation + 1) x prefix, same layout as metrics.
  void accuracy(double* out) const;

  // zero-based class of each base row (device, n) for classification, with
  // Y the one-hot indicator of the classes; null for regression
  const int* class_labels = nullptr;

  std::vector<int> status;          // per fold: 1 fitted, 2 empty
  std::vector<double> inst_sse;     // (P+1) x folds x prefixes
  std::vector<double> inst_sst;     // (P+1) x folds
  std::vector<int> heldout;         // held-out rows per fold
  long double total_ss = 0.0L;

 private:
  void form_gram(const double* kscale, cudaStream_t s);
  void run_group(const std::vector<int>& inst_fold,
                 const std::vector<int>& inst_perm, cudaStream_t s);
  // out (n x cols) = K rhs, rhs n x cols column-major (ld n): FP64 DMMA or,
  // when digits > 0, the int8 split product with the digits of K prepared by
  // form_gram (rhs_split receives the digits of rhs).
  void gram_product(const double* rhs, int cols, double* out, OzakiOperand& rhs_split,
                    cudaStream_t s);

  const T* X = nullptr;
  const int* perms = nullptr;
  int n = 0, p = 0, q = 0, P = 0, prefix_count = 0, scaling = 1, kmax = 0;
  int folds = 0, max_test = 1;
  bool center = true;
  int digits = 0;                 // int8 digits per FP64 value (0: FP64 DMMA)
  OzakiOperand gram_split, x_split;
  DeviceArray<double> gram, Y64, x64;
  DeviceArray<int> d_fold, d_ntrain, d_test_rows, d_test_off, d_slot, flag;
};

}  // namespace fpls
