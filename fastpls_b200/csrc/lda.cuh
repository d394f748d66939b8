// LDA on latent scores (host interface; see lda.cu).
#pragma once

#include "kernels.cuh"

#include <deque>
#include <vector>

namespace fpls {

struct LdaState {
  int n = 0, a = 0, c = 0;
  int* flag = nullptr;
  DeviceArray<double> gram;        // a x a  (T^T T)
  DeviceArray<double> sums;        // c x a  (per-class score sums)
  DeviceArray<double> counts_dev;  // c
  struct Prefix {
    int k = 0;
    DeviceArray<double> linear;     // c x k
    DeviceArray<double> constants;  // c (+ ridge at [c])
  };
  std::deque<Prefix> prefixes;

  // scores: n x a (ld lds) training scores; labels: one-based device labels.
  void train(const double* scores, int n, long lds, int a, const int* labels,
             int c, const std::vector<int>& counts, int* flag,
             cudaStream_t stream);
  const Prefix& prefix(int k, cudaStream_t stream);
  // out (rows x c) = constants + scores_k linear^T
  void discriminants(const double* scores, int rows, long lds, int k,
                     double* out, long ldo, cudaStream_t stream);
};

}  // namespace fpls
