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
constexpr int kMaxLanes = 4;
int& batch_lanes();
// Relative top-two margin under which a held-out class decision made with
// int8 products is refitted with FP64 products (process-wide; 0 disables),
// and the number of instances the last batched classification run refitted.
double& argmax_guard();
int& last_guard_refits();
// Autotuning of the group schedule (lanes x tile width), keyed on
// (n, p, q, instances, components, digits): 1 = time the candidates on the
// first group of a new key and keep the fastest (default), 0 = the fixed
// rule (batch_lanes() lanes, tile width from the wave count).
int& batch_autotune();
// Group statistics of the last batched call, for benchmarks and tests.
struct BatchedStats {
  int groups = 0;             // instance groups run
  int graph_replays = 0;      // group runs that replayed a captured CUDA graph
  int graph_captures = 0;     // graphs captured (first use of a group shape)
  int tuned = 0;              // groups whose schedule was chosen by timing
  int lanes = 0, tile_n = 0;  // schedule of the last group
};
BatchedStats& last_batched_stats();
// Frees the persistent per-device workspace of the batched engine (device
// buffers, lane streams and captured graphs); the next call rebuilds it.
void release_batched_workspace();

struct BatchedWorkspace;

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
  // classification head: false = argmax of the predicted indicators, true =
  // LDA on the latent scores (per instance, after the last component)
  bool lda_head = false;
  // (P+1) x folds, optional: instances the caller handles itself (not run;
  // their inst_sse entries are the caller's to fill after run)
  std::vector<unsigned char> skip;
  // (P+1) x folds, optional: candidate-block width of each instance (the
  // reference's block rule on its training rows and active classes); empty =
  // one direction per component everywhere
  std::vector<int> blocks;

  std::vector<int> status;          // per fold: 1 fitted, 2 empty (the caller may
                                    // set 4: one class in the training rows)
  std::vector<double> inst_sse;     // (P+1) x folds x prefixes
  std::vector<double> inst_sst;     // (P+1) x folds
  std::vector<int> heldout;         // held-out rows per fold
  long double total_ss = 0.0L;
  int refitted = 0;                 // classification instances refitted with
                                    // FP64 products by the argmax guard

 private:
  void form_gram(const double* kscale, cudaStream_t s);
  void run_group(const std::vector<int>& inst_fold,
                 const std::vector<int>& inst_perm, cudaStream_t s);
  // Enqueues the whole component sequence of one group (all lanes) on the
  // workspace's lane streams, forked from and joined back into s.
  void enqueue_group(int I, int nlanes, int tile_n, cudaStream_t s);
  // out (n x cols) = K rhs, rhs n x cols column-major (ld n): FP64 DMMA or,
  // when digits > 0, the int8 split product with the digits of K prepared by
  // form_gram (rhs_split receives the digits of rhs), tile width tile_n.
  void gram_product(const double* rhs, int cols, double* out, OzakiOperand& rhs_split,
                    int tile_n, cudaStream_t s);

  BatchedWorkspace* ws = nullptr;
  const T* X = nullptr;
  const int* perms = nullptr;
  int n = 0, p = 0, q = 0, P = 0, prefix_count = 0, scaling = 1, kmax = 0;
  int folds = 0, max_test = 1;
  bool center = true;
  int digits = 0;                 // int8 digits per FP64 value (0: FP64 DMMA)
  std::vector<int> amb_fold, amb_perm;  // instances flagged by the argmax guard
};

}  // namespace fpls
