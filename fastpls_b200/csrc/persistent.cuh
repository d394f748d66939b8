// Persistent single-fit SIMPLS (one cooperative launch for every component
// of one or several fits; see persistent.cu).
#pragma once

#include "model.cuh"

#include <memory>
#include <vector>

namespace fpls {

constexpr int kPersistMaxResponses = 32;
constexpr int kPersistMaxComponents = 256;
// Largest fit (n p elements of X) that runs as one persistent launch.
constexpr long kPersistMaxElements = 1L << 26;

// Device-side description of one fit of a persistent launch.
struct PersistentFit {
  const void* X;
  long ld;
  int n, p, m, a;
  const double* mean;
  const double* scale;
  const double* S0;
  double *S, *R, *V, *Q, *T;
  double* gpk;              // packed Gram of S (m (m + 1) / 2)
  double *pv, *v;           // p
  double* tpart;            // Cc x n (scores pass, one row per column range)
  double* ppart;            // Cr x p (loading pass, one row per row block)
  double* cpart;            // C x cslots (per-CTA partials)
  double* gpart;            // ceil(C / 32) x cslots (per-group sums)
  double* scal;             // scalar slots
  unsigned* bar;            // [groups arrived, generation, CTAs arrived per group...]
  int* flag;                // the fit's error flag
  int cta0, C;              // CTA range of this fit in the launch
  int Cr, rb;               // row blocks of X and their rows (C = Cr Cc)
  int Cc, pc;               // column ranges of X and their columns
  int elem;                 // bytes per element of X
  int cslots;               // per-CTA partial slots
  long long barrier_cycles; // bound of each barrier wait
  int absent_cta;           // test of the bounded waits: this CTA never arrives (-1: none)
};

// One planned fit: its descriptor and the scratch it owns until the launch
// has finished (every buffer is freed stream-ordered on the fit's stream).
struct PersistentPlan {
  PersistentFit fit{};
  int elem = 0;  // bytes per stored element of X (2 BF16, 4 FP32, 8 FP64)
  DeviceArray<double> S, part, cpart, scal;
  DeviceArray<unsigned> bar;
};

// Whether the persistent path takes a fit with m responses and a components.
bool persistent_supported(int m, int a);
// CTAs a fit of n x p gets (a function of the shape only; 0: the shape does
// not fit a persistent launch).
int persistent_ctas(int n, int p);
// CTAs one launch can hold co-resident for a storage type (0: unavailable).
int persistent_capacity(int elem);

// Plans the whole component loop of a SIMPLS fit (one direction per
// component) from S (p x m, deflated in place; the plan takes it over) and
// model.{mean, scale, S0}, to fill model.{R, Q, V, T}; gpk receives the
// packed Gram of the deflated S.
// Returns false (nothing planned, S untouched) when the shape or the device
// does not allow it.
template <class T>
bool plan_simpls_persistent(const T* X, int n, int p, long ld, int m, int a, DeviceModel& model,
                            DeviceArray<double>& S, double* gpk, Workspace& ws, cudaStream_t stream,
                            PersistentPlan& plan);

// One cooperative launch for the planned fits (one storage type, total CTAs
// within persistent_capacity) on `stream`, which must already be ordered
// after the work that produced each plan.
void launch_persistent(const std::vector<PersistentPlan*>& plans, cudaStream_t stream);

// When set on this thread, a SIMPLS fit that plans a persistent launch hands
// the plan to *sink instead of launching it (the caller batches plans).
std::unique_ptr<PersistentPlan>*& persistent_deferral();

// Process-wide switch (1 = use the persistent path where it applies).
int& persistent_enabled();

// Test of the bounded barrier waits: with absent set, CTA 0 of every fit
// leaves before its first barrier, so the other CTAs' waits run out after
// `cycles` clocks; they set the fit's error flag (5) and return, and the fit
// reports an error. cycles <= 0 keeps the default bound (about 2 s).
struct PersistentWaitTest {
  int absent = 0;
  long long cycles = 0;
};
PersistentWaitTest& persistent_wait_test();

}  // namespace fpls
