// Persistent single-fit SIMPLS (one cooperative launch per fit; see
// persistent.cu).
#pragma once

#include "model.cuh"

namespace fpls {

constexpr int kPersistMaxResponses = 32;
constexpr int kPersistMaxComponents = 256;

// Whether the persistent path takes a fit with m responses and a components.
bool persistent_supported(int m, int a);

// Runs the whole component loop of a SIMPLS fit (one direction per
// component, no candidate blocks) as one cooperative launch, from S (p x m,
// deflated in place), its packed Gram gpk, and model.{mean, scale, S0};
// fills model.{R, Q, V, T}. Returns false (nothing enqueued) when the shape
// or the device does not allow it; the caller then runs the per-kernel loop.
template <class T>
bool fit_simpls_persistent(const T* X, int n, int p, long ld, int m, int a, DeviceModel& model,
                           double* S, double* gpk, Workspace& ws, cudaStream_t stream);

// Process-wide switch (1 = use the persistent path where it applies).
int& persistent_enabled();

}  // namespace fpls
