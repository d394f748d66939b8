// Kernel launchers of the fitting library (declarations).
#pragma once

#include "common.cuh"

namespace fpls {

// ---------------------------------------------------------------- gemm.cu
struct GemmArgs {
  int M = 0, N = 0, K = 0;
  const void* A = nullptr;
  long lda = 0;
  bool a_f32 = false, trans_a = false;
  const void* B = nullptr;
  long ldb = 0;
  bool b_f32 = false, trans_b = false;
  const double* kscale = nullptr;  // optional diag(kscale) between op(A), op(B)
  double alpha = 1.0, beta = 0.0;
  double* C = nullptr;
  long ldc = 0;
  int splits = 1;         // split-K slices (beta must be 0 when > 1)
  long split_stride = 0;  // element stride between partial slices of C
  bool lower = false;     // symmetric result: compute lower tiles, mirror
};
void gemm_f64(const GemmArgs& g, cudaStream_t stream);
int gemm_pick_splits(int M, int N, int K);
void gemm_profile_enable(bool on);
// DMMA tensor-core path (gemm_mma.cu): FP64 A (not transposed), FP64 B,
// 16-byte aligned operands with even leading dimensions.
bool gemm_mma_supported(const GemmArgs& g);
void gemm_mma_launch(const GemmArgs& g, bool lower, cudaStream_t stream);
void mirror_lower_triangle(double* C, int n, long ldc, cudaStream_t stream);
void gemm_profile_read(double* ms, double* flops, unsigned long long* launches);

// Stream that the batched entry points run on when the caller set one
// (fastpls_b200_set_stream); nullptr means "create a private stream".
cudaStream_t& caller_stream();

// Measured FP64 FMA throughput of the device (TFLOP/s), probe.cu.
double fp64_fma_tflops();

// -------------------------------------------------------------- stream.cu
// Column moments of X (n x p, column-major, leading dimension ld):
// sum[j], sumsq[j] and cross[j + c*p] = sum_i X[i,j] * Yc[i,c] (FP64),
// Yc an n x m FP64 column-major block (m may be 0). One pass over X.
template <class T>
void column_moments(const T* X, int n, int p, long ld, const double* Yc, int m,
                    double* sum, double* sumsq, double* cross,
                    DeviceArray<double>& scratch, cudaStream_t stream);

// Classification: sum[j], sumsq[j] and cross[j + c*p] = X^T (onehot - prior)
// from one-based labels (n), classes m <= kClassMomentsMaxClasses, in one
// pass over X (per-class column sums minus prior * column sum).
constexpr int kClassMomentsMaxClasses = 32;
template <class T>
void class_moments(const T* X, int n, int p, long ld, const int* labels, int m,
                   const double* prior, double* sum, double* sumsq, double* cross,
                   DeviceArray<double>& scratch, cudaStream_t stream);

// out[i + c*n] = sum_j X[i,j] * R[j + c*ldr] - offset[c]   (c < nb)
// (scores of a scaled/centred X folded into R and offset). FP64 result.
// flag (optional): set to 5 if a bulk-copy stage of the one-pass form never
// arrives (a bounded wait ran out).
template <class T>
void xr_product(const T* X, int n, int p, long ld, const double* R, long ldr,
                int nb, const double* offset, double* out, long ldo,
                DeviceArray<double>& scratch, cudaStream_t stream, int* flag = nullptr);

// The one-pass form of xr_product for 3 <= nb <= 16 columns (persistent.cu):
// X streamed once through the single fit's bulk-copy stages, each stage also
// carrying its rows of R. Returns false (nothing enqueued) for shapes it does
// not take.
template <class T>
bool xr_ring(const T* X, int n, int p, long ld, const double* R, long ldr, int nb,
             const double* offset, double* out, long ldo, int* flag, cudaStream_t stream);

// out[j + c*p] = sum_i X[i,j] * V[i + c*ldv]   (c < nb, FP64)
template <class T>
void xtv_product(const T* X, int n, int p, long ld, const double* V, long ldv,
                 int nb, double* out, long ldo, DeviceArray<double>& scratch,
                 cudaStream_t stream);

// Copy rows idx[0..count) of a column-major (rows x cols) matrix.
template <class T>
void gather_rows(const T* src, long ld_src, int cols, const int* idx, int count,
                 T* dst, long ld_dst, cudaStream_t stream);

// ---------------------------------------------------------------- misc
// One-based top-k per row of a column-major (rows x classes) FP64 matrix;
// the lower class index wins ties (strict '>' scan).
void topk_rows(const double* values, int rows, int classes, int top, int* out,
               long ldo, cudaStream_t stream);

}  // namespace fpls
