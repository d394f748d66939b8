// Small dense FP64 linear algebra executed inside one block (device code).
#pragma once

#include "common.cuh"

namespace fpls {

// Cyclic Jacobi eigen-decomposition of a symmetric m x m matrix held in
// shared memory (column-major A[i + j*m]); eigenvectors accumulate in E.
// Executed by the first warp of the block; the caller synchronises after.
// Returns the number of sweeps used (<= max_sweeps).
__device__ inline int jacobi_eigen_warp(double* A, double* E, int m,
                                        int max_sweeps = 40) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x >= 32) return 0;
  for (int k = lane; k < m * m; k += 32) E[k] = (k % m == k / m) ? 1.0 : 0.0;
  __syncwarp();
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int k = lane; k < m * m; k += 32) {
      const int i = k % m, j = k / m;
      if (i != j) off += A[k] * A[k];
      else diag += A[k] * A[k];
    }
    off = warp_sum(off);
    diag = warp_sum(diag);
    if (off <= 1e-30 * diag || off == 0.0) break;
    for (int pp = 0; pp < m - 1; ++pp) {
      for (int qq = pp + 1; qq < m; ++qq) {
        const double apq = A[pp + qq * m];
        if (apq == 0.0) continue;
        const double app = A[pp + pp * m], aqq = A[qq + qq * m];
        const double theta = (aqq - app) / (2.0 * apq);
        const double tt = (theta >= 0 ? 1.0 : -1.0) /
                          (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(tt * tt + 1.0), s = tt * c;
        __syncwarp();
        // A <- J^T A J with J the (pp, qq) rotation: columns then rows
        for (int k = lane; k < m; k += 32) {
          const double akp = A[k + pp * m], akq = A[k + qq * m];
          A[k + pp * m] = c * akp - s * akq;
          A[k + qq * m] = s * akp + c * akq;
        }
        __syncwarp();
        for (int k = lane; k < m; k += 32) {
          const double apk = A[pp + k * m], aqk = A[qq + k * m];
          A[pp + k * m] = c * apk - s * aqk;
          A[qq + k * m] = s * apk + c * aqk;
        }
        for (int k = lane; k < m; k += 32) {
          const double ekp = E[k + pp * m], ekq = E[k + qq * m];
          E[k + pp * m] = c * ekp - s * ekq;
          E[k + qq * m] = s * ekp + c * ekq;
        }
        __syncwarp();
      }
    }
  }
  __syncwarp();
  return sweep;
}

// In-place Cholesky (lower) of an SPD k x k matrix A (+ ridge on the
// diagonal), one thread. Returns false on a non-positive or non-finite pivot.
__device__ inline bool cholesky_serial(double* A, int k, double ridge) {
  for (int i = 0; i < k; ++i) {
    for (int j = 0; j <= i; ++j) {
      double v = A[i + j * k] + (i == j ? ridge : 0.0);
      for (int q = 0; q < j; ++q) v -= A[i + q * k] * A[j + q * k];
      if (i == j) {
        if (!(v > 0.0) || !isfinite(v)) return false;
        A[i + i * k] = sqrt(v);
      } else {
        A[i + j * k] = v / A[j + j * k];
      }
    }
  }
  return true;
}

// Solve L L^T x = b in place (L lower, k x k, column-major), one thread.
__device__ inline bool cholesky_solve_serial(const double* L, int k, double* b) {
  for (int i = 0; i < k; ++i) {
    double v = b[i];
    for (int q = 0; q < i; ++q) v -= L[i + q * k] * b[q];
    b[i] = v / L[i + i * k];
  }
  for (int i = k - 1; i >= 0; --i) {
    double v = b[i];
    for (int q = i + 1; q < k; ++q) v -= L[q + i * k] * b[q];
    b[i] = v / L[i + i * k];
    if (!isfinite(b[i])) return false;
  }
  return true;
}

}  // namespace fpls
