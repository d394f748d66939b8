// Small dense FP64 linear algebra executed inside one block (device code).
#pragma once

#include "common.cuh"

namespace fpls {

// Jacobi eigen-decomposition of a symmetric m x m matrix held in shared
// memory (column-major A[i + j*m]); eigenvectors accumulate in E.
// Parallel ordering (Brent-Luk round robin): each sweep runs m - 1 (m even)
// or m (m odd) rounds of disjoint rotations. The rotations of a round go in
// groups of 32, one per lane: each lane computes its rotation, then the group
// is applied (columns of A and E, then rows of A). Rotations of one round
// touch disjoint rows and columns, so a rotation's 2 x 2 block is unchanged
// by the others of its round. Each rotation annihilates A[p, q] as in the
// classical cyclic method (tangent of the smaller root of t^2 + 2 theta t = 1,
// theta = (a_qq - a_pp) / (2 a_pq)).
// Executed by the first warp of the block; the caller synchronises after.
// Returns the number of sweeps used (<= max_sweeps). GMAX bounds the groups
// of 32 rotations per round: m <= 64 GMAX.
template <int GMAX = 1>
__device__ inline int jacobi_eigen_warp(double* A, double* E, int m,
                                        int max_sweeps = 40) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x >= 32) return 0;
  for (int k = lane; k < m * m; k += 32) E[k] = (k % m == k / m) ? 1.0 : 0.0;
  __syncwarp();
  const int players = m + (m & 1);  // a dummy player for odd m sits out
  const int half = players / 2;     // rotations per round
  const int groups = (half + 31) / 32;
  // round-robin schedule (circle method): slot 0 pairs the fixed player
  // players-1 with player `round`; slot s >= 1 pairs (round + s) and
  // (round - s) modulo players-1, so both advance by one each round
  int sa[GMAX], sb[GMAX];  // this lane's slots g*32 + lane, g < groups
  const int wrap = players - 1;
  // this lane's first work item (rotation k, row i) of a group, and the
  // step between items 32 apart: k += dk, i += di with carry
  const int dk = 32 / m, di = 32 % m;
  const int k0 = lane / m, i0 = lane % m;
  int sweep = 0;
  double prev = 0.0;
  for (; sweep < max_sweeps && m > 1; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int k = lane; k < m * m; k += 32) {
      const int i = k % m, j = k / m;
      if (i != j) off += A[k] * A[k];
      else diag += A[k] * A[k];
    }
    off = warp_sum(off);
    diag = warp_sum(diag);
    if (off <= 1e-30 * diag || off == 0.0) break;
    // at the rounding floor (large m) the off-diagonal mass stops shrinking
    if (sweep > 0 && off <= 1e-24 * diag && off > 0.25 * prev) break;
    prev = off;
#pragma unroll
    for (int g = 0; g < GMAX; ++g) {
      const int slot = g * 32 + lane;
      sa[g] = slot == 0 ? wrap : slot % wrap;
      sb[g] = slot == 0 ? 0 : (wrap - slot % wrap) % wrap;
    }
    for (int round = 0; round < wrap; ++round) {
#pragma unroll
      for (int g = 0; g < GMAX; ++g) {
        if (g >= groups) break;
        const int count = min(32, half - g * 32);
        int p = 0, q = 0;
        double c = 1.0, s = 0.0;
        if (lane < count) {
          const int a = min(sa[g], sb[g]), b = max(sa[g], sb[g]);
          if (b < m) {
            p = a;
            q = b;
            const double apq = A[p + q * m];
            if (apq != 0.0) {
              // t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)) with
              // theta = d / e, d = a_qq - a_pp, e = 2 a_pq, written as
              // sgn(d) e / (|d| + sqrt(d^2 + e^2)): one square root and one
              // division on the dependent path instead of two of each
              const double d = A[q + q * m] - A[p + p * m], e = 2.0 * apq;
              const double tt = (d >= 0 ? e : -e) / (fabs(d) + sqrt(fma(d, d, e * e)));
              c = rsqrt(fma(tt, tt, 1.0));
              s = tt * c;
            }
          }
        }
        __syncwarp();
        const int work = count * m;
        // A <- A J and E <- E J: columns p, q of every rotation of the group
        int k = k0, i = i0;
        for (int w = lane; w - lane < work; w += 32) {
          const int kk = w < work ? k : 0;
          const int pk = __shfl_sync(0xffffffffu, p, kk);
          const int qk = __shfl_sync(0xffffffffu, q, kk);
          const double ck = __shfl_sync(0xffffffffu, c, kk);
          const double sk = __shfl_sync(0xffffffffu, s, kk);
          if (w < work && sk != 0.0) {
            const double akp = A[i + pk * m], akq = A[i + qk * m];
            A[i + pk * m] = ck * akp - sk * akq;
            A[i + qk * m] = sk * akp + ck * akq;
            const double ekp = E[i + pk * m], ekq = E[i + qk * m];
            E[i + pk * m] = ck * ekp - sk * ekq;
            E[i + qk * m] = sk * ekp + ck * ekq;
          }
          k += dk;
          i += di;
          if (i >= m) {
            i -= m;
            ++k;
          }
        }
        __syncwarp();
        // A <- J^T A: rows p, q of every rotation of the group
        k = k0;
        i = i0;
        for (int w = lane; w - lane < work; w += 32) {
          const int kk = w < work ? k : 0;
          const int pk = __shfl_sync(0xffffffffu, p, kk);
          const int qk = __shfl_sync(0xffffffffu, q, kk);
          const double ck = __shfl_sync(0xffffffffu, c, kk);
          const double sk = __shfl_sync(0xffffffffu, s, kk);
          if (w < work && sk != 0.0) {
            const double apk = A[pk + i * m], aqk = A[qk + i * m];
            A[pk + i * m] = ck * apk - sk * aqk;
            A[qk + i * m] = sk * apk + ck * aqk;
          }
          k += dk;
          i += di;
          if (i >= m) {
            i -= m;
            ++k;
          }
        }
        __syncwarp();
        // next round: slots >= 1 advance both players by one
        const int slot = g * 32 + lane;
        if (slot == 0) {
          ++sb[g];
        } else {
          sa[g] = sa[g] + 1 == wrap ? 0 : sa[g] + 1;
          sb[g] = sb[g] + 1 == wrap ? 0 : sb[g] + 1;
        }
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
