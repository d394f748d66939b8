// Small dense FP64 linear algebra executed inside one block (device code).
#pragma once

#include "common.cuh"

namespace fpls {

// Jacobi eigen-decomposition of a symmetric m x m matrix (m <= 128) held in
// shared memory (column-major A[i + j*m]); eigenvectors accumulate in E.
// Parallel ordering (Brent-Luk round robin): each sweep runs m - 1 (m even)
// or m (m odd) rounds of up to m / 2 disjoint rotations. All threads of the
// block cooperate (every thread must call it, with the same arguments): the
// rotations of a round are computed one per thread into shared memory, then
// applied together, element by element over the block (columns of A and E,
// then rows of A). Rotations of one round touch disjoint rows and columns, so
// a rotation's 2 x 2 block is unchanged by the others of its round. Each
// rotation annihilates A[p, q] as in the classical cyclic method (tangent of
// the smaller root of t^2 + 2 theta t = 1, theta = (a_qq - a_pp) / (2 a_pq)).
// Stops at off <= 1e-30 diag (sums of squares) or at the rounding floor.
// Returns the number of sweeps used (<= max_sweeps). Matrices of order
// m <= warp_limit run in the first warp alone.
constexpr int kJacobiMaxRotations = 64;

// threads for a block that runs jacobi_eigen on an m x m matrix
inline unsigned jacobi_threads(int m) { return m > 16 ? 256u : 64u; }

__device__ inline int jacobi_eigen(double* A, double* E, int m, int max_sweeps = 40, int warp_limit = 8) {
  __shared__ int rot_p[kJacobiMaxRotations], rot_q[kJacobiMaxRotations];
  __shared__ double rot_c[kJacobiMaxRotations], rot_s[kJacobiMaxRotations];
  __shared__ double red[32];
  if (m > 2 * kJacobiMaxRotations) return 0;  // callers keep m <= 128
  // small matrices (m <= warp_limit): the first warp alone (warp barriers
  // are cheaper than block barriers on the latency-bound path); the other
  // threads wait at the final barrier
  const bool warp_only = m <= warp_limit;
  if (warp_only && threadIdx.x >= 32) {
    __syncthreads();
    return 0;
  }
  const int tid = threadIdx.x, nt = warp_only ? 32 : (int)blockDim.x;
  auto sync = [&]() {
    if (warp_only) __syncwarp();
    else __syncthreads();
  };
  auto total = [&](double v) { return warp_only ? warp_sum(v) : block_sum(v, red); };
  for (int k = tid; k < m * m; k += nt) E[k] = (k % m == k / m) ? 1.0 : 0.0;
  sync();
  const int players = m + (m & 1);  // a dummy player for odd m sits out
  const int half = players / 2;     // rotations per round (<= 64)
  const int wrap = players - 1;
  const int work = half * m;
  // this thread's first work item (rotation k, row i) and the step nt
  // between its items: k += dk, i += di with carry
  const int dk = nt / m, di = nt % m;
  const int k0 = tid / m, i0 = tid % m;
  int sweep = 0;
  double prev = 0.0;
  for (; sweep < max_sweeps && m > 1; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int k = tid; k < m * m; k += nt) {
      const int i = k % m, j = k / m;
      if (i != j) off += A[k] * A[k];
      else diag += A[k] * A[k];
    }
    off = total(off);
    diag = total(diag);
    if (off <= 1e-30 * diag || off == 0.0) break;
    // at the rounding floor (large m) the off-diagonal mass stops shrinking
    if (sweep > 0 && off <= 1e-24 * diag && off > 0.25 * prev) break;
    prev = off;
    // this thread's slot `tid` (one per thread when nt >= half) advances
    // incrementally; further slots (nt < half) use the closed form
    int sa = tid == 0 ? wrap : tid % wrap;
    int sb = tid == 0 ? 0 : (wrap - tid % wrap) % wrap;
    for (int round = 0; round < wrap; ++round) {
      for (int slot = tid; slot < half; slot += nt) {
        // circle method: player players-1 fixed, the others rotate
        int a = slot == tid ? sa : (slot == 0 ? wrap : (round + slot) % wrap);
        int b = slot == tid ? sb : (slot == 0 ? round : (round - slot + wrap) % wrap);
        if (a > b) {
          const int t = a;
          a = b;
          b = t;
        }
        double c = 1.0, s = 0.0;
        if (b < m) {
          const double apq = A[a + b * m];
          if (apq != 0.0) {
            // t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)) with
            // theta = d / e, d = a_qq - a_pp, e = 2 a_pq, written as
            // sgn(d) e / (|d| + sqrt(d^2 + e^2)): one square root and one
            // division on the dependent path instead of two of each
            const double d = A[b + b * m] - A[a + a * m], e = 2.0 * apq;
            const double tt = (d >= 0 ? e : -e) / (fabs(d) + sqrt(fma(d, d, e * e)));
            c = rsqrt(fma(tt, tt, 1.0));
            s = tt * c;
          }
        } else {
          a = b = 0;
        }
        rot_p[slot] = a;
        rot_q[slot] = b;
        rot_c[slot] = c;
        rot_s[slot] = s;
      }
      if (tid == 0) {
        ++sb;
      } else {
        sa = sa + 1 == wrap ? 0 : sa + 1;
        sb = sb + 1 == wrap ? 0 : sb + 1;
      }
      sync();
      // A <- A J and E <- E J: columns p, q of every rotation of the round
      {
        int k = k0, i = i0;
        for (int w = tid; w < work; w += nt) {
          const double sk = rot_s[k];
          if (sk != 0.0) {
            const int pk = rot_p[k], qk = rot_q[k];
            const double ck = rot_c[k];
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
      }
      sync();
      // A <- J^T A: rows p, q of every rotation of the round
      {
        int k = k0, i = i0;
        for (int w = tid; w < work; w += nt) {
          const double sk = rot_s[k];
          if (sk != 0.0) {
            const int pk = rot_p[k], qk = rot_q[k];
            const double ck = rot_c[k];
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
      }
      sync();
    }
  }
  __syncthreads();
  return sweep;
}

// Dominant eigenpair of a symmetric positive semidefinite m x m matrix A
// (shared, column-major), whole block. Repeated squaring: B = A / tr(A),
// then B <- B^2 / tr(B^2). For B of trace one, tr(B^2) is the sum of its
// squared eigenvalues, 1 exactly when B has rank one; each squaring raises
// the eigenvalue ratios to the power two, so once tr(B^2) >= 1 - 1e-12 two
// more squarings leave the non-dominant part below rounding. Then v = the
// column of B with the largest diagonal entry, normalised (B = v v^T up to
// rounding), and lam = v^T A v. On random SPD matrices up to 32 x 32
// (clustered, rank one, condition 1e12) the residual |A v - lam v| / |A|
// stays below 1e-15 in about 13 squarings (at most 64; an exactly repeated
// leading eigenvalue yields a vector of its eigenspace). B and C are m x m
// shared scratch (C with one extra slot), v (m + 1 slots) the shared
// output; lam is returned in every thread. Returns false when tr(A) is not
// positive and finite.
// dominant_pair for order M <= 4 in one thread's registers: the same
// operations in the same order as the shared-memory form below (so the same
// bits), without its barriers. A is read from shared memory; v (M + 1) and
// C[M] receive the result as in that form.
template <int M>
__device__ inline void dominant_pair_regs(const double* A, double* C, double* v, int max_squarings) {
  double a[M * M], b[M * M], c[M * M];
#pragma unroll
  for (int k = 0; k < M * M; ++k) a[k] = A[k];
  double tr = 0.0;
#pragma unroll
  for (int i = 0; i < M; ++i) tr += a[i * (M + 1)];
  if (!(tr > 0.0) || !isfinite(tr)) {
    v[M] = 0.0;
    C[M] = 0.0;
    return;
  }
  const double inv_tr = 1.0 / tr;
#pragma unroll
  for (int k = 0; k < M * M; ++k) b[k] = a[k] * inv_tr;
  int left = -1;
  for (int it = 0; it < max_squarings; ++it) {
#pragma unroll
    for (int k = 0; k < M * M; ++k) {
      const int i = k % M, j = k / M;
      double acc = 0.0;
#pragma unroll
      for (int l = 0; l < M; ++l) acc = fma(b[i + l * M], b[l + j * M], acc);
      c[k] = acc;
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < M; ++i) s += c[i * (M + 1)];
    if (left < 0 && 1.0 - s <= 1e-12) left = 2;
    if (left == 0) break;
    const double inv_s = 1.0 / s;
#pragma unroll
    for (int k = 0; k < M * M; ++k) b[k] = c[k] * inv_s;
    if (left > 0) --left;
  }
  int j = 0;
  double bjj = b[0];
#pragma unroll
  for (int i = 1; i < M; ++i)
    if (b[i * (M + 1)] > bjj) {
      bjj = b[i * (M + 1)];
      j = i;
    }
  double col[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    double bij = b[i];
#pragma unroll
    for (int jj = 1; jj < M; ++jj)
      if (jj == j) bij = b[i + jj * M];
    col[i] = bij;
  }
  double n2 = 0.0;
#pragma unroll
  for (int i = 0; i < M; ++i) n2 = fma(col[i], col[i], n2);
  const double inv_n = 1.0 / sqrt(n2);
  double vv[M];
#pragma unroll
  for (int i = 0; i < M; ++i) vv[i] = col[i] * inv_n;
  double lam = 0.0;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    double acc = 0.0;
#pragma unroll
    for (int l = 0; l < M; ++l) acc = fma(a[i + l * M], vv[l], acc);
    lam = fma(vv[i], acc, lam);
  }
#pragma unroll
  for (int i = 0; i < M; ++i) v[i] = vv[i];
  v[M] = 1.0;
  C[M] = lam;
}

constexpr int kDominantMaxOrder = 64;  // callers size 3 m^2 + m + 2 shared doubles up to this order
__device__ inline bool dominant_pair(const double* A, double* B, double* C, double* v, int m,
                                     double& lam, int max_squarings = 64) {
  // orders up to 8: the first warp alone with warp barriers (the squarings
  // are a few FMAs per lane; block barriers would dominate); the other
  // warps wait at the final barrier and read lam from the shared v slot
  if (m <= 4) {
    // one thread, registers only
    if (threadIdx.x == 0) {
      if (m == 1) dominant_pair_regs<1>(A, C, v, max_squarings);
      else if (m == 2) dominant_pair_regs<2>(A, C, v, max_squarings);
      else if (m == 3) dominant_pair_regs<3>(A, C, v, max_squarings);
      else dominant_pair_regs<4>(A, C, v, max_squarings);
    }
    __syncthreads();
    const bool found = v[m] != 0.0;
    lam = C[m];
    __syncthreads();
    return found;
  }
  const bool one_warp = m <= 8;
  if (one_warp && threadIdx.x >= 32) {
    __syncthreads();
    const bool found = v[m] != 0.0;
    lam = C[m];
    __syncthreads();
    return found;
  }
  const int tid = threadIdx.x, nt = one_warp ? 32 : blockDim.x, mm = m * m;
  auto sync = [&] {
    if (one_warp) __syncwarp();
    else __syncthreads();
  };
  // the result for the other warps (one_warp): v[m] = found, C[m] = lam
  auto finish = [&](bool found, double l) {
    if (one_warp) {
      if (tid == 0) {
        v[m] = found ? 1.0 : 0.0;
        C[m] = l;
      }
      __syncwarp();
      __syncthreads();
      __syncthreads();
    }
    return found;
  };
  double tr = 0.0;
  for (int i = 0; i < m; ++i) tr += A[i * (m + 1)];
  if (!(tr > 0.0) || !isfinite(tr)) {
    lam = 0.0;
    return finish(false, 0.0);
  }
  const double inv_tr = 1.0 / tr;
  for (int k = tid; k < mm; k += nt) B[k] = A[k] * inv_tr;
  sync();
  int left = -1;  // squarings still to run once converged
  for (int it = 0; it < max_squarings; ++it) {
    for (int k = tid; k < mm; k += nt) {
      const int i = k % m, j = k / m;
      double acc = 0.0;
      for (int l = 0; l < m; ++l) acc = fma(B[i + l * m], B[l + j * m], acc);
      C[k] = acc;
    }
    sync();
    double s = 0.0;  // tr(B^2), the same in every thread
    for (int i = 0; i < m; ++i) s += C[i * (m + 1)];
    if (left < 0 && 1.0 - s <= 1e-12) left = 2;
    if (left == 0) break;
    const double inv_s = 1.0 / s;
    for (int k = tid; k < mm; k += nt) B[k] = C[k] * inv_s;
    sync();
    if (left > 0) --left;
  }
  int j = 0;
  for (int i = 1; i < m; ++i)
    if (B[i * (m + 1)] > B[j * (m + 1)]) j = i;
  double n2 = 0.0;
  for (int i = 0; i < m; ++i) n2 = fma(B[i + j * m], B[i + j * m], n2);
  const double inv_n = 1.0 / sqrt(n2);
  sync();  // every thread has read B
  for (int i = tid; i < m; i += nt) v[i] = B[i + j * m] * inv_n;
  sync();
  for (int i = tid; i < m; i += nt) {
    double acc = 0.0;
    for (int l = 0; l < m; ++l) acc = fma(A[i + l * m], v[l], acc);
    C[i] = acc;
  }
  sync();
  lam = 0.0;
  for (int i = 0; i < m; ++i) lam = fma(v[i], C[i], lam);
  sync();
  return finish(true, lam);
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
