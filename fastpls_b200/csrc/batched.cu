// Batched SIMPLS over many fits that share one predictor matrix: the folds of
// a cross-validation, each refitted on permuted responses (permutation test)
// and evaluated along the whole component path (ncomp sweep).
//
// Reference semantics: every instance is the fold fit of
// resident_pls_cv_regression (src/cuda_resident_api.cuh:770-1023) /
// cross_validate_regression (cross_validation.hpp:1790-2173) on the responses
// Y[perm] (permutation refits, R/main.R:9419-9450 and 12048-12080: folds and
// solver fixed across the observed and null fits).
//
// B200 design -- kernel-form SIMPLS in sample space:
//   SIMPLS only ever touches X through products with vectors that live in
//   the row space of the centred training block Xf. Writing every p-vector as
//   Xf^T (n-vector) turns both per-component products into products with the
//   Gram K = X D^2 X^T (n x n, FP64, formed once per scaling group):
//     t_F  = P_F (K u~)_F          scores of the training rows
//     t_te = (K u~)_te - mean_F((K u~)_F)   scores of the held-out rows
//     K t  = P_F (K t~)_F          loading step (t~ = t on F, 0 elsewhere)
//   with P_F the centring projector over the training rows F. Fold masks make
//   every instance (fold x permutation) a column of ONE n x I right-hand side,
//   so a component step for all instances is two FP64 GEMMs with the shared K
//   (gemm.cu) plus O(n a) vector work per instance. The held-out scores fall
//   out of the same product, so the prefix-path predictions and their SSE are
//   accumulated on the fly; no p-length vector is ever formed.
//   Orthogonalisation of the deflation basis uses V^T p = W^T K t = KW^T t
//   with W (coefficients) and KW stored per instance, FP64 throughout.
#include "batched.cuh"
#include "kernels.cuh"
#include "reduce.cuh"
#include "small.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

namespace fpls {

namespace {

constexpr int BT = 256;
// The deflation runs one CTA per instance through dependent phases; 128
// threads keep every instance of a lane (~670) resident in one wave.
constexpr int DEFL_BT = 128;

struct InstanceView {
  int n, q, kmax, B;        // rows, responses, max components, perms per fold
  int center;               // 1: centre over training rows (scaling 1, 2)
  const int* fold_of_row;   // n (one-based)
  const int* inst_fold;     // I: fold index (0-based)
  const int* inst_perm;     // I: permutation index (-1 = identity)
  const int* perms;         // P x n (0-based source rows)
  const int* ntrain;        // per fold
  const int* test_rows;     // concatenated held-out rows per fold
  const int* test_off;      // F + 1
  const double* Y;          // n x q base responses (FP64)
  const int* labels;        // n zero-based classes of the base rows, or null
                            // (regression); classification counts hits
};

__device__ __forceinline__ int src_row(const InstanceView& v, int perm, int r) {
  return perm < 0 ? r : v.perms[(long)perm * v.n + r];
}

// One held-out row at a prefix slot: squared error over the responses
// (regression), or 1 when the argmax over the classes present in the
// instance's training rows (prior > 0; first index wins ties) is the row's
// class (classification, as the reference's argmax head over its active
// classes, src/cuda_resident_api.cuh:700-745).
__device__ __forceinline__ double heldout_term(const InstanceView& v, int i, int b, int r,
                                               const double* ymean, const double* yh, long ld) {
  const int q = v.q;
  if (v.labels) {
    int best = -1;
    double bv = 0.0;
    for (int c = 0; c < q; ++c) {
      const double ym = ymean[(long)i * q + c];
      if (ym > 0.0) {
        const double score = ym + yh[(long)c * ld];
        if (best < 0 || score > bv) {
          best = c;
          bv = score;
        }
      }
    }
    return best == v.labels[src_row(v, b, r)] ? 1.0 : 0.0;
  }
  double err = 0.0;
  for (int c = 0; c < q; ++c) {
    const double e = v.Y[src_row(v, b, r) + (long)c * v.n] - (ymean[(long)i * q + c] + yh[(long)c * ld]);
    err = fma(e, e, err);
  }
  return err;
}

// C0 (n x q) = responses of this instance centred over its training rows
// (zero on held-out rows); ymean; held-out SS about the training mean.
__global__ void init_instances(InstanceView v, double* C0, double* C,
                               double* ymean, double* sst, double* yhat,
                               int yhat_ld, double* sse, int prefix_count) {
  __shared__ double scratch[32];
  const int i = blockIdx.x;
  const int f = v.inst_fold[i], b = v.inst_perm[i];
  const int n = v.n, q = v.q;
  double* c0 = C0 + (long)i * n * q;
  double* c = C + (long)i * n * q;
  const int nt = v.ntrain[f];
  double tss = 0.0;
  for (int col = 0; col < q; ++col) {
    double s = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x)
      if (v.fold_of_row[r] != f + 1) s += v.Y[src_row(v, b, r) + (long)col * n];
    const double mu = block_sum(s, scratch) / nt;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const bool train = v.fold_of_row[r] != f + 1;
      const double y = v.Y[src_row(v, b, r) + (long)col * n];
      const double val = train ? y - mu : 0.0;
      c0[r + (long)col * n] = val;
      c[r + (long)col * n] = val;
      if (!train) tss = fma(y - mu, y - mu, tss);
    }
    if (threadIdx.x == 0) ymean[(long)i * q + col] = mu;
  }
  tss = block_sum(tss, scratch);
  if (threadIdx.x == 0) sst[i] = tss;
  const int nte = v.test_off[f + 1] - v.test_off[f];
  double* yh = yhat + (long)i * yhat_ld * q;
  for (int k = threadIdx.x; k < nte * q; k += blockDim.x) yh[(k % nte) + (long)(k / nte) * yhat_ld] = 0.0;
  for (int k = threadIdx.x; k < prefix_count; k += blockDim.x) sse[(long)i * prefix_count + k] = 0.0;
}

// G0 = C0^T (K C0~) restricted to training rows (packed lower triangle).
__global__ void initial_gram(InstanceView v, const double* C0, const double* KC0,
                             double* G) {
  __shared__ double scratch[32];
  const int i = blockIdx.x;
  const int f = v.inst_fold[i];
  const int n = v.n, q = v.q;
  const double* c0 = C0 + (long)i * n * q;
  const double* kc = KC0 + (long)i * n * q;
  double* g = G + (long)i * q * (q + 1) / 2;
  for (int c = 0; c < q; ++c)
    for (int d = 0; d <= c; ++d) {
      double s1 = 0.0, s2 = 0.0;
      for (int r = threadIdx.x; r < n; r += blockDim.x)
        if (v.fold_of_row[r] != f + 1) {
          s1 = fma(c0[r + (long)c * n], kc[r + (long)d * n], s1);
          s2 = fma(c0[r + (long)d * n], kc[r + (long)c * n], s2);
        }
      s1 = block_sum(s1, scratch);
      s2 = block_sum(s2, scratch);
      if (threadIdx.x == 0) g[c * (c + 1) / 2 + d] = 0.5 * (s1 + s2);
    }
}

// zs = z / sqrt(lambda) for the dominant eigenpair of the instance's q x q
// Gram (packed lower triangle), sign fixed so the largest |z| entry is
// positive. A, E: 2 q^2 doubles of shared memory.
__device__ void dominant_z(const InstanceView& v, int i, const double* G, int* flag,
                           double* A, double* E, double* zs) {
  const int q = v.q;
  const double* g = G + (long)i * q * (q + 1) / 2;
  for (int c = threadIdx.x; c < q; c += blockDim.x)
    for (int d = 0; d <= c; ++d) {
      A[c + d * q] = g[c * (c + 1) / 2 + d];
      A[d + c * q] = g[c * (c + 1) / 2 + d];
    }
  __syncthreads();
  jacobi_eigen(A, E, q);
  __syncthreads();
  if (threadIdx.x == 0) {
    int best = 0;
    for (int k = 1; k < q; ++k)
      if (A[k + k * q] > A[best + best * q]) best = k;
    const double lam = A[best + best * q];
    const bool ok = lam > 0.0 && isfinite(lam);
    if (!ok) flag_error(flag, 1);
    int arg = 0;
    for (int k = 1; k < q; ++k)
      if (fabs(E[k + best * q]) > fabs(E[arg + best * q])) arg = k;
    const double sgn = E[arg + best * q] < 0.0 ? -1.0 : 1.0;
    const double inv = ok ? 1.0 / sqrt(lam) : 0.0;
    for (int k = 0; k < q; ++k) zs[k] = sgn * E[k + best * q] * inv;
  }
  __syncthreads();
}

// Dominant direction of instance i: u = C z / sqrt(lambda) (zero on held-out
// rows, re-centred over the training rows), written to column i of U. When
// KC0 is given (first component, C = C0) the product K u is formed directly
// as (K C0) z / sqrt(lambda) into column i of Y1, replacing one GEMM.
__device__ void direction_body(const InstanceView& v, int i, const double* G,
                               const double* C, double* U, const double* KC0,
                               double* Y1, int* flag, double* A, double* E,
                               double* zs, double* scratch) {
  const int f = v.inst_fold[i];
  const int n = v.n, q = v.q;
  dominant_z(v, i, G, flag, A, E, zs);
  const double* c = C + (long)i * n * q;
  double* u = U + (long)i * n;
  double s = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    double val = 0.0;
    for (int k = 0; k < q; ++k) val = fma(c[r + (long)k * n], zs[k], val);
    u[r] = val;
    s += val;
  }
  if (v.center) {
    const double mu = block_sum(s, scratch) / v.ntrain[f];
    for (int r = threadIdx.x; r < n; r += blockDim.x)
      if (v.fold_of_row[r] != f + 1) u[r] -= mu;
  }
  if (KC0) {
    const double* kc = KC0 + (long)i * n * q;
    double* y = Y1 + (long)i * n;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      double val = 0.0;
      for (int k = 0; k < q; ++k) val = fma(kc[r + (long)k * n], zs[k], val);
      y[r] = val;
    }
  }
}

__global__ void direction_batched(InstanceView v, const double* G,
                                  const double* C, double* U,
                                  const double* KC0, double* Y1, int* flag) {
  extern __shared__ double sm[];
  __shared__ double scratch[32];
  __shared__ double zs[kBatchMaxResponses];
  direction_body(v, blockIdx.x, G, C, U, KC0, Y1, flag, sm, sm + v.q * v.q, zs, scratch);
}

// Scores from Y1 = K U: centre over training rows, normalise, emit the
// masked training scores t~ (in place of U), q = C0^T t, and advance the
// held-out predictions / SSE for this prefix.
__global__ void scores_batched(InstanceView v, const double* Y1, double* Tm,
                               const double* C0, const double* ymean,
                               double* yhat, int yhat_ld, int a,
                               const int* prefix_slot, int prefix_count,
                               double* sse, double* qbuf, int* flag) {
  __shared__ double scratch[32];
  __shared__ double qs[kBatchMaxResponses];
  const int i = blockIdx.x;
  const int f = v.inst_fold[i], b = v.inst_perm[i];
  const int n = v.n, q = v.q;
  const double* y = Y1 + (long)i * n;
  double* t = Tm + (long)i * n;
  double s = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x)
    if (v.fold_of_row[r] != f + 1) s += y[r];
  const double mu = v.center ? block_sum(s, scratch) / v.ntrain[f] : 0.0;
  double ss = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x)
    if (v.fold_of_row[r] != f + 1) {
      const double tv = y[r] - mu;
      ss = fma(tv, tv, ss);
    }
  ss = block_sum(ss, scratch);
  const double tn = sqrt(ss);
  const bool ok = tn > 0.0 && isfinite(tn);
  if (!ok && threadIdx.x == 0) flag_error(flag, 1);
  const double inv = ok ? 1.0 / tn : 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x)
    t[r] = (v.fold_of_row[r] != f + 1) ? (y[r] - mu) * inv : 0.0;
  __syncthreads();
  const double* c0 = C0 + (long)i * n * q;
  for (int c = 0; c < q; ++c) {
    double acc = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) acc = fma(c0[r + (long)c * n], t[r], acc);
    acc = block_sum(acc, scratch);
    if (threadIdx.x == 0) {
      qs[c] = acc;
      if (qbuf) qbuf[(long)i * q + c] = acc;
    }
  }
  __syncthreads();
  // held-out scores and predictions
  const int* te = v.test_rows + v.test_off[f];
  const int nte = v.test_off[f + 1] - v.test_off[f];
  double* yh = yhat + (long)i * yhat_ld * q;
  const int slot = prefix_slot[a];
  double err = 0.0;
  for (int k = threadIdx.x; k < nte; k += blockDim.x) {
    const int r = te[k];
    const double tt = (y[r] - mu) * inv;
    for (int c = 0; c < q; ++c)
      yh[k + (long)c * yhat_ld] = fma(tt, qs[c], yh[k + (long)c * yhat_ld]);
    if (slot >= 0) err += heldout_term(v, i, b, r, ymean, yh + k, yhat_ld);
  }
  if (slot >= 0) {
    err = block_sum(err, scratch);
    if (threadIdx.x == 0) sse[(long)i * prefix_count + slot] = err;
  }
}

// Deflation from Y2 = K t~ and the next direction, per instance:
//   Kt = P_F Y2_F ; h = KW^T t ; w = t - W h ; Kw = Kt - KW h ;
//   v = sqrt(w^T Kw) ; row = Kw^T C / v ; C -= (w / v) row ; G -= row row^T ;
//   u = C z / sqrt(lambda) for the dominant eigenpair of G (next direction).
// W and KW hold the columns unnormalised, with the scale 1/v of column k in
// wscale[k] (applied where the columns are read), so no pass rewrites them;
// Kw^T C is accumulated in the same sweep that forms w and Kw, and the C
// update shares its sweep with u = C z. Dynamic shared memory:
// 2 q^2 + 2 kmax + q doubles. QMAX >= q bounds the per-thread Kw^T C sums.
template <int QMAX>
__global__ void deflate_batched(InstanceView v, const double* Y2,
                                double* Tm, double* W, double* KW, double* wscale,
                                double* C, double* G, int a, int* flag) {
  extern __shared__ double sm[];
  __shared__ double scratch[32];
  __shared__ double rowpart[(BT / 32) * kBatchMaxResponses];
  __shared__ double zs[kBatchMaxResponses];
  const int i = blockIdx.x;
  const int f = v.inst_fold[i];
  const int n = v.n, q = v.q, kmax = v.kmax;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  double* A = sm;
  double* E = A + q * q;
  double* h = E + q * q;      // h_k * wscale_k (kmax)
  double* hsc = h + kmax;     // scratch for the warp-per-column dots (kmax)
  double* row = hsc + kmax;   // q
  const double* y = Y2 + (long)i * n;
  double* t = Tm + (long)i * n;
  double* w = W + (long)i * n * kmax;
  double* kw = KW + (long)i * n * kmax;
  const double* ws = wscale + (long)i * kmax;
  double* c = C + (long)i * n * q;
  double s = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x)
    if (v.fold_of_row[r] != f + 1) s += y[r];
  const double mu = v.center ? block_sum(s, scratch) / v.ntrain[f] : 0.0;
  // h = KW^T t (warp per column), times the column scales
  for (int k = warp; k < a; k += warps) {
    double acc = 0.0;
#pragma unroll 4
    for (int r = lane; r < n; r += 32) acc = fma(kw[r + (long)k * n], t[r], acc);
    acc = warp_sum(acc);
    if (lane == 0) hsc[k] = acc;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < a; k += blockDim.x) h[k] = hsc[k] * ws[k] * ws[k];
  __syncthreads();
  // w = t - W h, Kw = (Y2 - mu) - KW h (training rows), stored unscaled;
  // w^T Kw and Kw^T C in the same sweep
  double* wa = w + (long)a * n;
  double* kwa = kw + (long)a * n;
  double vv = 0.0;
  double rc[QMAX];
#pragma unroll
  for (int cc = 0; cc < QMAX; ++cc) rc[cc] = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    double wr = 0.0, kr = 0.0;
    if (v.fold_of_row[r] != f + 1) {
      wr = t[r];
      kr = y[r] - mu;
#pragma unroll 4
      for (int k = 0; k < a; ++k) {
        wr = fma(-w[r + (long)k * n], h[k], wr);
        kr = fma(-kw[r + (long)k * n], h[k], kr);
      }
      vv = fma(wr, kr, vv);
#pragma unroll
      for (int cc = 0; cc < QMAX; ++cc)
        if (cc < q) rc[cc] = fma(kr, c[r + (long)cc * n], rc[cc]);
    }
    wa[r] = wr;
    kwa[r] = kr;
  }
  vv = block_sum(vv, scratch);
  const double vn = sqrt(vv);
  const bool ok = vn > 0.0 && isfinite(vn);
  if (!ok && threadIdx.x == 0) flag_error(flag, 1);
  const double inv = ok ? 1.0 / vn : 0.0;
#pragma unroll
  for (int cc = 0; cc < QMAX; ++cc)
    if (cc < q) {
      const double part = warp_sum(rc[cc]);
      if (lane == 0) rowpart[warp * q + cc] = part;
    }
  __syncthreads();
  if (threadIdx.x < q) {
    double tot = 0.0;
    for (int ww = 0; ww < warps; ++ww) tot += rowpart[ww * q + threadIdx.x];
    row[threadIdx.x] = tot * inv;
  }
  if (threadIdx.x == 0) wscale[(long)i * kmax + a] = inv;
  __syncthreads();
  if (threadIdx.x == 0) {
    double* g = G + (long)i * q * (q + 1) / 2;
    for (int cc = 0; cc < q; ++cc)
      for (int d = 0; d <= cc; ++d) g[cc * (cc + 1) / 2 + d] -= row[cc] * row[d];
  }
  __syncthreads();
  dominant_z(v, i, G, flag, A, E, zs);
  // C -= (w / v) row^T and the next direction u = C z (over t~)
  double su = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const double wr = wa[r] * inv;
    double u = 0.0;
    for (int cc = 0; cc < q; ++cc) {
      const double cv = fma(-wr, row[cc], c[r + (long)cc * n]);
      c[r + (long)cc * n] = cv;
      u = fma(cv, zs[cc], u);
    }
    t[r] = u;
    su += u;
  }
  if (v.center) {
    const double mu_u = block_sum(su, scratch) / v.ntrain[f];
    for (int r = threadIdx.x; r < n; r += blockDim.x)
      if (v.fold_of_row[r] != f + 1) t[r] -= mu_u;
  }
}

// ---------------------------------------------------------------------------
// Register-resident form of the score step (n <= RPT * BT): each thread
// keeps its rows r = threadIdx.x + j BT (j < RPT) of the instance's score
// vector in registers across the phases, so that Y1 is read from HBM once.
// Same arithmetic as scores_batched.

// Totals of per-warp partials: part[w * count + c] -> out[c] (c < count).
__device__ __forceinline__ void warp_partials_total(const double* part, int count, double* out) {
  __syncthreads();
  for (int c = threadIdx.x; c < count; c += blockDim.x) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += part[w * count + c];
    out[c] = tot;
  }
  __syncthreads();
}

template <int RPT>
__global__ void __launch_bounds__(BT)
    scores_rows(InstanceView v, const double* Y1, double* Tm, const double* C0,
                const double* ymean, double* yhat, int yhat_ld, int a,
                const int* prefix_slot, int prefix_count, double* sse, int* flag) {
  __shared__ double scratch[32];
  __shared__ double part[(BT / 32) * kBatchMaxResponses];
  __shared__ double qs[kBatchMaxResponses];
  const int i = blockIdx.x;
  const int f = v.inst_fold[i], b = v.inst_perm[i];
  const int n = v.n, q = v.q;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double* y = Y1 + (long)i * n;
  double* t = Tm + (long)i * n;
  double val[RPT];
  unsigned train = 0u;
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < RPT; ++j) {
    const int r = threadIdx.x + j * BT;
    val[j] = 0.0;
    if (r < n && v.fold_of_row[r] != f + 1) {
      val[j] = y[r];
      train |= 1u << j;
      s += val[j];
    }
  }
  const double mu = v.center ? block_sum(s, scratch) / v.ntrain[f] : 0.0;
  double ss = 0.0;
#pragma unroll
  for (int j = 0; j < RPT; ++j)
    if (train >> j & 1u) {
      const double tv = val[j] - mu;
      ss = fma(tv, tv, ss);
    }
  ss = block_sum(ss, scratch);
  const double tn = sqrt(ss);
  const bool ok = tn > 0.0 && isfinite(tn);
  if (!ok && threadIdx.x == 0) flag_error(flag, 1);
  const double inv = ok ? 1.0 / tn : 0.0;
#pragma unroll
  for (int j = 0; j < RPT; ++j) {
    const int r = threadIdx.x + j * BT;
    val[j] = (train >> j & 1u) ? (val[j] - mu) * inv : 0.0;
    if (r < n) t[r] = val[j];
  }
  const double* c0 = C0 + (long)i * n * q;
  for (int c = 0; c < q; ++c) {
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
      const int r = threadIdx.x + j * BT;
      if (r < n) acc = fma(c0[r + (long)c * n], val[j], acc);
    }
    acc = warp_sum(acc);
    if (lane == 0) part[warp * q + c] = acc;
  }
  warp_partials_total(part, q, qs);
  // held-out scores and predictions
  const int* te = v.test_rows + v.test_off[f];
  const int nte = v.test_off[f + 1] - v.test_off[f];
  double* yh = yhat + (long)i * yhat_ld * q;
  const int slot = prefix_slot[a];
  double err = 0.0;
  for (int k = threadIdx.x; k < nte; k += blockDim.x) {
    const int r = te[k];
    const double tt = (y[r] - mu) * inv;
    for (int c = 0; c < q; ++c)
      yh[k + (long)c * yhat_ld] = fma(tt, qs[c], yh[k + (long)c * yhat_ld]);
    if (slot >= 0) err += heldout_term(v, i, b, r, ymean, yh + k, yhat_ld);
  }
  if (slot >= 0) {
    err = block_sum(err, scratch);
    if (threadIdx.x == 0) sse[(long)i * prefix_count + slot] = err;
  }
}

template <class T>
__global__ void to_f64(const T* __restrict__ in, long count, double* out) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < count;
       k += (long)gridDim.x * blockDim.x)
    out[k] = as_f64(in[k]);
}

// Column sums / sums of squares of the held-out rows of one fold.
template <class T>
__global__ void heldout_moments(const T* __restrict__ X, int n, int p,
                                const int* __restrict__ rows, int count,
                                double* sum, double* sumsq) {
  __shared__ double scratch[32];
  for (int j = blockIdx.x; j < p; j += gridDim.x) {
    double s = 0.0, ss = 0.0;
    for (int k = threadIdx.x; k < count; k += blockDim.x) {
      const double x = as_f64(X[rows[k] + (long)j * n]);
      s += x;
      ss = fma(x, x, ss);
    }
    s = block_sum(s, scratch);
    ss = block_sum(ss, scratch);
    if (threadIdx.x == 0) {
      sum[j] = s;
      sumsq[j] = ss;
    }
  }
}

// kscale[j] = 1 / sd_train[j]^2 (autoscaling; sd with n-1, 1 when degenerate)
__global__ void fold_kscale(const double* tsum, const double* tsumsq,
                            const double* hsum, const double* hsumsq, int p,
                            int ntrain, double* kscale) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x) {
    const double s = tsum[j] - hsum[j], ss = tsumsq[j] - hsumsq[j];
    const double mu = s / ntrain;
    double sd = sqrt(fmax(0.0, ss - ntrain * mu * mu) / (double)max(ntrain - 1, 1));
    if (!isfinite(sd) || sd <= 0.0) sd = 1.0;
    kscale[j] = 1.0 / (sd * sd);
  }
}

// out = X * sqrt(kscale) column-wise (kscale = 1 / sd^2 under autoscaling)
template <class T>
__global__ void scale_columns_f64(const T* __restrict__ X, int n, int p,
                                  const double* __restrict__ kscale,
                                  double* __restrict__ out) {
  const long total = (long)n * p;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total;
       k += (long)gridDim.x * blockDim.x) {
    const double v = as_f64(X[k]);
    out[k] = kscale ? v * sqrt(kscale[k / n]) : v;
  }
}

__global__ void response_moments(const double* __restrict__ Y, int n, double* out) {
  __shared__ double scratch[32];
  double s = 0.0, ss = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = Y[i + (long)blockIdx.x * n];
    s += v;
    ss = fma(v, v, ss);
  }
  s = block_sum(s, scratch);
  ss = block_sum(ss, scratch);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = s;
    out[2 * blockIdx.x + 1] = ss;
  }
}

}  // namespace

int& batch_lanes() {
  static int lanes = 3;
  return lanes;
}

namespace {

// Rows per thread of the register-resident score kernel for n rows (0: too
// many, use the general kernel).
int rows_per_thread(int n) {
  const int need = (n + BT - 1) / BT;
  for (int r : {8, 16, 20, 24, 32})
    if (need <= r) return r;
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
template <class T>
void BatchedCv<T>::form_gram(const double* kscale, cudaStream_t s) {
  gram.reserve((size_t)n * n, s);
  if (digits > 0) {
    // int8 digits of the rows of X D^1/2, the symmetric product on the int8
    // tensor cores (lower tiles + mirror), then the digits of K's rows for
    // every later product with K
    ozaki_split_colmajor<T>(X, n, p, n, kscale, digits, x_split, flag.get(), s);
    ozaki_gemm(x_split, x_split, gram.get(), n, true, flag.get(), s);
    ozaki_split_rows(gram.get(), n, n, n, digits, gram_split, flag.get(), s);
    return;
  }
  // FP64 copy of X with the scaling folded in (X D^1/2), then the symmetric
  // product on the FP64 tensor-core path (lower tiles + mirror).
  x64.reserve((size_t)n * p, s);
  const long total = (long)n * p;
  scale_columns_f64<T><<<(unsigned)std::min<long>((total + 255) / 256, 16L * num_sms()), 256, 0, s>>>(
      X, n, p, kscale, x64.get());
  count_launch();
  FPLS_LAUNCH("scale_columns_f64");
  GemmArgs g;
  g.M = n;
  g.N = n;
  g.K = p;
  g.A = x64.get();
  g.lda = n;
  g.B = x64.get();
  g.ldb = n;
  g.trans_b = true;
  g.C = gram.get();
  g.ldc = n;
  g.lower = gemm_mma_supported(g);
  gemm_f64(g, s);
}

template <class T>
void BatchedCv<T>::gram_product(const double* rhs, int cols, double* out,
                                OzakiOperand& rhs_split, cudaStream_t s) {
  if (digits > 0) {
    // K is symmetric: its rows are its columns (contiguous, ld n)
    ozaki_split_rows(rhs, n, cols, n, digits, rhs_split, flag.get(), s);
    ozaki_gemm(gram_split, rhs_split, out, n, false, flag.get(), s);
    return;
  }
  GemmArgs g;
  g.M = n;
  g.N = cols;
  g.K = n;
  g.A = gram.get();
  g.lda = n;
  g.B = rhs;
  g.ldb = n;
  g.C = out;
  g.ldc = n;
  gemm_f64(g, s);
}

// The instances of a group run in lanes of their own CUDA stream, enqueued
// component by component in turn, so that the memory-bound score and
// deflation kernels of one lane overlap the tensor-core products of the
// other. Lanes share the Gram and its digits (read only).
template <class T>
void BatchedCv<T>::run_group(const std::vector<int>& inst_fold,
                             const std::vector<int>& inst_perm,
                             cudaStream_t s) {
  const int I = (int)inst_fold.size();
  if (I == 0) return;
  const int q = this->q, kmax = this->kmax;
  const size_t nq = (size_t)n * q;
  const int nlanes = std::max(1, std::min(batch_lanes(), I / kLaneMinInstances));
  struct OwnStream {
    cudaStream_t st = nullptr;
    bool own = false;
    ~OwnStream() {
      if (own) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
    }
  };
  struct Lane {
    OwnStream hold;  // destroyed last: every array below is freed on it first
    int off = 0, cnt = 0;
    InstanceView v;
    DeviceArray<int> d_if, d_ip;
    DeviceArray<double> C0, C, G, ym, sst, sse, yhat, Wb, KWb, Ws, U, Y1, KC0;
    OzakiOperand rhs;
  };
  std::vector<Lane> lanes(nlanes);
  cudaEvent_t ready = nullptr;
  FPLS_CHECK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  struct EventGuard {
    cudaEvent_t e;
    ~EventGuard() { cudaEventDestroy(e); }
  } ready_guard{ready};
  FPLS_CHECK(cudaEventRecord(ready, s));

  const size_t smem_dir = 2 * (size_t)q * q * sizeof(double);
  const int rpt = rows_per_thread(n);
  for (int l = 0; l < nlanes; ++l) {
    Lane& L = lanes[l];
    L.off = l * (I / nlanes);
    L.cnt = l + 1 == nlanes ? I - L.off : I / nlanes;
    if (nlanes == 1) {
      L.hold.st = s;
    } else {
      FPLS_CHECK(cudaStreamCreateWithFlags(&L.hold.st, cudaStreamNonBlocking));
      L.hold.own = true;
      FPLS_CHECK(cudaStreamWaitEvent(L.hold.st, ready, 0));
    }
    const cudaStream_t st = L.hold.st;
    const int c = L.cnt;
    L.d_if.allocate(c, st);
    L.d_ip.allocate(c, st);
    FPLS_CHECK(cudaMemcpyAsync(L.d_if.get(), inst_fold.data() + L.off, sizeof(int) * c,
                               cudaMemcpyHostToDevice, st));
    FPLS_CHECK(cudaMemcpyAsync(L.d_ip.get(), inst_perm.data() + L.off, sizeof(int) * c,
                               cudaMemcpyHostToDevice, st));
    InstanceView& v = L.v;
    v.n = n;
    v.q = q;
    v.kmax = kmax;
    v.B = 0;
    v.center = center ? 1 : 0;
    v.fold_of_row = d_fold.get();
    v.inst_fold = L.d_if.get();
    v.inst_perm = L.d_ip.get();
    v.perms = perms;
    v.ntrain = d_ntrain.get();
    v.test_rows = d_test_rows.get();
    v.test_off = d_test_off.get();
    v.Y = Y64.get();
    v.labels = class_labels;
    L.C0.allocate(nq * c, st);
    L.C.allocate(nq * c, st);
    L.G.allocate((size_t)c * q * (q + 1) / 2, st);
    L.ym.allocate((size_t)c * q, st);
    L.sst.allocate(c, st);
    L.sse.allocate((size_t)c * prefix_count, st);
    L.yhat.allocate((size_t)c * max_test * q, st);
    L.Wb.allocate((size_t)c * n * kmax, st);
    L.KWb.allocate((size_t)c * n * kmax, st);
    L.Ws.allocate((size_t)c * kmax, st);
    L.U.allocate((size_t)n * c, st);
    L.Y1.allocate((size_t)n * c, st);
    L.KC0.allocate(nq * c, st);

    init_instances<<<c, BT, 0, st>>>(v, L.C0.get(), L.C.get(), L.ym.get(), L.sst.get(),
                                     L.yhat.get(), max_test, L.sse.get(), prefix_count);
    count_launch();
    FPLS_LAUNCH("init_instances");
    // G0 = C0^T K C0 via one product over all instances' C0 columns
    gram_product(L.C0.get(), q * c, L.KC0.get(), L.rhs, st);
    initial_gram<<<c, BT, 0, st>>>(v, L.C0.get(), L.KC0.get(), L.G.get());
    count_launch();
    FPLS_LAUNCH("initial_gram");
    // first direction; K u comes from K C0 (no GEMM)
    direction_batched<<<c, BT, smem_dir, st>>>(v, L.G.get(), L.C.get(), L.U.get(), L.KC0.get(),
                                               L.Y1.get(), flag.get());
    count_launch();
    FPLS_LAUNCH("direction_batched");
    L.KC0.release();
  }
  for (int a = 0; a < kmax; ++a) {
    for (Lane& L : lanes) {
      const cudaStream_t st = L.hold.st;
      const int c = L.cnt;
      const InstanceView& v = L.v;
      if (a > 0) gram_product(L.U.get(), c, L.Y1.get(), L.rhs, st);  // Y1 = K u
      switch (rpt) {
#define FPLS_SCORES(R)                                                                         \
  case R:                                                                                      \
    scores_rows<R><<<c, BT, 0, st>>>(v, L.Y1.get(), L.U.get(), L.C0.get(), L.ym.get(),         \
                                     L.yhat.get(), max_test, a, d_slot.get(), prefix_count,    \
                                     L.sse.get(), flag.get());                                 \
    break;
        FPLS_SCORES(8)
        FPLS_SCORES(16)
        FPLS_SCORES(20)
        FPLS_SCORES(24)
        FPLS_SCORES(32)
#undef FPLS_SCORES
        default:
          scores_batched<<<c, BT, 0, st>>>(v, L.Y1.get(), L.U.get(), L.C0.get(), L.ym.get(),
                                           L.yhat.get(), max_test, a, d_slot.get(),
                                           prefix_count, L.sse.get(), nullptr, flag.get());
      }
      count_launch();
      FPLS_LAUNCH("scores_batched");
      if (a + 1 == kmax) continue;  // the last deflation is never used
      // Y1 = K t~ (U holds the masked training scores)
      gram_product(L.U.get(), c, L.Y1.get(), L.rhs, st);
      const size_t smem_defl = (2 * (size_t)q * q + 2 * (size_t)kmax + q) * sizeof(double);
      if (q <= 4)
        deflate_batched<4><<<c, DEFL_BT, smem_defl, st>>>(v, L.Y1.get(), L.U.get(), L.Wb.get(),
                                                     L.KWb.get(), L.Ws.get(), L.C.get(),
                                                     L.G.get(), a, flag.get());
      else
        deflate_batched<kBatchMaxResponses><<<c, DEFL_BT, smem_defl, st>>>(
            v, L.Y1.get(), L.U.get(), L.Wb.get(), L.KWb.get(), L.Ws.get(), L.C.get(), L.G.get(),
            a, flag.get());
      count_launch();
      FPLS_LAUNCH("deflate_batched");
    }
  }
  // collect per-instance sums
  std::vector<double> h_sse((size_t)I * prefix_count), h_sst(I);
  for (Lane& L : lanes) {
    FPLS_CHECK(cudaMemcpyAsync(h_sse.data() + (size_t)L.off * prefix_count, L.sse.get(),
                               sizeof(double) * L.cnt * prefix_count, cudaMemcpyDeviceToHost,
                               L.hold.st));
    FPLS_CHECK(cudaMemcpyAsync(h_sst.data() + L.off, L.sst.get(), sizeof(double) * L.cnt,
                               cudaMemcpyDeviceToHost, L.hold.st));
  }
  for (Lane& L : lanes) {
    FPLS_CHECK(cudaStreamSynchronize(L.hold.st));
    if (L.hold.own) {
      // later work on the caller's stream follows this lane
      cudaEvent_t done = nullptr;
      FPLS_CHECK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
      FPLS_CHECK(cudaEventRecord(done, L.hold.st));
      FPLS_CHECK(cudaStreamWaitEvent(s, done, 0));
      cudaEventDestroy(done);
    }
  }
  for (int k = 0; k < I; ++k) {
    const int f = inst_fold[k];
    const int b = inst_perm[k] + 1;  // 0 = observed responses
    for (int j = 0; j < prefix_count; ++j)
      inst_sse[((size_t)b * folds + f) * prefix_count + j] = h_sse[(size_t)k * prefix_count + j];
    inst_sst[(size_t)b * folds + f] = h_sst[k];
  }
}

template <class T>
void BatchedCv<T>::run(const T* X_, int n_, int p_, const T* Y_, int q_,
                       const int* folds_host, const int* perms_dev,
                       int perm_count, const int* prefixes_, int count,
                       int scaling_, cudaStream_t s) {
  X = X_;
  n = n_;
  p = p_;
  q = q_;
  perms = perms_dev;
  P = perm_count;
  prefix_count = count;
  scaling = scaling_;
  center = scaling != 3;
  digits = ozaki_slices();
  require(q >= 1 && q <= kBatchMaxResponses, "batched CV supports 1..32 responses");
  kmax = 0;
  for (int j = 0; j < count; ++j) {
    if (prefixes_[j] <= kmax) throw std::invalid_argument("CUDA CV component path must be strictly increasing");
    kmax = prefixes_[j];
  }
  folds = 0;
  for (int i = 0; i < n; ++i) {
    if (folds_host[i] < 1) throw std::invalid_argument("invalid CUDA CV fold");
    folds = std::max(folds, folds_host[i]);
  }
  std::vector<std::vector<int>> test(folds);
  for (int i = 0; i < n; ++i) test[folds_host[i] - 1].push_back(i);
  std::vector<int> ntrain(folds), test_rows, test_off(folds + 1, 0);
  max_test = 1;
  status.assign(folds, 0);
  for (int f = 0; f < folds; ++f) {
    ntrain[f] = n - (int)test[f].size();
    max_test = std::max(max_test, (int)test[f].size());
    test_off[f + 1] = test_off[f] + (int)test[f].size();
    test_rows.insert(test_rows.end(), test[f].begin(), test[f].end());
    if (!test[f].empty() && kmax > std::min(ntrain[f] - 1, p))
      throw std::invalid_argument("CUDA CV component count exceeds a fold rank");
    status[f] = test[f].empty() ? 2 : 1;
  }
  heldout.assign(folds, 0);
  for (int f = 0; f < folds; ++f) heldout[f] = (int)test[f].size();
  std::vector<int> slot(kmax + 1, -1);
  for (int j = 0; j < count; ++j) slot[prefixes_[j] - 1] = j;
  d_fold.allocate(n, s);
  d_ntrain.allocate(folds, s);
  d_test_rows.allocate(std::max(1, (int)test_rows.size()), s);
  d_test_off.allocate(folds + 1, s);
  d_slot.allocate(kmax + 1, s);
  flag.allocate(1, s);
  FPLS_CHECK(cudaMemsetAsync(flag.get(), 0, sizeof(int), s));
  FPLS_CHECK(cudaMemcpyAsync(d_fold.get(), folds_host, sizeof(int) * n, cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(d_ntrain.get(), ntrain.data(), sizeof(int) * folds, cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(d_test_rows.get(), test_rows.data(), sizeof(int) * test_rows.size(), cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(d_test_off.get(), test_off.data(), sizeof(int) * (folds + 1), cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(d_slot.get(), slot.data(), sizeof(int) * (kmax + 1), cudaMemcpyHostToDevice, s));
  Y64.allocate((size_t)n * q, s);
  to_f64<T><<<std::min<unsigned>(ceil_div((size_t)n * q, 256), 4 * num_sms()), 256, 0, s>>>(Y_, (long)n * q, Y64.get());
  count_launch();
  FPLS_LAUNCH("to_f64");
  {
    DeviceArray<double> cs((size_t)2 * q, s);
    response_moments<<<q, 256, 0, s>>>(Y64.get(), n, cs.get());
    count_launch();
    FPLS_LAUNCH("response_moments");
    std::vector<double> h(2 * q);
    FPLS_CHECK(cudaMemcpyAsync(h.data(), cs.get(), sizeof(double) * 2 * q, cudaMemcpyDeviceToHost, s));
    FPLS_CHECK(cudaStreamSynchronize(s));
    total_ss = 0.0L;
    for (int c = 0; c < q; ++c)
      total_ss += (long double)h[2 * c + 1] - (long double)h[2 * c] * h[2 * c] / n;
  }

  const int B = P + 1;
  inst_sse.assign((size_t)B * folds * count, 0.0);
  inst_sst.assign((size_t)B * folds, 0.0);

  // instances per group bounded by device memory (per instance: C0, C, W,
  // KW, U, Y1 and held-out predictions)
  size_t free_b = 0, total_b = 0;
  FPLS_CHECK(cudaMemGetInfo(&free_b, &total_b));
  const size_t per_inst = sizeof(double) * ((size_t)n * (2 * q + 2 * kmax + 2 + q) + (size_t)max_test * q + 64);
  const size_t budget = free_b > ((size_t)n * n * 8 + (1ull << 30)) ? free_b - (size_t)n * n * 8 - (1ull << 30) : per_inst;
  const int max_group = std::max(1, (int)std::min<size_t>(budget * 7 / 10 / per_inst, 1 << 20));

  auto run_instances = [&](const std::vector<int>& fl, const std::vector<int>& pl) {
    for (size_t off = 0; off < fl.size(); off += max_group) {
      const size_t cnt = std::min(fl.size() - off, (size_t)max_group);
      std::vector<int> a(fl.begin() + off, fl.begin() + off + cnt);
      std::vector<int> b(pl.begin() + off, pl.begin() + off + cnt);
      run_group(a, b, s);
    }
  };

  if (scaling == 2) {
    // autoscaling: one Gram per fold with that fold's training-row scales
    DeviceArray<double> mom((size_t)2 * p, s), hmom((size_t)2 * p, s), ks(p, s);
    DeviceArray<double> scratch;
    column_moments<T>(X, n, p, n, nullptr, 0, mom.get(), mom.get() + p, nullptr, scratch, s);
    for (int f = 0; f < folds; ++f) {
      if (test[f].empty()) continue;
      heldout_moments<T><<<std::min(p, 8 * num_sms()), 256, 0, s>>>(
          X, n, p, d_test_rows.get() + test_off[f], (int)test[f].size(), hmom.get(), hmom.get() + p);
      fold_kscale<<<std::min<unsigned>(ceil_div(p, 256), 4 * num_sms()), 256, 0, s>>>(
          mom.get(), mom.get() + p, hmom.get(), hmom.get() + p, p, ntrain[f], ks.get());
      count_launch(2);
      FPLS_LAUNCH("fold scales");
      form_gram(ks.get(), s);
      std::vector<int> fl, pl;
      for (int b = 0; b < B; ++b) {
        fl.push_back(f);
        pl.push_back(b - 1);
      }
      run_instances(fl, pl);
    }
  } else {
    form_gram(nullptr, s);
    std::vector<int> fl, pl;
    for (int b = 0; b < B; ++b)
      for (int f = 0; f < folds; ++f) {
        if (test[f].empty()) continue;
        fl.push_back(f);
        pl.push_back(b - 1);
      }
    run_instances(fl, pl);
  }
  int bad = 0;
  FPLS_CHECK(cudaMemcpyAsync(&bad, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaStreamSynchronize(s));
  if (bad) throw std::runtime_error("resident SIMPLS failed: invalid labels, decomposition or component norm");
}

template <class T>
void BatchedCv<T>::metrics(int metric, double* metric_out, double* q2,
                           double* rmsd, double* r2) const {
  const int B = P + 1;
  const double nan = std::numeric_limits<double>::quiet_NaN();
  for (int b = 0; b < B; ++b) {
    for (int j = 0; j < prefix_count; ++j) {
      double sse = 0.0, fss = 0.0, cnt = 0.0;
      for (int f = 0; f < folds; ++f) {
        if (status[f] != 1) continue;
        sse += inst_sse[((size_t)b * folds + f) * prefix_count + j];
        fss += inst_sst[(size_t)b * folds + f];
      }
      cnt = (double)n * q;
      const double rm = cnt > 0 ? std::sqrt(sse / cnt) : nan;
      const double qq = fss > 0 ? 1.0 - sse / fss : nan;
      const double rr = total_ss > 0.0L ? 1.0 - sse / (double)total_ss : nan;
      const size_t o = (size_t)b * prefix_count + j;
      if (q2) q2[o] = qq;
      if (rmsd) rmsd[o] = rm;
      if (r2) r2[o] = rr;
      if (metric_out) metric_out[o] = metric == 4 ? rm : metric == 3 ? qq : rr;
    }
  }
}

template <class T>
void BatchedCv<T>::accuracy(double* out) const {
  const int B = P + 1;
  for (int b = 0; b < B; ++b)
    for (int j = 0; j < prefix_count; ++j) {
      double hits = 0.0, rows = 0.0;
      for (int f = 0; f < folds; ++f) {
        if (status[f] != 1) continue;
        hits += inst_sse[((size_t)b * folds + f) * prefix_count + j];
        rows += heldout[f];
      }
      out[(size_t)b * prefix_count + j] =
          rows > 0 ? hits / rows : std::numeric_limits<double>::quiet_NaN();
    }
}

template struct BatchedCv<float>;
template struct BatchedCv<double>;

}  // namespace fpls
