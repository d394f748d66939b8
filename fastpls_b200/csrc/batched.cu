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
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
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
  int* amb;                 // per instance: set to 1 when a held-out argmax
                            // decision fell inside the int8-product margin
                            // (null: FP64 products, no margin)
  double guard;             // relative argmax margin (argmax_guard())
  // LDA head (classification): the training scores (n x kmax per instance,
  // zero on held-out rows) and held-out scores (max_test x kmax) are kept and
  // the head runs after the last component; null for the argmax head
  double* ttr;
  double* tte;
  int max_test;
  // candidate blocks (classification fits with n_train p classes >= 5e8 and
  // 4+ components): per instance the block width (1: a direction per
  // component), the scaled eigenvectors z_j / sqrt(lambda_j) of the block's
  // start Gram (q x q) and its coefficients C at the block start (n x q);
  // null when no instance takes blocks
  const int* blk;
  double* zblk;
  double* cblk;
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
    double bv = 0.0, sv = 0.0;
    bool second = false;
    for (int c = 0; c < q; ++c) {
      const double ym = ymean[(long)i * q + c];
      if (ym > 0.0) {
        const double score = ym + yh[(long)c * ld];
        if (best < 0 || score > bv) {
          if (best >= 0) {
            sv = bv;
            second = true;
          }
          best = c;
          bv = score;
        } else if (!second || score > sv) {
          sv = score;
          second = true;
        }
      }
    }
    if (v.amb && second && !(bv - sv > v.guard * fmax(fabs(bv), fabs(sv))))
      v.amb[i] = 1;
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

// The `count` leading eigenpairs of the instance's q x q Gram, by decreasing
// eigenvalue (ties: lower index first), scaled z_j / sqrt(lambda_j) with the
// largest |z_j| entry positive, into zblk (q x count) of instance i; zs gets
// the first (the candidate block of simpls_fit / direction_kernel).
__device__ void block_z(const InstanceView& v, int i, const double* G, int* flag, int count,
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
    double* zb = v.zblk + (long)i * q * q;
    double inv0 = 0.0;
    for (int j = 0; j < count; ++j) {
      int best = -1;
      for (int k = 0; k < q; ++k)
        if (best < 0 || A[k + k * q] > A[best + best * q]) best = k;
      const double lam = A[best + best * q];
      A[best + best * q] = -INFINITY;  // taken
      const bool ok = lam > 0.0 && isfinite(lam);
      // a later candidate beyond the rank of the Gram takes the leading
      // pair's scale (the direction's scale cancels in the scores)
      if (!ok && j == 0) flag_error(flag, 1);
      int arg = 0;
      for (int k = 1; k < q; ++k)
        if (fabs(E[k + best * q]) > fabs(E[arg + best * q])) arg = k;
      const double sgn = E[arg + best * q] < 0.0 ? -1.0 : 1.0;
      const double inv = ok ? 1.0 / sqrt(lam) : inv0;
      if (j == 0) inv0 = inv;
      for (int k = 0; k < q; ++k) zb[k + (long)j * q] = sgn * E[k + best * q] * inv;
    }
    for (int k = 0; k < q; ++k) zs[k] = zb[k];
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
  const int blk = v.blk ? v.blk[i] : 1;
  if (blk > 1) block_z(v, i, G, flag, blk, A, E, zs);
  else dominant_z(v, i, G, flag, A, E, zs);
  const double* c = C + (long)i * n * q;
  double* cb = blk > 1 ? v.cblk + (long)i * n * q : nullptr;
  double* u = U + (long)i * n;
  double s = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    double val = 0.0;
    for (int k = 0; k < q; ++k) {
      if (cb) cb[r + (long)k * n] = c[r + (long)k * n];
      val = fma(c[r + (long)k * n], zs[k], val);
    }
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
  double* ttr = v.ttr ? v.ttr + ((long)i * v.kmax + a) * n : nullptr;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const double tv = (v.fold_of_row[r] != f + 1) ? (y[r] - mu) * inv : 0.0;
    t[r] = tv;
    if (ttr) ttr[r] = tv;
  }
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
  double* tte = v.tte ? v.tte + ((long)i * v.kmax + a) * v.max_test : nullptr;
  for (int k = threadIdx.x; k < nte; k += blockDim.x) {
    const int r = te[k];
    const double tt = (y[r] - mu) * inv;
    if (tte) {
      tte[k] = tt;  // the LDA head reads the held-out scores after the last component
      continue;
    }
    for (int c = 0; c < q; ++c)
      yh[k + (long)c * yhat_ld] = fma(tt, qs[c], yh[k + (long)c * yhat_ld]);
    if (slot >= 0) err += heldout_term(v, i, b, r, ymean, yh + k, yhat_ld);
  }
  if (slot >= 0 && !tte) {
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
  // next direction: the dominant pair of the deflated Gram, or within a
  // candidate block the block start's next eigenpair applied to the block
  // start's coefficients
  const int blk = v.blk ? v.blk[i] : 1;
  const int nxt = a + 1;
  const bool start = blk > 1 && nxt % blk == 0;
  const bool inside = blk > 1 && !start;
  if (start) {
    block_z(v, i, G, flag, blk, A, E, zs);
  } else if (inside) {
    if (threadIdx.x < q) zs[threadIdx.x] = v.zblk[(long)i * q * q + (long)(nxt % blk) * q + threadIdx.x];
    __syncthreads();
  } else {
    dominant_z(v, i, G, flag, A, E, zs);
  }
  double* cb = blk > 1 ? v.cblk + (long)i * n * q : nullptr;
  // C -= (w / v) row^T and the next direction u = C z (over t~)
  double su = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const double wr = wa[r] * inv;
    double u = 0.0;
    for (int cc = 0; cc < q; ++cc) {
      const double cv = fma(-wr, row[cc], c[r + (long)cc * n]);
      c[r + (long)cc * n] = cv;
      if (start) cb[r + (long)cc * n] = cv;
      u = fma(inside ? cb[r + (long)cc * n] : cv, zs[cc], u);
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
  double* ttr = v.ttr ? v.ttr + ((long)i * v.kmax + a) * n : nullptr;
#pragma unroll
  for (int j = 0; j < RPT; ++j) {
    const int r = threadIdx.x + j * BT;
    val[j] = (train >> j & 1u) ? (val[j] - mu) * inv : 0.0;
    if (r < n) {
      t[r] = val[j];
      if (ttr) ttr[r] = val[j];
    }
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
  double* tte = v.tte ? v.tte + ((long)i * v.kmax + a) * v.max_test : nullptr;
  for (int k = threadIdx.x; k < nte; k += blockDim.x) {
    const int r = te[k];
    const double tt = (y[r] - mu) * inv;
    if (tte) {
      tte[k] = tt;  // the LDA head reads the held-out scores after the last component
      continue;
    }
    for (int c = 0; c < q; ++c)
      yh[k + (long)c * yhat_ld] = fma(tt, qs[c], yh[k + (long)c * yhat_ld]);
    if (slot >= 0) err += heldout_term(v, i, b, r, ymean, yh + k, yhat_ld);
  }
  if (slot >= 0 && !tte) {
    err = block_sum(err, scratch);
    if (threadIdx.x == 0) sse[(long)i * prefix_count + slot] = err;
  }
}

// LDA head of one instance, after its last component (classification with
// the LDA head): training scores T (n x kmax, zero on held-out rows), the
// counts of its active classes (those present in its training rows), the
// score Gram T^T T and the class sums; then per prefix k the pooled
// within-class covariance (T_k^T T_k - sum_c n_c mu_c mu_c^T) / max(1, n - c),
// the first ridge rho * trace / k (rho in 1e-8, 1e-6, 1e-5, 1e-4, 1e-3,
// 1e-2) whose Cholesky factorisation and solves succeed, the linear terms
// Sigma^-1 mu_c and constants -mu_c^T Sigma^-1 mu_c / 2 + log prior_c
// (train_lda_prefixes / finalize_lda_prefixes,
// inst/include/fastpls/core/lda.hpp:86-223), and the held-out argmax over
// the active classes (first wins on ties) against the row's class. The hit
// count of prefix slot j goes to sse[j]. Dynamic shared memory:
// 3 K^2 + 2 q K + q + K doubles (K = kmax <= kLdaMaxComponents).
constexpr int kLdaMaxComponents = 32;
constexpr int LDA_BT = 128;

__global__ void __launch_bounds__(LDA_BT)
    lda_heads(InstanceView v, const int* __restrict__ prefixes, int prefix_count, double* sse,
              int* flag) {
  extern __shared__ double sm[];
  __shared__ int cnt[kBatchMaxResponses];
  __shared__ int active[kBatchMaxResponses];
  __shared__ int nact_s;
  __shared__ double red[32];
  const int i = blockIdx.x;
  const int f = v.inst_fold[i], b = v.inst_perm[i];
  const int n = v.n, q = v.q, K = v.kmax;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  double* gram = sm;               // K x K
  double* sums = gram + K * K;     // q x K (class-major)
  double* cov = sums + q * K;      // K x K
  double* L = cov + K * K;         // K x K
  double* lin = L + K * K;         // q x K (active classes first)
  double* cst = lin + q * K;       // q
  double* rhs = cst + q;           // K
  const double* T = v.ttr + (long)i * K * n;
  const double* Tt = v.tte + (long)i * K * v.max_test;
  for (int c = threadIdx.x; c < q; c += blockDim.x) cnt[c] = 0;
  __syncthreads();
  for (int r = threadIdx.x; r < n; r += blockDim.x)
    if (v.fold_of_row[r] != f + 1) atomicAdd(&cnt[v.labels[src_row(v, b, r)]], 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    int na = 0;
    for (int c = 0; c < q; ++c)
      if (cnt[c] > 0) active[na++] = c;
    nact_s = na;
  }
  // Gram of the training scores (held-out rows hold zeros), lower triangle
  const int pairs = K * (K + 1) / 2;
  for (int k = warp; k < pairs; k += warps) {
    int c1 = (int)((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
    while (c1 * (c1 + 1) / 2 > k) --c1;
    while ((c1 + 1) * (c1 + 2) / 2 <= k) ++c1;
    const int c2 = k - c1 * (c1 + 1) / 2;
    double acc = 0.0;
    for (int r = lane; r < n; r += 32) acc = fma(T[(long)c1 * n + r], T[(long)c2 * n + r], acc);
    acc = warp_sum(acc);
    if (lane == 0) {
      gram[c1 + c2 * K] = acc;
      gram[c2 + c1 * K] = acc;
    }
  }
  __syncthreads();
  const int nact = nact_s;
  // class sums of the training scores (active classes, in class order)
  for (int k = warp; k < nact * K; k += warps) {
    const int ci = k / K, comp = k % K;
    const int cls = active[ci];
    double acc = 0.0;
    for (int r = lane; r < n; r += 32)
      if (v.fold_of_row[r] != f + 1 && v.labels[src_row(v, b, r)] == cls)
        acc += T[(long)comp * n + r];
    acc = warp_sum(acc);
    if (lane == 0) sums[ci * K + comp] = acc;
  }
  __syncthreads();
  const int ntr = v.ntrain[f];
  const int* te = v.test_rows + v.test_off[f];
  const int nte = v.test_off[f + 1] - v.test_off[f];
  for (int j = 0; j < prefix_count; ++j) {
    const int k = prefixes[j];
    if (threadIdx.x == 0) {
      // means (in sums' slots scaled on the fly), pooled covariance, ridge grid
      const double denom = (double)max(1, ntr > nact ? ntr - nact : 1);
      double trace = 0.0;
      for (int c2 = 0; c2 < k; ++c2)
        for (int c1 = 0; c1 < k; ++c1) {
          double val = gram[c1 + c2 * K];
          for (int ci = 0; ci < nact; ++ci) {
            const double nc = (double)cnt[active[ci]];
            val -= nc * (sums[ci * K + c1] / nc) * (sums[ci * K + c2] / nc);
          }
          cov[c1 + c2 * k] = val / denom;
          if (c1 == c2) trace += cov[c1 + c2 * k];
        }
      double scale = trace / k;
      if (!isfinite(scale) || scale <= 0.0) scale = 1.0;
      const double grid[6] = {1e-8, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2};
      bool solved = false;
      for (int g = 0; g < 6 && !solved; ++g) {
        for (int idx = 0; idx < k * k; ++idx) L[idx] = cov[idx];
        if (!cholesky_serial(L, k, grid[g] * scale)) continue;
        bool ok = true;
        for (int ci = 0; ci < nact && ok; ++ci) {
          const double nc = (double)cnt[active[ci]];
          for (int c1 = 0; c1 < k; ++c1) rhs[c1] = sums[ci * K + c1] / nc;
          ok = cholesky_solve_serial(L, k, rhs);
          for (int c1 = 0; c1 < k; ++c1) lin[ci * K + c1] = rhs[c1];
        }
        solved = ok;
      }
      if (!solved) flag_error(flag, 6);
      for (int ci = 0; ci < nact; ++ci) {
        const double nc = (double)cnt[active[ci]];
        double prod = 0.0;
        for (int c1 = 0; c1 < k; ++c1) prod += (sums[ci * K + c1] / nc) * lin[ci * K + c1];
        cst[ci] = -0.5 * prod + log(fmax(nc / (double)ntr, DBL_MIN));
      }
    }
    __syncthreads();
    double hits = 0.0;
    for (int kk = threadIdx.x; kk < nte; kk += blockDim.x) {
      const int r = te[kk];
      int best = -1;
      double bv = 0.0, sv = 0.0;
      bool second = false;
      for (int ci = 0; ci < nact; ++ci) {
        double d = cst[ci];
        for (int c1 = 0; c1 < k; ++c1) d = fma(Tt[(long)c1 * v.max_test + kk], lin[ci * K + c1], d);
        if (best < 0 || d > bv) {
          if (best >= 0) {
            sv = bv;
            second = true;
          }
          best = ci;
          bv = d;
        } else if (!second || d > sv) {
          sv = d;
          second = true;
        }
      }
      if (v.amb && second && !(bv - sv > v.guard * fmax(fabs(bv), fabs(sv)))) v.amb[i] = 1;
      if (best >= 0 && active[best] == v.labels[src_row(v, b, r)]) hits += 1.0;
    }
    hits = block_sum(hits, red);
    if (threadIdx.x == 0) sse[(long)i * prefix_count + j] = hits;
    __syncthreads();
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

// Relative margin of the argmax guard. The int8 digit products (6 digits)
// move held-out scores by well under 1e-6 of their magnitude (worst case seen
// in the kernel-form simulation at the benchmark size: 3.9e-7 on
// predictions); a decision whose top-two gap is within this fraction of the
// score magnitude is not trusted, and its instance is refitted with FP64
// products, so the labels equal those of the FP64 path.
double& argmax_guard() {
  static double margin = 1e-5;
  return margin;
}

int& last_guard_refits() {
  static int count = 0;
  return count;
}

int& batch_autotune() {
  static int on = 1;
  return on;
}

BatchedStats& last_batched_stats() {
  static BatchedStats stats;
  return stats;
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
// Persistent per-device workspace. Every buffer a group's component sequence
// touches lives here, with a stable address across calls (buffers only
// grow), so the sequence can be captured once as a CUDA graph and replayed
// by later calls of the same shape. The engine runs on the workspace's own
// streams: `main` (joined to the caller's stream by events) and one stream
// per lane.
struct LaneState {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  int off = 0, cnt = 0;
  InstanceView v{};
  OzakiOperand rhs;  // int8 digits of this lane's right-hand sides
};

struct GroupGraph {
  std::vector<long long> key;
  cudaGraphExec_t exec = nullptr;
  unsigned long long launches = 0;
};

struct TuneDecision {
  int lanes = 1, tile_n = 0;
  double ms = 0.0;
};

struct BatchedWorkspace {
  int device = -1;
  cudaStream_t main = nullptr;
  cudaEvent_t fork = nullptr, joined = nullptr, t0 = nullptr, t1 = nullptr;
  LaneState lanes[kMaxLanes];
  // group-wide instance arrays; lane l works on instances [off, off + cnt)
  DeviceArray<int> d_if, d_ip, amb;
  DeviceArray<double> C0, C, G, ym, sst, sse, yhat, Wb, KWb, Ws, U, Y1, KC0;
  // per-call inputs and the shared Gram
  OzakiOperand gram_split, x_split;
  DeviceArray<double> gram, Y64, x64;
  DeviceArray<int> d_fold, d_ntrain, d_test_rows, d_test_off, d_slot, d_pre, flag, perms, labels;
  DeviceArray<double> Ttr, Tte;  // LDA head: training / held-out scores per instance
  DeviceArray<int> d_blk;          // candidate-block width per instance
  DeviceArray<double> zblk, cblk;  // candidate blocks: start eigenvectors, start coefficients
  std::vector<GroupGraph> graphs;

  BatchedWorkspace() {
    FPLS_CHECK(cudaGetDevice(&device));
    FPLS_CHECK(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking));
    FPLS_CHECK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    FPLS_CHECK(cudaEventCreateWithFlags(&joined, cudaEventDisableTiming));
    FPLS_CHECK(cudaEventCreate(&t0));
    FPLS_CHECK(cudaEventCreate(&t1));
    for (LaneState& L : lanes) {
      FPLS_CHECK(cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking));
      FPLS_CHECK(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
    }
  }
  BatchedWorkspace(const BatchedWorkspace&) = delete;
  BatchedWorkspace& operator=(const BatchedWorkspace&) = delete;
  ~BatchedWorkspace() {
    cudaStreamSynchronize(main);
    for (LaneState& L : lanes) cudaStreamSynchronize(L.st);
    drop_graphs();
    // free every buffer while the streams it was allocated on still exist
    for (LaneState& L : lanes) {
      L.rhs.digits.release();
      L.rhs.scale.release();
    }
    for (auto* a : {&d_if, &d_ip, &amb, &d_fold, &d_ntrain, &d_test_rows, &d_test_off, &d_slot,
                    &d_pre, &flag, &perms, &labels, &d_blk})
      a->release();
    for (auto* a : {&C0, &C, &G, &ym, &sst, &sse, &yhat, &Wb, &KWb, &Ws, &U, &Y1, &KC0, &gram,
                    &Y64, &x64, &Ttr, &Tte, &zblk, &cblk})
      a->release();
    for (OzakiOperand* o : {&gram_split, &x_split}) {
      o->digits.release();
      o->scale.release();
    }
    cudaStreamSynchronize(main);
    for (LaneState& L : lanes) {
      cudaStreamSynchronize(L.st);
      cudaEventDestroy(L.done);
      cudaStreamDestroy(L.st);
    }
    for (cudaEvent_t e : {fork, joined, t0, t1}) cudaEventDestroy(e);
    cudaStreamDestroy(main);
  }
  void drop_graphs() {
    for (GroupGraph& g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
  }
  // Device bytes held by the instance arrays and the Gram (reused by the
  // next call, so they count as available when a group is sized).
  size_t held_bytes() const {
    size_t b = (d_if.size() + d_ip.size() + amb.size()) * sizeof(int);
    for (const auto* a : {&C0, &C, &G, &ym, &sst, &sse, &yhat, &Wb, &KWb, &Ws, &U, &Y1, &KC0,
                          &gram, &Ttr, &Tte, &zblk, &cblk})
      b += a->size() * sizeof(double);
    return b + gram_split.digits.size();
  }
};

namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kMaxGraphs = 16;

std::mutex& workspace_mutex() {
  static std::mutex mu;
  return mu;
}

BatchedWorkspace*& workspace_slot(int device) {
  static BatchedWorkspace* slots[kMaxDevices] = {};
  return slots[device];
}

// Grow-only buffer sizing (the address is kept while it is large enough).
template <class U>
void grow(DeviceArray<U>& a, size_t count, cudaStream_t s) {
  if (count == 0) count = 1;
  if (count > a.size() || !a) a.allocate(count, s);
}

// Schedule decisions of the autotuner, keyed on the group shape; optionally
// persisted in the file named by FASTPLS_B200_TUNE_FILE (one decision per
// line: n p q instances components digits classification lanes tile ms).
struct Tuner {
  std::mutex mu;
  std::map<std::vector<long long>, TuneDecision> decisions;
  bool loaded = false;

  const char* path() const { return std::getenv("FASTPLS_B200_TUNE_FILE"); }
  void load() {
    if (loaded) return;
    loaded = true;
    const char* f = path();
    if (!f) return;
    std::ifstream in(f);
    std::vector<long long> k(7);
    TuneDecision d;
    while (in >> k[0] >> k[1] >> k[2] >> k[3] >> k[4] >> k[5] >> k[6] >> d.lanes >> d.tile_n >> d.ms)
      if (d.lanes >= 1 && d.lanes <= kMaxLanes && (d.tile_n == 192 || d.tile_n == 256))
        decisions[k] = d;
  }
  bool find(const std::vector<long long>& key, TuneDecision* out) {
    std::lock_guard<std::mutex> lock(mu);
    load();
    auto it = decisions.find(key);
    if (it == decisions.end()) return false;
    *out = it->second;
    return true;
  }
  void store(const std::vector<long long>& key, const TuneDecision& d) {
    std::lock_guard<std::mutex> lock(mu);
    load();
    decisions[key] = d;
    if (const char* f = path()) {
      std::ofstream out(f, std::ios::app);
      for (long long v : key) out << v << ' ';
      out << d.lanes << ' ' << d.tile_n << ' ' << d.ms << '\n';
    }
  }
};

Tuner& tuner() {
  static Tuner t;
  return t;
}

}  // namespace

void release_batched_workspace() {
  std::lock_guard<std::mutex> lock(workspace_mutex());
  for (int d = 0; d < kMaxDevices; ++d) {
    delete workspace_slot(d);
    workspace_slot(d) = nullptr;
  }
}

// ---------------------------------------------------------------------------
template <class T>
void BatchedCv<T>::form_gram(const double* kscale, cudaStream_t s) {
  grow(ws->gram, (size_t)n * n, s);
  if (digits > 0) {
    // int8 digits of the rows of X D^1/2, the symmetric product on the int8
    // tensor cores (lower tiles + mirror), then the digits of K's rows for
    // every later product with K; X's digits are freed once K is formed
    ozaki_split_colmajor<T>(X, n, p, n, kscale, digits, ws->x_split, ws->flag.get(), s);
    ozaki_gemm(ws->x_split, ws->x_split, ws->gram.get(), n, true, ws->flag.get(), s);
    ozaki_split_rows(ws->gram.get(), n, n, n, digits, ws->gram_split, ws->flag.get(), s);
    ws->x_split.digits.release();
    ws->x_split.scale.release();
    return;
  }
  // FP64 copy of X with the scaling folded in (X D^1/2), then the symmetric
  // product on the FP64 tensor-core path (lower tiles + mirror).
  grow(ws->x64, (size_t)n * p, s);
  const long total = (long)n * p;
  scale_columns_f64<T><<<(unsigned)std::min<long>((total + 255) / 256, 16L * num_sms()), 256, 0, s>>>(
      X, n, p, kscale, ws->x64.get());
  count_launch();
  FPLS_LAUNCH("scale_columns_f64");
  GemmArgs g;
  g.M = n;
  g.N = n;
  g.K = p;
  g.A = ws->x64.get();
  g.lda = n;
  g.B = ws->x64.get();
  g.ldb = n;
  g.trans_b = true;
  g.C = ws->gram.get();
  g.ldc = n;
  g.lower = gemm_mma_supported(g);
  gemm_f64(g, s);
}

template <class T>
void BatchedCv<T>::gram_product(const double* rhs, int cols, double* out,
                                OzakiOperand& rhs_split, int tile_n, cudaStream_t s) {
  if (digits > 0) {
    // K is symmetric: its rows are its columns (contiguous, ld n)
    ozaki_split_rows(rhs, n, cols, n, digits, rhs_split, ws->flag.get(), s);
    ozaki_gemm(ws->gram_split, rhs_split, out, n, false, ws->flag.get(), s, tile_n);
    return;
  }
  GemmArgs g;
  g.M = n;
  g.N = cols;
  g.K = n;
  g.A = ws->gram.get();
  g.lda = n;
  g.B = rhs;
  g.ldb = n;
  g.C = out;
  g.ldc = n;
  gemm_f64(g, s);
}

// The whole component sequence of one group. The instances run in lanes of
// their own CUDA stream, enqueued component by component in turn, so that
// the memory-bound score and deflation kernels of one lane overlap the
// tensor-core products of another. Lanes share the Gram and its digits
// (read only). Fork from s at the start, join into s at the end; nothing in
// here allocates, synchronises or reads back, so it can be captured.
template <class T>
void BatchedCv<T>::enqueue_group(int I, int nlanes, int tile_n, cudaStream_t s) {
  const size_t smem_dir = 2 * (size_t)q * q * sizeof(double);
  const size_t smem_defl = (2 * (size_t)q * q + 2 * (size_t)kmax + q) * sizeof(double);
  const size_t nq = (size_t)n * q;
  const int rpt = rows_per_thread(n);
  FPLS_CHECK(cudaEventRecord(ws->fork, s));
  for (int l = 0; l < nlanes; ++l) {
    LaneState& L = ws->lanes[l];
    const cudaStream_t st = L.st;
    const int c = L.cnt;
    const size_t o = L.off;
    const InstanceView& v = L.v;
    FPLS_CHECK(cudaStreamWaitEvent(st, ws->fork, 0));
    if (v.amb) FPLS_CHECK(cudaMemsetAsync(v.amb, 0, sizeof(int) * c, st));
    init_instances<<<c, BT, 0, st>>>(v, ws->C0.get() + o * nq, ws->C.get() + o * nq,
                                     ws->ym.get() + o * q, ws->sst.get() + o,
                                     ws->yhat.get() + o * max_test * q, max_test,
                                     ws->sse.get() + o * prefix_count, prefix_count);
    count_launch();
    FPLS_LAUNCH("init_instances");
    // G0 = C0^T K C0 via one product over all instances' C0 columns
    gram_product(ws->C0.get() + o * nq, q * c, ws->KC0.get() + o * nq, L.rhs, tile_n, st);
    initial_gram<<<c, BT, 0, st>>>(v, ws->C0.get() + o * nq, ws->KC0.get() + o * nq,
                                   ws->G.get() + o * q * (q + 1) / 2);
    count_launch();
    FPLS_LAUNCH("initial_gram");
    // first direction; K u comes from K C0 (no GEMM)
    direction_batched<<<c, BT, smem_dir, st>>>(v, ws->G.get() + o * q * (q + 1) / 2,
                                               ws->C.get() + o * nq, ws->U.get() + o * n,
                                               ws->KC0.get() + o * nq, ws->Y1.get() + o * n,
                                               ws->flag.get());
    count_launch();
    FPLS_LAUNCH("direction_batched");
  }
  for (int a = 0; a < kmax; ++a) {
    for (int l = 0; l < nlanes; ++l) {
      LaneState& L = ws->lanes[l];
      const cudaStream_t st = L.st;
      const int c = L.cnt;
      const size_t o = L.off;
      const InstanceView& v = L.v;
      double* U = ws->U.get() + o * n;
      double* Y1 = ws->Y1.get() + o * n;
      double* C0 = ws->C0.get() + o * nq;
      double* ym = ws->ym.get() + o * q;
      double* yhat = ws->yhat.get() + o * max_test * q;
      double* sse = ws->sse.get() + o * prefix_count;
      if (a > 0) gram_product(U, c, Y1, L.rhs, tile_n, st);  // Y1 = K u
      switch (rpt) {
#define FPLS_SCORES(R)                                                                  \
  case R:                                                                               \
    scores_rows<R><<<c, BT, 0, st>>>(v, Y1, U, C0, ym, yhat, max_test, a, ws->d_slot.get(), \
                                     prefix_count, sse, ws->flag.get());                \
    break;
        FPLS_SCORES(8)
        FPLS_SCORES(16)
        FPLS_SCORES(20)
        FPLS_SCORES(24)
        FPLS_SCORES(32)
#undef FPLS_SCORES
        default:
          scores_batched<<<c, BT, 0, st>>>(v, Y1, U, C0, ym, yhat, max_test, a, ws->d_slot.get(),
                                           prefix_count, sse, nullptr, ws->flag.get());
      }
      count_launch();
      FPLS_LAUNCH("scores_batched");
      if (a + 1 == kmax) continue;  // the last deflation is never used
      // Y1 = K t~ (U holds the masked training scores)
      gram_product(U, c, Y1, L.rhs, tile_n, st);
      double* Wb = ws->Wb.get() + o * n * kmax;
      double* KWb = ws->KWb.get() + o * n * kmax;
      double* Ws = ws->Ws.get() + o * kmax;
      double* C = ws->C.get() + o * nq;
      double* G = ws->G.get() + o * q * (q + 1) / 2;
      if (q <= 4)
        deflate_batched<4><<<c, DEFL_BT, smem_defl, st>>>(v, Y1, U, Wb, KWb, Ws, C, G, a,
                                                          ws->flag.get());
      else
        deflate_batched<kBatchMaxResponses><<<c, DEFL_BT, smem_defl, st>>>(
            v, Y1, U, Wb, KWb, Ws, C, G, a, ws->flag.get());
      count_launch();
      FPLS_LAUNCH("deflate_batched");
    }
  }
  if (lda_head) {
    const size_t smem_lda =
        (3 * (size_t)kmax * kmax + 2 * (size_t)q * kmax + q + kmax) * sizeof(double);
    for (int l = 0; l < nlanes; ++l) {
      LaneState& L = ws->lanes[l];
      lda_heads<<<L.cnt, LDA_BT, smem_lda, L.st>>>(L.v, ws->d_pre.get(), prefix_count,
                                                     ws->sse.get() + (size_t)L.off * prefix_count,
                                                     ws->flag.get());
      count_launch();
      FPLS_LAUNCH("lda_heads");
    }
  }
  for (int l = 0; l < nlanes; ++l) {
    FPLS_CHECK(cudaEventRecord(ws->lanes[l].done, ws->lanes[l].st));
    FPLS_CHECK(cudaStreamWaitEvent(s, ws->lanes[l].done, 0));
  }
}

// One group of instances: lay the lanes out over the group-wide arrays, pick
// the schedule (autotuned on the first group of a new shape), run the
// component sequence (a replayed CUDA graph when the products are int8), and
// collect each instance's sums.
template <class T>
void BatchedCv<T>::run_group(const std::vector<int>& inst_fold,
                             const std::vector<int>& inst_perm, cudaStream_t s) {
  const int I = (int)inst_fold.size();
  if (I == 0) return;
  BatchedStats& stats = last_batched_stats();
  const size_t nq = (size_t)n * q;
  const size_t cI = (size_t)I;
  grow(ws->d_if, cI, s);
  grow(ws->d_ip, cI, s);
  grow(ws->amb, cI, s);
  grow(ws->C0, nq * cI, s);
  grow(ws->C, nq * cI, s);
  grow(ws->G, cI * q * (q + 1) / 2, s);
  grow(ws->ym, cI * q, s);
  grow(ws->sst, cI, s);
  grow(ws->sse, cI * prefix_count, s);
  grow(ws->yhat, cI * max_test * q, s);
  grow(ws->Wb, cI * n * kmax, s);
  grow(ws->KWb, cI * n * kmax, s);
  grow(ws->Ws, cI * kmax, s);
  grow(ws->U, (size_t)n * cI, s);
  grow(ws->Y1, (size_t)n * cI, s);
  grow(ws->KC0, nq * cI, s);
  if (lda_head) {
    grow(ws->Ttr, (size_t)n * kmax * cI, s);
    grow(ws->Tte, (size_t)max_test * kmax * cI, s);
  }
  // candidate-block widths of this group's instances
  std::vector<int> hblk(I, 1);
  bool any_block = false;
  if (!blocks.empty())
    for (int k = 0; k < I; ++k) {
      hblk[k] = std::max(1, blocks[(size_t)(inst_perm[k] + 1) * folds + inst_fold[k]]);
      any_block = any_block || hblk[k] > 1;
    }
  if (any_block) {
    grow(ws->d_blk, cI, s);
    grow(ws->zblk, (size_t)q * q * cI, s);
    grow(ws->cblk, nq * cI, s);
    FPLS_CHECK(cudaMemcpyAsync(ws->d_blk.get(), hblk.data(), sizeof(int) * I,
                               cudaMemcpyHostToDevice, s));
  }
  FPLS_CHECK(cudaMemcpyAsync(ws->d_if.get(), inst_fold.data(), sizeof(int) * I,
                             cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(ws->d_ip.get(), inst_perm.data(), sizeof(int) * I,
                             cudaMemcpyHostToDevice, s));
  const bool guard = class_labels && digits > 0 && argmax_guard() > 0.0;

  // candidate schedules: lanes (each at least kLaneMinInstances instances)
  // x tile widths 192 / 256, which combine the digit diagonals in the same
  // FP64 order, so every candidate gives bit-identical results
  const int max_lanes = std::max(1, std::min(kMaxLanes, I / kLaneMinInstances));
  std::vector<TuneDecision> cands;
  TuneDecision chosen;
  chosen.lanes = std::max(1, std::min(batch_lanes(), max_lanes));
  chosen.tile_n = digits > 0 ? ozaki_wide_tile(n, ceil_div(I, chosen.lanes)) : 0;
  const std::vector<long long> key = {n, p, q, I, kmax, digits, class_labels ? 1 : 0};
  bool tune = false;
  if (digits > 0 && batch_autotune() && !ozaki_profile_enabled()) {
    TuneDecision d;
    if (tuner().find(key, &d) && d.lanes <= max_lanes) {
      chosen = d;
    } else {
      tune = true;
      for (int nl = 1; nl <= max_lanes; ++nl)
        for (int tn : {192, 256}) cands.push_back({nl, tn, 0.0});
    }
  }
  if (!tune) cands.assign(1, chosen);

  auto layout = [&](int nlanes, int tile_n) {
    for (int l = 0; l < nlanes; ++l) {
      LaneState& L = ws->lanes[l];
      L.off = l * (I / nlanes);
      L.cnt = l + 1 == nlanes ? I - L.off : I / nlanes;
      InstanceView& v = L.v;
      v.n = n;
      v.q = q;
      v.kmax = kmax;
      v.B = 0;
      v.center = center ? 1 : 0;
      v.fold_of_row = ws->d_fold.get();
      v.inst_fold = ws->d_if.get() + L.off;
      v.inst_perm = ws->d_ip.get() + L.off;
      v.perms = perms;
      v.ntrain = ws->d_ntrain.get();
      v.test_rows = ws->d_test_rows.get();
      v.test_off = ws->d_test_off.get();
      v.Y = ws->Y64.get();
      v.labels = class_labels;
      v.guard = argmax_guard();
      v.amb = guard ? ws->amb.get() + L.off : nullptr;
      v.max_test = max_test;
      v.ttr = lda_head ? ws->Ttr.get() + (size_t)L.off * n * kmax : nullptr;
      v.tte = lda_head ? ws->Tte.get() + (size_t)L.off * max_test * kmax : nullptr;
      v.blk = any_block ? ws->d_blk.get() + L.off : nullptr;
      v.zblk = any_block ? ws->zblk.get() + (size_t)L.off * q * q : nullptr;
      v.cblk = any_block ? ws->cblk.get() + (size_t)L.off * nq : nullptr;
      if (digits > 0) {
        // size the digits of the largest right-hand side (K C0: q columns
        // per instance) so the products inside the sequence never allocate
        ozaki_reserve(L.rhs, std::max(q, 1) * L.cnt, n, digits, L.st);
      }
    }
    (void)tile_n;
  };

  const bool use_graph = digits > 0 && !ozaki_profile_enabled();
  auto run_schedule = [&](const TuneDecision& d, bool timed) -> double {
    layout(d.lanes, d.tile_n);
    if (timed) FPLS_CHECK(cudaEventRecord(ws->t0, s));
    if (use_graph) {
      std::vector<long long> gkey = {n, q, I, kmax, prefix_count, max_test, digits, center,
                                     d.lanes, d.tile_n, class_labels ? 1 : 0, guard ? 1 : 0,
                                     lda_head ? 1 : 0, any_block ? 1 : 0};
      long long gbits = 0;
      const double gv = argmax_guard();
      std::memcpy(&gbits, &gv, sizeof(gbits));
      gkey.push_back(gbits);
      for (const void* ptr :
           {(const void*)ws->d_if.get(), (const void*)ws->d_ip.get(), (const void*)ws->amb.get(),
            (const void*)ws->C0.get(), (const void*)ws->C.get(), (const void*)ws->G.get(),
            (const void*)ws->ym.get(), (const void*)ws->sst.get(), (const void*)ws->sse.get(),
            (const void*)ws->yhat.get(), (const void*)ws->Wb.get(), (const void*)ws->KWb.get(),
            (const void*)ws->Ws.get(), (const void*)ws->U.get(), (const void*)ws->Y1.get(),
            (const void*)ws->KC0.get(), (const void*)ws->gram_split.digits.get(),
            (const void*)ws->gram_split.scale.get(), (const void*)ws->Y64.get(),
            (const void*)ws->d_fold.get(), (const void*)ws->d_ntrain.get(),
            (const void*)ws->d_test_rows.get(), (const void*)ws->d_test_off.get(),
            (const void*)ws->d_slot.get(), (const void*)ws->flag.get(), (const void*)perms,
            (const void*)class_labels, (const void*)ws->d_pre.get(), (const void*)ws->Ttr.get(),
            (const void*)ws->Tte.get(), (const void*)ws->d_blk.get(), (const void*)ws->zblk.get(),
            (const void*)ws->cblk.get()})
        gkey.push_back((long long)(uintptr_t)ptr);
      for (int l = 0; l < d.lanes; ++l) {
        gkey.push_back((long long)(uintptr_t)ws->lanes[l].rhs.digits.get());
        gkey.push_back((long long)(uintptr_t)ws->lanes[l].rhs.scale.get());
      }
      GroupGraph* found = nullptr;
      for (GroupGraph& g : ws->graphs)
        if (g.key == gkey) found = &g;
      if (!found) {
        const unsigned long long before = launch_count();
        cudaGraph_t graph = nullptr;
        FPLS_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
          enqueue_group(I, d.lanes, d.tile_n, s);
        } catch (...) {
          cudaStreamEndCapture(s, &graph);
          if (graph) cudaGraphDestroy(graph);
          cudaGetLastError();
          throw;
        }
        FPLS_CHECK(cudaStreamEndCapture(s, &graph));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t rc = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        FPLS_CHECK(rc);
        if (ws->graphs.size() >= kMaxGraphs) {
          cudaGraphExecDestroy(ws->graphs.front().exec);
          ws->graphs.erase(ws->graphs.begin());
        }
        GroupGraph g;
        g.key = gkey;
        g.exec = exec;
        // nothing ran during the capture: count the kernels when replayed
        g.launches = launch_count() - before;
        uncount_launch(g.launches);
        ws->graphs.push_back(std::move(g));
        found = &ws->graphs.back();
        ++stats.graph_captures;
      }
      FPLS_CHECK(cudaGraphLaunch(found->exec, s));
      count_launch((unsigned)found->launches);
      ++stats.graph_replays;
    } else {
      enqueue_group(I, d.lanes, d.tile_n, s);
    }
    if (!timed) return 0.0;
    FPLS_CHECK(cudaEventRecord(ws->t1, s));
    FPLS_CHECK(cudaEventSynchronize(ws->t1));
    float ms = 0.f;
    FPLS_CHECK(cudaEventElapsedTime(&ms, ws->t0, ws->t1));
    return ms;
  };

  if (tune) {
    // every candidate computes the full group (identical results); the
    // first run of each also captures its graph, so time a second replay
    TuneDecision best;
    best.ms = -1.0;
    for (TuneDecision& c : cands) {
      run_schedule(c, false);
      c.ms = run_schedule(c, true);
      if (best.ms < 0.0 || c.ms < best.ms) best = c;
    }
    tuner().store(key, best);
    chosen = best;
    ++stats.tuned;
    // the last candidate's results are in place; when it is not the chosen
    // schedule the results are the same, bit for bit
  } else {
    run_schedule(chosen, false);
  }
  ++stats.groups;
  stats.lanes = chosen.lanes;
  stats.tile_n = chosen.tile_n;

  // collect per-instance sums
  std::vector<double> h_sse((size_t)I * prefix_count), h_sst(I);
  std::vector<int> h_amb(I, 0);
  if (guard)
    FPLS_CHECK(cudaMemcpyAsync(h_amb.data(), ws->amb.get(), sizeof(int) * I,
                               cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaMemcpyAsync(h_sse.data(), ws->sse.get(), sizeof(double) * I * prefix_count,
                             cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaMemcpyAsync(h_sst.data(), ws->sst.get(), sizeof(double) * I,
                             cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaStreamSynchronize(s));
  for (int k = 0; k < I; ++k) {
    if (h_amb[k]) {
      amb_fold.push_back(inst_fold[k]);
      amb_perm.push_back(inst_perm[k]);
    }
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
                       int scaling_, cudaStream_t caller) {
  X = X_;
  n = n_;
  p = p_;
  q = q_;
  P = perm_count;
  prefix_count = count;
  scaling = scaling_;
  center = scaling != 3;
  digits = ozaki_slices();
  require(q >= 1 && q <= kBatchMaxResponses, "batched CV supports 1..32 responses");
  require(!lda_head || class_labels, "the LDA head needs class labels");
  kmax = 0;
  for (int j = 0; j < count; ++j) {
    if (prefixes_[j] <= kmax) throw std::invalid_argument("CUDA CV component path must be strictly increasing");
    kmax = prefixes_[j];
  }
  require(!lda_head || kmax <= kLdaMaxComponents,
          "batched classification with the LDA head takes up to 32 components");
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

  // One batched call at a time uses the device's persistent workspace;
  // a concurrent call (another host thread) gets a private one.
  int dev = 0;
  FPLS_CHECK(cudaGetDevice(&dev));
  require(dev >= 0 && dev < kMaxDevices, "device index beyond the batched workspace table");
  std::unique_lock<std::mutex> lock(workspace_mutex(), std::try_to_lock);
  std::unique_ptr<BatchedWorkspace> own;
  if (lock.owns_lock()) {
    if (!workspace_slot(dev)) workspace_slot(dev) = new BatchedWorkspace();
    ws = workspace_slot(dev);
  } else {
    own.reset(new BatchedWorkspace());
    ws = own.get();
  }
  last_batched_stats() = BatchedStats{};
  if (digits > 0) ozaki_configure_kernels();  // attributes are not set inside a capture
  const cudaStream_t s = ws->main;
  // the caller's earlier work (input copies) before ours; ours before its later work
  FPLS_CHECK(cudaEventRecord(ws->fork, caller));
  FPLS_CHECK(cudaStreamWaitEvent(s, ws->fork, 0));
  struct Join {
    BatchedWorkspace* ws;
    cudaStream_t caller;
    ~Join() {
      if (cudaEventRecord(ws->joined, ws->main) == cudaSuccess)
        cudaStreamWaitEvent(caller, ws->joined, 0);
    }
  } join{ws, caller};

  grow(ws->d_fold, n, s);
  grow(ws->d_ntrain, folds, s);
  grow(ws->d_test_rows, test_rows.size(), s);
  grow(ws->d_test_off, folds + 1, s);
  grow(ws->d_slot, kmax + 1, s);
  grow(ws->d_pre, count, s);
  grow(ws->flag, 1, s);
  FPLS_CHECK(cudaMemsetAsync(ws->flag.get(), 0, sizeof(int), s));
  FPLS_CHECK(cudaMemcpyAsync(ws->d_fold.get(), folds_host, sizeof(int) * n, cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(ws->d_ntrain.get(), ntrain.data(), sizeof(int) * folds, cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(ws->d_test_rows.get(), test_rows.data(), sizeof(int) * test_rows.size(), cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(ws->d_test_off.get(), test_off.data(), sizeof(int) * (folds + 1), cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(ws->d_slot.get(), slot.data(), sizeof(int) * (kmax + 1), cudaMemcpyHostToDevice, s));
  FPLS_CHECK(cudaMemcpyAsync(ws->d_pre.get(), prefixes_, sizeof(int) * count, cudaMemcpyHostToDevice, s));
  // permutations and labels are copied in, so that captured groups always
  // read them at the workspace's addresses
  perms = nullptr;
  if (P > 0) {
    grow(ws->perms, (size_t)P * n, s);
    FPLS_CHECK(cudaMemcpyAsync(ws->perms.get(), perms_dev, sizeof(int) * (size_t)P * n,
                               cudaMemcpyDeviceToDevice, s));
    perms = ws->perms.get();
  }
  const int* caller_labels = class_labels;
  if (caller_labels) {
    grow(ws->labels, n, s);
    FPLS_CHECK(cudaMemcpyAsync(ws->labels.get(), caller_labels, sizeof(int) * n,
                               cudaMemcpyDeviceToDevice, s));
    class_labels = ws->labels.get();
  }
  grow(ws->Y64, (size_t)n * q, s);
  to_f64<T><<<std::min<unsigned>(ceil_div((size_t)n * q, 256), 4 * num_sms()), 256, 0, s>>>(Y_, (long)n * q, ws->Y64.get());
  count_launch();
  FPLS_LAUNCH("to_f64");
  {
    DeviceArray<double> cs((size_t)2 * q, s);
    response_moments<<<q, 256, 0, s>>>(ws->Y64.get(), n, cs.get());
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
  // KW, U, Y1 and held-out predictions); the workspace's instance arrays are
  // reused, so they count as available
  size_t free_b = 0, total_b = 0;
  FPLS_CHECK(cudaMemGetInfo(&free_b, &total_b));
  free_b += ws->held_bytes();
  const size_t per_inst = sizeof(double) * ((size_t)n * (3 * q + 2 * kmax + 2) + (size_t)max_test * q + 64);
  const size_t gram_b = (size_t)n * n * 8 + (digits > 0 ? (size_t)digits * n * n : 0);
  const size_t budget = free_b > gram_b + (1ull << 30) ? free_b - gram_b - (1ull << 30) : per_inst;
  const int max_group = std::max(1, (int)std::min<size_t>(budget * 7 / 10 / per_inst, 1 << 20));

  auto run_instances = [&](const std::vector<int>& fl, const std::vector<int>& pl) {
    for (size_t off = 0; off < fl.size(); off += max_group) {
      const size_t cnt = std::min(fl.size() - off, (size_t)max_group);
      std::vector<int> a(fl.begin() + off, fl.begin() + off + cnt);
      std::vector<int> b(pl.begin() + off, pl.begin() + off + cnt);
      run_group(a, b, s);
    }
  };
  // Classification with int8 products: instances with a held-out decision
  // inside the argmax margin are refitted with FP64 products (FP64 Gram and
  // DMMA products), replacing their hit counts.
  amb_fold.clear();
  amb_perm.clear();
  refitted = 0;
  auto refit_ambiguous = [&](const double* kscale) {
    if (amb_fold.empty()) return;
    const int saved = digits;
    std::vector<int> fl, pl;
    fl.swap(amb_fold);
    pl.swap(amb_perm);
    refitted += (int)fl.size();
    digits = 0;
    form_gram(kscale, s);
    run_instances(fl, pl);
    digits = saved;
    amb_fold.clear();
    amb_perm.clear();
  };

  if (scaling == 2) {
    // autoscaling: one Gram per fold with that fold's training-row scales
    DeviceArray<double> mom((size_t)2 * p, s), hmom((size_t)2 * p, s), ks(p, s);
    DeviceArray<double> scratch;
    column_moments<T>(X, n, p, n, nullptr, 0, mom.get(), mom.get() + p, nullptr, scratch, s);
    for (int f = 0; f < folds; ++f) {
      if (test[f].empty()) continue;
      heldout_moments<T><<<std::min(p, 8 * num_sms()), 256, 0, s>>>(
          X, n, p, ws->d_test_rows.get() + test_off[f], (int)test[f].size(), hmom.get(), hmom.get() + p);
      fold_kscale<<<std::min<unsigned>(ceil_div(p, 256), 4 * num_sms()), 256, 0, s>>>(
          mom.get(), mom.get() + p, hmom.get(), hmom.get() + p, p, ntrain[f], ks.get());
      count_launch(2);
      FPLS_LAUNCH("fold scales");
      form_gram(ks.get(), s);
      std::vector<int> fl, pl;
      for (int b = 0; b < B; ++b) {
        if (!skip.empty() && skip[(size_t)b * folds + f]) continue;
        fl.push_back(f);
        pl.push_back(b - 1);
      }
      run_instances(fl, pl);
      refit_ambiguous(ks.get());
    }
  } else {
    form_gram(nullptr, s);
    std::vector<int> fl, pl;
    for (int b = 0; b < B; ++b)
      for (int f = 0; f < folds; ++f) {
        if (test[f].empty()) continue;
        if (!skip.empty() && skip[(size_t)b * folds + f]) continue;
        fl.push_back(f);
        pl.push_back(b - 1);
      }
    run_instances(fl, pl);
    refit_ambiguous(nullptr);
  }
  last_guard_refits() = refitted;
  int bad = 0;
  FPLS_CHECK(cudaMemcpyAsync(&bad, ws->flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  FPLS_CHECK(cudaStreamSynchronize(s));
  class_labels = caller_labels;
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
        if (status[f] != 1 && status[f] != 4) continue;
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
