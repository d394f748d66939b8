// Persistent single-fit SIMPLS: every component of a fit in one cooperative
// launch.
//
// The per-component step of the p-space SIMPLS loop (the reference's
// ComponentWorkspace::step, src/cuda_resident_component.cuh:94-130, and the
// FP64 CPU body, inst/include/fastpls/core/simpls.hpp:588-756) is two
// HBM-streaming passes over X (t = X r, p = X^T t) plus O(p (a + m)) vector
// work whose reductions are grid-wide. As separate kernels that is about ten
// launches per component, most of them tiny and latency-bound. Here one
// grid of CTAs stays resident for the whole fit and walks through the
// phases of each component, separated by group barriers:
//
//   B0  (last CTA) reduce the Gram of the deflated S, Jacobi -> z / sqrt(lambda)
//   P1  r = S z, rt = r / scale, partial  c = mean . rt             -> B1: c
//   P2  t partials over column chunks: sum_j X[i, j] rt[j]          -> B2
//   P3  t = sum of partials - c, partial |t|^2 and sum t            -> B3: |t|, sum t
//   P4  loading partials over row chunks: sum_i X[i, j] t[i]        -> B4
//   P5  p = (X^T t - mean sum t) / (scale |t|), R[:, a] = r / |t|,
//       partial V^T p and S0^T R[:, a]                              -> B5: h, q
//   P6  v = p - V h, partial v.v and S^T v                          -> B6: |v|, S^T v
//   P7  V[:, a] = v / |v|, S -= V[:, a] (S^T v / |v|)^T, partial Gram
//       of S, T[:, a] /= |t|
//
// At each barrier the last CTA to arrive adds the per-CTA partials in CTA
// order (deterministic) and publishes the result before releasing the
// others. Chunk sizes depend only on (n, p), so the result does not depend
// on the storage type of X: BF16 storage gives the same bits as FP32
// storage of the same values. All arithmetic is FP64.
//
// Every barrier wait is bounded (about 2 s): on expiry the CTA sets the
// error flag (5) and returns, so a fit never hangs. Blocks of one fit wait on
// each other only inside this one cooperative launch (all of its CTAs are
// co-resident).
#include "kernels.cuh"
#include "model.cuh"
#include "persistent.cuh"
#include "small.cuh"

#include <algorithm>
#include <memory>
#include <vector>

namespace fpls {

namespace {

constexpr int PT = 256;                       // threads per CTA
constexpr int kMaxXrCols = 2048;              // columns of rt staged per item
constexpr int kMaxXtvRows = 4096;             // rows of t staged per item
constexpr int kGramRows = 64;                 // S rows staged per Gram step
constexpr int kSmemDoubles = 4096;            // 32 KB of dynamic shared memory
constexpr long long kBarrierCycles = 4000000000LL;  // about 2 s

// scalar slots of a fit (global, FP64)
constexpr int SC_Z = 0;            // z / sqrt(lambda): kPersistMaxResponses
constexpr int SC_C = 32;           // mean . rt
constexpr int SC_T2 = 33;          // |t|^2
constexpr int SC_ST = 34;          // sum t
constexpr int SC_VV = 35;          // |v|^2
constexpr int SC_Q = 40;           // q (m)
constexpr int SC_SV = 72;          // S^T v (m)
constexpr int SC_U = 104;          // S^T (mean / scale) (m)
constexpr int SC_H = 136;          // V^T p (a)

using Fit = PersistentFit;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Barrier of the fit's CTAs. Every thread of the CTA calls it after writing
// its partials. The last CTA to arrive runs reduce() (whole CTA, reading the
// other CTAs' partials with L1-bypassing loads) before releasing the rest.
// Returns false when a wait ran out (flag set to 5); the caller returns.
template <class F>
__device__ bool group_sync(const Fit& f, int* flag, F&& reduce) {
  __shared__ int last_s, ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned gen = ld_acquire(f.bar + 1);
    __threadfence();
    const unsigned ticket = atomicAdd(f.bar, 1u);
    last_s = ticket == (unsigned)f.C - 1u;
    ok_s = 1;
    if (!last_s) {
      const long long t0 = clock64();
      while (ld_acquire(f.bar + 1) == gen) {
        if (clock64() - t0 > f.barrier_cycles) {
          flag_error(flag, 5);
          ok_s = 0;
          break;
        }
        __nanosleep(64);
      }
    }
  }
  __syncthreads();
  if (last_s) {
    __threadfence();
    reduce();
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicExch(f.bar, 0u);
      __threadfence();
      atomicAdd(f.bar + 1, 1u);
    }
  }
  __syncthreads();
  __threadfence();
  return ok_s != 0;
}

// CTA-level sum; every thread receives it.
__device__ __forceinline__ double cta_sum(double v, double* red) { return block_sum(v, red); }

// Contiguous column range [j0, j1) of CTA `c` out of C over p columns.
__device__ __forceinline__ void col_range(int p, int C, int c, int& j0, int& j1) {
  const int per = (p + C - 1) / C;
  j0 = min(p, c * per);
  j1 = min(p, j0 + per);
}

// Sums over the C per-CTA partials of slots 0 .. count-1 (stride cslots),
// by the whole CTA: warp w takes slots w, w + 8, ...; lane l adds the
// partials of CTAs l, l + 32, ... in order, then the warp's shuffle tree
// (a fixed order). store(k, sum) runs on lane 0.
template <class F>
__device__ __forceinline__ void reduce_slots(const Fit& f, int count, F&& store) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = warp; k < count; k += PT / 32) {
    double s = 0.0;
#pragma unroll 4
    for (int c = lane; c < f.C; c += 32) s += __ldcg(f.cpart + (long)c * f.cslots + k);
    s = warp_sum(s);
    if (lane == 0) store(k, s);
  }
}

template <class T> struct Vec16;
template <> struct Vec16<float> {
  static constexpr int N = 4;
  using type = float4;
  static __device__ __forceinline__ void get(const type& v, double (&o)[4]) {
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
};
template <> struct Vec16<double> {
  static constexpr int N = 2;
  using type = double2;
  static __device__ __forceinline__ void get(const type& v, double (&o)[2]) {
    o[0] = v.x; o[1] = v.y;
  }
};
template <> struct Vec16<bf16> {
  static constexpr int N = 8;
  using type = uint4;
  static __device__ __forceinline__ void get(const type& v, double (&o)[8]) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      o[2 * k] = (double)__uint_as_float(w[k] << 16);
      o[2 * k + 1] = (double)__uint_as_float(w[k] & 0xffff0000u);
    }
  }
};

// P2: partial scores of one item (row tile x column chunk k): thread rows
// i .. i + VEC - 1, columns of the chunk in order.
template <class T>
__device__ void xr_item(const Fit& f, const T* X, int tile, int k, const double* zs,
                        double* rts) {
  constexpr int VN = Vec16<T>::N;
  const int c0 = k * f.cc;
  const int cols = min(f.cc, f.p - c0);
  __syncthreads();
  // rt = (S z) / scale for the chunk's columns (S is not deflated until P7)
  for (int j = threadIdx.x; j < cols; j += PT) {
    double rv = 0.0;
    for (int c = 0; c < f.m; ++c) rv = fma(__ldcg(f.S + c0 + j + (long)c * f.p), zs[c], rv);
    rts[j] = rv / f.scale[c0 + j];
  }
  __syncthreads();
  const int vec = f.vec;  // VN or 1
  const int rows_tile = PT * vec;
  const int i = tile * rows_tile + threadIdx.x * vec;
  if (i >= f.n) return;
  double* out = f.tpart + (long)k * f.n;
  const T* base = X + (long)c0 * f.ld + i;
  if (vec == VN && i + VN <= f.n) {
    using V = typename Vec16<T>::type;
    double acc[VN];
#pragma unroll
    for (int u = 0; u < VN; ++u) acc[u] = 0.0;
    int j = 0;
    for (; j + 7 < cols; j += 8) {
      V x[8];
#pragma unroll
      for (int u = 0; u < 8; ++u)
        x[u] = __ldg(reinterpret_cast<const V*>(base + (long)(j + u) * f.ld));
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        double e[VN];
        Vec16<T>::get(x[u], e);
        const double w = rts[j + u];
#pragma unroll
        for (int q = 0; q < VN; ++q) acc[q] = fma(e[q], w, acc[q]);
      }
    }
    for (; j < cols; ++j) {
      double e[VN];
      Vec16<T>::get(__ldg(reinterpret_cast<const V*>(base + (long)j * f.ld)), e);
      const double w = rts[j];
#pragma unroll
      for (int q = 0; q < VN; ++q) acc[q] = fma(e[q], w, acc[q]);
    }
#pragma unroll
    for (int q = 0; q < VN; ++q) out[i + q] = acc[q];
  } else {
    // scalar rows (unaligned storage, or the last rows of X)
    const int cnt = min(vec, f.n - i);
    for (int q = 0; q < cnt; ++q) {
      double acc = 0.0;
      for (int j = 0; j < cols; ++j) acc = fma(as_f64(base[q + (long)j * f.ld]), rts[j], acc);
      out[i + q] = acc;
    }
  }
}

// Eight consecutive rows of a column as FP64 (16-byte aligned source): one
// 16-byte load for BF16, two for FP32, four for FP64.
template <class T> struct Oct;
template <> struct Oct<bf16> {
  static __device__ __forceinline__ void load(const bf16* p, double (&x)[8]) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x[2 * k] = (double)__uint_as_float(w[k] << 16);
      x[2 * k + 1] = (double)__uint_as_float(w[k] & 0xffff0000u);
    }
  }
};
template <> struct Oct<float> {
  static __device__ __forceinline__ void load(const float* p, double (&x)[8]) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
  }
};
template <> struct Oct<double> {
  static __device__ __forceinline__ void load(const double* p, double (&x)[8]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double2 v = __ldg(reinterpret_cast<const double2*>(p) + k);
      x[2 * k] = v.x;
      x[2 * k + 1] = v.y;
    }
  }
};

// P4: loading partials of one item (row chunk kc x 32 columns from jt*32).
// Warp w owns columns w, w + 8, w + 16, w + 24 of the tile and walks them
// together; lane l takes the row octets l, l + 32, ... (8 consecutive rows
// per load, in row order), then the leftover rows one per lane; the t rows
// are staged in shared memory. The summation order depends only on the
// row count, so it is the same for every storage type.
template <class T>
__device__ void xtv_item(const Fit& f, const T* X, int kc, int jt, const double* tcol,
                         double* ts) {
  const int r0 = kc * f.rc;
  const int rows = min(f.rc, f.n - r0);
  __syncthreads();
  for (int r = threadIdx.x; r < rows; r += PT) ts[r] = __ldcg(tcol + r0 + r);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T* col[4];
  bool ok[4];
  double acc[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int j = jt * 32 + warp + 8 * c;
    ok[c] = j < f.p;
    col[c] = X + (long)(ok[c] ? j : 0) * f.ld + r0;
    acc[c] = 0.0;
  }
  const int octs = f.oct ? rows >> 3 : 0;
  for (int o = lane; o < octs; o += 32) {
    const double* tv = ts + 8 * o;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (!ok[c]) continue;
      double x[8];
      Oct<T>::load(col[c] + 8 * o, x);
#pragma unroll
      for (int e = 0; e < 8; ++e) acc[c] = fma(x[e], tv[e], acc[c]);
    }
  }
  for (int r = 8 * octs + lane; r < rows; r += 32) {
    const double tv = ts[r];
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (ok[c]) acc[c] = fma(as_f64(col[c][r]), tv, acc[c]);
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double v = warp_sum(acc[c]);
    if (lane == 0 && ok[c]) f.ppart[(long)kc * f.p + jt * 32 + warp + 8 * c] = v;
  }
}

// Dominant eigenpair of the packed m x m Gram (whole CTA): zs = s z / sqrt(lambda),
// sign fixed so the largest |z| entry is positive (as direction_kernel).
__device__ void direction_step(const Fit& f, double* sm, int* flag) {
  const int m = f.m;
  double* A = sm;
  double* E = sm + m * m;
  for (int c = threadIdx.x; c < m; c += blockDim.x)
    for (int d = 0; d <= c; ++d) {
      const double v = __ldcg(f.gpk + c * (c + 1) / 2 + d);
      A[c + d * m] = v;
      A[d + c * m] = v;
    }
  __syncthreads();
  jacobi_eigen(A, E, m);
  __syncthreads();
  if (threadIdx.x == 0) {
    int best = 0;
    for (int k = 1; k < m; ++k)
      if (A[k + k * m] > A[best + best * m]) best = k;
    const double lam = A[best + best * m];
    const bool ok = lam > 0.0 && isfinite(lam);
    if (!ok) flag_error(flag, 1);
    const double inv = ok ? 1.0 / sqrt(lam) : 0.0;
    int arg = 0;
    for (int k = 1; k < m; ++k)
      if (fabs(E[k + best * m]) > fabs(E[arg + best * m])) arg = k;
    const double sgn = E[arg + best * m] < 0.0 ? -1.0 : 1.0;
    for (int k = 0; k < m; ++k) f.scal[SC_Z + k] = sgn * E[k + best * m] * inv;
  }
  __syncthreads();
}

// Over this CTA's columns [j0, j1): when a >= 0, V[:, a] = v / |v| and the
// deflation S -= V[:, a] (S^T v / |v|)^T; then the partials of the Gram of S
// (slots 0 .. G-1, packed lower triangle) and of u = S^T (mean / scale)
// (slots G .. G+m-1) into the CTA's partial row. Whole CTA.
__device__ void gram_u_partials(const Fit& f, int cta, int j0, int j1, int a, double inv_v,
                                const double* sv, double* sm) {
  const int m = f.m, p = f.p;
  const int G = m * (m + 1) / 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* ss = sm;                                        // kGramRows x m
  double* gacc = sm + kGramRows * kPersistMaxResponses;   // G + m running sums (warp-owned)
  double* wsc = gacc + 640;                               // kGramRows mean / scale
  __syncthreads();
  for (int k = threadIdx.x; k < G + m; k += PT) gacc[k] = 0.0;
  for (int g0 = j0; g0 < j1; g0 += kGramRows) {
    const int rows = min(kGramRows, j1 - g0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < rows * m; idx += PT) {
      const int jl = idx % rows, c = idx / rows;
      const int j = g0 + jl;
      double sval = __ldcg(f.S + j + (long)c * p);
      if (a >= 0) {
        const double vj = __ldcg(f.v + j) * inv_v;
        if (c == 0) f.V[j + (long)a * p] = vj;
        sval = fma(-vj, sv[c] * inv_v, sval);
        f.S[j + (long)c * p] = sval;
      }
      ss[jl + c * kGramRows] = sval;
      if (c == 0) wsc[jl] = f.mean[j] / f.scale[j];
    }
    __syncthreads();
    for (int k = warp; k < G + m; k += PT / 32) {
      double s = 0.0;
      if (k < G) {
        int c = (int)((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
        while (c * (c + 1) / 2 > k) --c;
        while ((c + 1) * (c + 2) / 2 <= k) ++c;
        const int d = k - c * (c + 1) / 2;
        for (int jl = lane; jl < rows; jl += 32)
          s = fma(ss[jl + c * kGramRows], ss[jl + d * kGramRows], s);
      } else {
        const int c = k - G;
        for (int jl = lane; jl < rows; jl += 32) s = fma(ss[jl + c * kGramRows], wsc[jl], s);
      }
      s = warp_sum(s);
      if (lane == 0) gacc[k] += s;
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < G + m; k += PT) f.cpart[(long)cta * f.cslots + k] = gacc[k];
}

template <class T>
__global__ void __launch_bounds__(PT, 3)
    persistent_simpls(const Fit* __restrict__ fits, int nfits) {
  extern __shared__ double psm[];
  __shared__ double red[32];
  __shared__ double zs[kPersistMaxResponses];
  __shared__ double hs[kPersistMaxComponents];
  __shared__ double sv[kPersistMaxResponses];
  __shared__ double scal_s[4];
  int fi = 0;
  while (fi + 1 < nfits && (int)blockIdx.x >= fits[fi + 1].cta0) ++fi;
  const Fit f = fits[fi];
  int* const flag = f.flag;
  const int cta = (int)blockIdx.x - f.cta0;
  if (cta == f.absent_cta) return;  // bounded-wait test only
  const T* X = static_cast<const T*>(f.X);
  const int n = f.n, p = f.p, m = f.m, C = f.C;
  const int tid = threadIdx.x;
  int j0, j1;
  col_range(p, C, cta, j0, j1);

  __shared__ int item_s;
  const int G = m * (m + 1) / 2;
  // partials of the Gram of S and of u = S^T (mean / scale) over this CTA's
  // columns, before the first component (S = S0)
  gram_u_partials(f, cta, j0, j1, -1, 0.0, sv, psm);
  for (int a = 0; a < f.a; ++a) {
    // B0: Gram and u of the (deflated) S, the direction z / sqrt(lambda), and
    // the score offset c = mean . (S z / scale) = z . u
    if (!group_sync(f, flag, [&] {
          reduce_slots(f, G + m, [&](int k, double v) {
            if (k < G) f.gpk[k] = v;
            else f.scal[SC_U + k - G] = v;
          });
          __syncthreads();
          __threadfence();
          direction_step(f, psm, flag);
          if (tid == 0) {
            double cz = 0.0;
            for (int c = 0; c < m; ++c) cz = fma(f.scal[SC_Z + c], __ldcg(f.scal + SC_U + c), cz);
            f.scal[SC_C] = cz;
            atomicExch(f.bar + 2, 0u);  // item counter of the score pass
          }
        }))
      return;
    for (int c = tid; c < m; c += PT) zs[c] = __ldcg(f.scal + SC_Z + c);
    __syncthreads();
    // P2: score partials, items (row tile, column chunk) claimed in order
    {
      const int tiles = (n + PT * f.vec - 1) / (PT * f.vec);
      const int items = tiles * f.kt;
      for (;;) {
        if (tid == 0) item_s = (int)atomicAdd(f.bar + 2, 1u);
        __syncthreads();
        const int it = item_s;
        if (it >= items) break;
        xr_item<T>(f, X, it % tiles, it / tiles, zs, psm);
      }
    }
    if (!group_sync(f, flag, [] {})) return;
    // P3: t = sum of the chunk partials - c; |t|^2 and sum t
    {
      const double cc = __ldcg(f.scal + SC_C);
      double* tcol = f.T + (long)a * n;
      double s2 = 0.0, s1 = 0.0;
      for (int i = cta * PT + tid; i < n; i += C * PT) {
        // eight interleaved partial sums (more loads in flight), fixed order
        double q[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) q[u] = 0.0;
        int k = 0;
        for (; k + 7 < f.kt; k += 8) {
#pragma unroll
          for (int u = 0; u < 8; ++u) q[u] += __ldcg(f.tpart + (long)(k + u) * n + i);
        }
        for (; k < f.kt; ++k) q[0] += __ldcg(f.tpart + (long)k * n + i);
        const double t = (((q[0] + q[1]) + (q[2] + q[3])) + ((q[4] + q[5]) + (q[6] + q[7]))) - cc;
        tcol[i] = t;
        s2 = fma(t, t, s2);
        s1 += t;
      }
      s2 = cta_sum(s2, red);
      s1 = cta_sum(s1, red);
      if (tid == 0) {
        f.cpart[(long)cta * f.cslots] = s2;
        f.cpart[(long)cta * f.cslots + 1] = s1;
      }
    }
    if (!group_sync(f, flag, [&] {
          reduce_slots(f, 2, [&](int k, double v) { f.scal[k == 0 ? SC_T2 : SC_ST] = v; });
          if (tid == 0) atomicExch(f.bar + 3, 0u);  // item counter of the loading pass
        }))
      return;
    // P4: loading partials, items (row chunk, 32-column tile) claimed in order
    {
      const int jtiles = (p + 31) / 32;
      const int items = jtiles * f.kp;
      const double* tcol = f.T + (long)a * n;
      for (;;) {
        if (tid == 0) item_s = (int)atomicAdd(f.bar + 3, 1u);
        __syncthreads();
        const int it = item_s;
        if (it >= items) break;
        xtv_item<T>(f, X, it % f.kp, it / f.kp, tcol, psm);
      }
    }
    if (!group_sync(f, flag, [] {})) return;
    // P5: p, R[:, a] = (S z) / |t|; partial V^T p (a) and S0^T R[:, a] (m)
    if (tid == 0) {
      const double t2 = __ldcg(f.scal + SC_T2);
      const double tn = sqrt(t2);
      const bool ok = tn > 0.0 && isfinite(tn);
      if (!ok && cta == 0) flag_error(flag, 1);
      scal_s[0] = ok ? 1.0 / tn : 0.0;
      scal_s[1] = __ldcg(f.scal + SC_ST);
    }
    __syncthreads();
    const double inv_t = scal_s[0], sum_t = scal_s[1];
    double* ps = psm;          // p values of this CTA's columns (<= 2048)
    double* rs = psm + 2048;   // R values
    for (int jl = tid; jl < j1 - j0; jl += PT) {
      const int j = j0 + jl;
      double q0 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0;
      int k = 0;
      for (; k + 3 < f.kp; k += 4) {
        q0 += __ldcg(f.ppart + (long)k * p + j);
        q1 += __ldcg(f.ppart + (long)(k + 1) * p + j);
        q2 += __ldcg(f.ppart + (long)(k + 2) * p + j);
        q3 += __ldcg(f.ppart + (long)(k + 3) * p + j);
      }
      for (; k < f.kp; ++k) q0 += __ldcg(f.ppart + (long)k * p + j);
      const double pr = (q0 + q1) + (q2 + q3);
      double rv = 0.0;
      for (int c = 0; c < m; ++c) rv = fma(__ldcg(f.S + j + (long)c * p), zs[c], rv);
      const double pj = (pr - f.mean[j] * sum_t) / f.scale[j] * inv_t;
      const double rj = rv * inv_t;
      f.pv[j] = pj;
      f.R[j + (long)a * p] = rj;
      ps[jl] = pj;
      rs[jl] = rj;
    }
    __syncthreads();
    {
      const int lane = tid & 31, warp = tid >> 5;
      const int cols = j1 - j0;
      for (int k = warp; k < a + m; k += PT / 32) {
        double s = 0.0;
        if (k < a) {
          const double* vk = f.V + (long)k * p + j0;
          for (int jl = lane; jl < cols; jl += 32) s = fma(__ldcg(vk + jl), ps[jl], s);
        } else {
          const double* sk = f.S0 + (long)(k - a) * p + j0;
          for (int jl = lane; jl < cols; jl += 32) s = fma(sk[jl], rs[jl], s);
        }
        s = warp_sum(s);
        if (lane == 0) f.cpart[(long)cta * f.cslots + k] = s;
      }
    }
    if (!group_sync(f, flag, [&] {
          reduce_slots(f, a + m, [&](int k, double v) {
            if (k < a) {
              f.scal[SC_H + k] = v;
            } else {
              f.scal[SC_Q + k - a] = v;
              f.Q[(k - a) + (long)a * m] = v;
            }
          });
        }))
      return;
    // P6: v = p - V h; partial v.v and S^T v
    for (int k = tid; k < a; k += PT) hs[k] = __ldcg(f.scal + SC_H + k);
    __syncthreads();
    double* vs = psm;  // v of this CTA's columns
    double vvp = 0.0;
    for (int jl = tid; jl < j1 - j0; jl += PT) {
      const int j = j0 + jl;
      double vj = __ldcg(f.pv + j);
#pragma unroll 4
      for (int k = 0; k < a; ++k) vj = fma(-__ldcg(f.V + j + (long)k * p), hs[k], vj);
      f.v[j] = vj;
      vs[jl] = vj;
      vvp = fma(vj, vj, vvp);
    }
    vvp = cta_sum(vvp, red);  // (synchronises: vs complete)
    {
      const int lane = tid & 31, warp = tid >> 5;
      const int cols = j1 - j0;
      for (int c = warp; c < m; c += PT / 32) {
        const double* sc = f.S + (long)c * p + j0;
        double s = 0.0;
        for (int jl = lane; jl < cols; jl += 32) s = fma(__ldcg(sc + jl), vs[jl], s);
        s = warp_sum(s);
        if (lane == 0) f.cpart[(long)cta * f.cslots + 1 + c] = s;
      }
      if (tid == 0) f.cpart[(long)cta * f.cslots] = vvp;
    }
    if (!group_sync(f, flag, [&] {
          reduce_slots(f, 1 + m, [&](int k, double v) {
            if (k == 0) f.scal[SC_VV] = v;
            else f.scal[SC_SV + k - 1] = v;
          });
        }))
      return;
    // P7: V[:, a], deflate S, partials of the Gram and u of the deflated S;
    // T[:, a] /= |t|
    if (tid == 0) {
      const double vn = sqrt(__ldcg(f.scal + SC_VV));
      const bool ok = vn > 0.0 && isfinite(vn);
      if (!ok && cta == 0) flag_error(flag, 1);
      scal_s[2] = ok ? 1.0 / vn : 0.0;
    }
    for (int c = tid; c < m; c += PT) sv[c] = __ldcg(f.scal + SC_SV + c);
    __syncthreads();
    gram_u_partials(f, cta, j0, j1, a, scal_s[2], sv, psm);
    double* tcol = f.T + (long)a * n;
    for (int i = cta * PT + tid; i < n; i += C * PT) tcol[i] = __ldcg(tcol + i) * inv_t;
  }
}

int round_up(long v, long m) { return (int)((v + m - 1) / m * m); }

}  // namespace

int& persistent_enabled() {
  static int on = 1;
  return on;
}

bool persistent_supported(int m, int a) {
  return m >= 1 && m <= kPersistMaxResponses && a >= 1 && a <= kPersistMaxComponents;
}

PersistentWaitTest& persistent_wait_test() {
  static PersistentWaitTest t;
  return t;
}

std::unique_ptr<PersistentPlan>*& persistent_deferral() {
  thread_local std::unique_ptr<PersistentPlan>* sink = nullptr;
  return sink;
}

int persistent_ctas(int n, int p) {
  // from (n, p) only, never from the storage type: at most three per SM
  const long elems = (long)n * p;
  return (int)std::max(1L, std::min<long>(3L * num_sms(), (elems + (1L << 17) - 1) >> 17));
}

namespace {

template <class T>
int capacity_of() {
  static const int cap = [] {
    int v = 0, coop = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
        cudaFuncSetAttribute(persistent_simpls<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmemDoubles * (int)sizeof(double)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, persistent_simpls<T>, PT,
                                                      kSmemDoubles * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    return v >= 3 ? v * num_sms() : 0;
  }();
  return cap;
}

}  // namespace

int persistent_capacity(int elem) {
  return elem == 2 ? capacity_of<bf16>() : elem == 4 ? capacity_of<float>() : capacity_of<double>();
}

template <class T>
bool plan_simpls_persistent(const T* X, int n, int p, long ld, int m, int a, DeviceModel& model,
                            DeviceArray<double>& S, double* gpk, Workspace& ws, cudaStream_t stream,
                            PersistentPlan& plan) {
  if (!persistent_enabled() || !persistent_supported(m, a) || n < 2 || p < 1) return false;
  // Large fits take the per-kernel loop: its streaming kernels keep more
  // loads in flight (many CTAs per SM) and a component's two passes over X
  // dwarf its launch latency; the persistent launch pays off where the
  // passes are short and the per-component launches dominate.
  if ((long)n * p > kPersistMaxElements) return false;
  const int C = persistent_ctas(n, p);
  const int cap = capacity_of<T>();
  if (cap == 0 || C > cap) return false;
  // per-CTA column ranges must fit the shared staging of P5/P6 (2048 each)
  if ((p + C - 1) / C > 2048) return false;

  Fit& f = plan.fit;
  f = Fit{};
  f.X = X;
  f.ld = ld;
  f.n = n;
  f.p = p;
  f.m = m;
  f.a = a;
  f.mean = model.mean.get();
  f.scale = model.scale.get();
  f.S0 = model.S0.get();
  f.R = model.R.get();
  f.V = model.V.get();
  f.Q = model.Q.get();
  f.T = model.T.get();
  f.gpk = gpk;
  f.pv = ws.vec_p[2].get();
  f.v = ws.vec_p[3].get();
  f.flag = ws.flag.get();
  f.C = C;
  // t pass: chunks of columns so that (row tiles of 1024) x chunks gives
  // about four items per CTA; loading pass: 32-column tiles x row chunks
  const int target = 4 * C;
  const long row_tiles = (n + 1023) / 1024;
  f.cc = std::max(32, std::min(kMaxXrCols, round_up((p * row_tiles + target - 1) / target, 32)));
  f.kt = (p + f.cc - 1) / f.cc;
  const int jtiles = (p + 31) / 32;
  int kp = std::max((target + jtiles - 1) / jtiles, (n + kMaxXtvRows - 1) / kMaxXtvRows);
  kp = std::max(1, std::min(kp, (n + 63) / 64));
  f.rc = std::min(kMaxXtvRows, round_up((n + kp - 1) / kp, 64));
  f.kp = (n + f.rc - 1) / f.rc;
  constexpr int VN = sizeof(T) == 2 ? 8 : (sizeof(T) == 4 ? 4 : 2);
  const bool aligned16 = reinterpret_cast<uintptr_t>(X) % 16 == 0 && ld % VN == 0;
  f.vec = aligned16 ? VN : 1;
  // octet loads in the loading pass: the same condition for every storage
  // type (so BF16 and FP32 storage of the same values sum in one order)
  f.oct = (reinterpret_cast<uintptr_t>(X) % 16 == 0 && ld % 8 == 0) ? 1 : 0;
  f.cslots = std::max(a + m, std::max(1 + m, m * (m + 1) / 2 + m));
  const PersistentWaitTest& wt = persistent_wait_test();
  f.barrier_cycles = wt.cycles > 0 ? wt.cycles : kBarrierCycles;
  f.absent_cta = wt.absent ? 0 : -1;

  // scratch of this fit (stream-ordered, freed behind the launch); the
  // kernel forms the Gram of S itself (into gpk) before the first component
  plan.elem = (int)sizeof(T);
  plan.S = std::move(S);
  f.S = plan.S.get();
  plan.part.allocate((size_t)f.kt * n + (size_t)f.kp * p, stream);
  f.tpart = plan.part.get();
  f.ppart = f.tpart + (size_t)f.kt * n;
  plan.cpart.allocate((size_t)C * f.cslots, stream);
  plan.scal.allocate((size_t)SC_H + kPersistMaxComponents + 8, stream);
  plan.bar.allocate(4, stream);
  plan.bar.zero(stream);
  f.cpart = plan.cpart.get();
  f.scal = plan.scal.get();
  f.bar = plan.bar.get();
  model.a = a;
  return true;
}

void launch_persistent(const std::vector<PersistentPlan*>& plans, cudaStream_t stream) {
  if (plans.empty()) return;
  const int elem = plans[0]->elem;
  std::vector<Fit> fits;
  int total = 0;
  for (PersistentPlan* pl : plans) {
    require(pl->elem == elem, "one persistent launch takes one storage type");
    Fit f = pl->fit;
    f.cta0 = total;
    total += f.C;
    fits.push_back(f);
  }
  require(total <= persistent_capacity(elem), "persistent launch exceeds the co-resident CTAs");
  DeviceArray<Fit> d_fits(fits.size(), stream);
  FPLS_CHECK(cudaMemcpyAsync(d_fits.get(), fits.data(), sizeof(Fit) * fits.size(),
                             cudaMemcpyHostToDevice, stream));
  const Fit* fp = d_fits.get();
  int nfits = (int)fits.size();
  void* args[] = {(void*)&fp, (void*)&nfits};
  const void* fn = elem == 2 ? (const void*)persistent_simpls<bf16>
                 : elem == 4 ? (const void*)persistent_simpls<float>
                             : (const void*)persistent_simpls<double>;
  FPLS_CHECK(cudaLaunchCooperativeKernel(fn, dim3(total), dim3(PT), args,
                                         kSmemDoubles * sizeof(double), stream));
  count_launch();
  FPLS_LAUNCH("persistent_simpls");
  // the descriptors are freed stream-ordered, behind the launch
}

template bool plan_simpls_persistent<float>(const float*, int, int, long, int, int, DeviceModel&,
                                            DeviceArray<double>&, double*, Workspace&, cudaStream_t,
                                            PersistentPlan&);
template bool plan_simpls_persistent<double>(const double*, int, int, long, int, int, DeviceModel&,
                                             DeviceArray<double>&, double*, Workspace&, cudaStream_t,
                                             PersistentPlan&);
template bool plan_simpls_persistent<bf16>(const bf16*, int, int, long, int, int, DeviceModel&,
                                           DeviceArray<double>&, double*, Workspace&, cudaStream_t,
                                           PersistentPlan&);

}  // namespace fpls
