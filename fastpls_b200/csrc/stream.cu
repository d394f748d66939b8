// HBM-streaming kernels over the resident predictor matrix X (n x p,
// column-major, BF16, FP32 or FP64 storage, FP64 arithmetic).
//
// These are the GEMV-shaped steps of a single fit: the column moments
// (centre, scale, X^T Yc) in one pass, t = X r (scores) and p = X^T t
// (loadings). Each reads X exactly once per call with coalesced, unrolled
// loads (many independent loads in flight per warp) and reduces in a fixed
// order through per-chunk partials, so results are deterministic.
// Algorithmic bytes per call: n * p * sizeof(T) (+ O((n + p) * nb * 8)).
#include "common.cuh"
#include "kernels.cuh"

#include <algorithm>

namespace fpls {

namespace {

constexpr int kThreads = 256;

// Two consecutive rows of one column in one load (bf16x2, float2, double2):
// 4-16 bytes per lane, 128-512 bytes per warp request. Used when the column
// stride is even and X is aligned to the pair size.
template <class T> struct Pair;
template <> struct Pair<float> {
  using type = float2;
  static __device__ __forceinline__ double lo(type v) { return v.x; }
  static __device__ __forceinline__ double hi(type v) { return v.y; }
};
template <> struct Pair<double> {
  using type = double2;
  static __device__ __forceinline__ double lo(type v) { return v.x; }
  static __device__ __forceinline__ double hi(type v) { return v.y; }
};
template <> struct Pair<bf16> {
  using type = __nv_bfloat162;
  static __device__ __forceinline__ double lo(type v) { return __low2float(v); }
  static __device__ __forceinline__ double hi(type v) { return __high2float(v); }
};

template <class T>
bool pair_aligned(const T* X, long ld) {
  return ld % 2 == 0 && reinterpret_cast<uintptr_t>(X) % (2 * sizeof(T)) == 0;
}

// ---------------------------------------------------------------------------
// X^T V (and optionally column sums / sums of squares) -- warp per column.
// Block = 8 warps over a tile of 32 columns and a chunk of `rc` rows whose
// V rows are staged in shared memory. partial layout: [chunk][j][slot] with
// slots = nb (+2 when MOMENTS: sum, sumsq at slots nb, nb+1).
// ---------------------------------------------------------------------------
template <class T, int MB, bool MOMENTS>
__global__ void __launch_bounds__(kThreads)
    xtv_kernel(const T* __restrict__ X, int n, int p, long ld,
               const double* __restrict__ V, long ldv, int nb, int rc,
               double* __restrict__ partial) {
  extern __shared__ double vs[];  // rc x nb
  const int chunk = blockIdx.y;
  const int r0 = chunk * rc;
  const int rows = min(rc, n - r0);
  for (int idx = threadIdx.x; idx < rows * nb; idx += blockDim.x) {
    const int r = idx % rows, c = idx / rows;
    vs[r + c * rc] = V[(r0 + r) + (long)c * ldv];
  }
  __syncthreads();
  const int slots = nb + (MOMENTS ? 2 : 0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int jj = warp; jj < 32; jj += kThreads / 32) {
    const int j = blockIdx.x * 32 + jj;
    if (j >= p) break;
    const T* col = X + (long)j * ld + r0;
    double acc[MB > 0 ? MB : 1];
#pragma unroll
    for (int c = 0; c < (MB > 0 ? MB : 1); ++c) acc[c] = 0.0;
    double s = 0.0, ss = 0.0;
    int r = lane;
    for (; r + 96 < rows; r += 128) {
      double x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) x[u] = as_f64(col[r + 32 * u]);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (MOMENTS) {
          s += x[u];
          ss = fma(x[u], x[u], ss);
        }
#pragma unroll
        for (int c = 0; c < MB; ++c)
          if (c < nb) acc[c] = fma(x[u], vs[r + 32 * u + c * rc], acc[c]);
      }
    }
    for (; r < rows; r += 32) {
      const double x = as_f64(col[r]);
      if (MOMENTS) {
        s += x;
        ss = fma(x, x, ss);
      }
#pragma unroll
      for (int c = 0; c < MB; ++c)
        if (c < nb) acc[c] = fma(x, vs[r + c * rc], acc[c]);
    }
    double* out = partial + ((long)chunk * p + j) * slots;
#pragma unroll
    for (int c = 0; c < MB; ++c) {
      if (c < nb) {
        const double v = warp_sum(acc[c]);
        if (lane == 0) out[c] = v;
      }
    }
    if (MOMENTS) {
      s = warp_sum(s);
      ss = warp_sum(ss);
      if (lane == 0) {
        out[nb] = s;
        out[nb + 1] = ss;
      }
    }
  }
}

// Same contract as xtv_kernel, with each lane reading row pairs: lane l takes
// rows 2(l + 32u) and 2(l + 32u) + 1 of the chunk (rc even, column stride even).
template <class T, int MB, bool MOMENTS>
__global__ void __launch_bounds__(kThreads)
    xtv_pair_kernel(const T* __restrict__ X, int n, int p, long ld,
                    const double* __restrict__ V, long ldv, int nb, int rc,
                    double* __restrict__ partial) {
  using P = Pair<T>;
  using T2 = typename P::type;
  extern __shared__ double vs[];  // rc x nb
  const int chunk = blockIdx.y;
  const int r0 = chunk * rc;
  const int rows = min(rc, n - r0);
  for (int idx = threadIdx.x; idx < rows * nb; idx += blockDim.x) {
    const int r = idx % rows, c = idx / rows;
    vs[r + c * rc] = V[(r0 + r) + (long)c * ldv];
  }
  __syncthreads();
  const int slots = nb + (MOMENTS ? 2 : 0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pairs = rows >> 1;
  for (int jj = warp; jj < 32; jj += kThreads / 32) {
    const int j = blockIdx.x * 32 + jj;
    if (j >= p) break;
    const T* col = X + (long)j * ld + r0;
    const T2* col2 = reinterpret_cast<const T2*>(col);
    double acc[MB > 0 ? MB : 1];
#pragma unroll
    for (int c = 0; c < (MB > 0 ? MB : 1); ++c) acc[c] = 0.0;
    double s = 0.0, ss = 0.0;
    int q = lane;
    for (; q + 96 < pairs; q += 128) {
      T2 x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) x[u] = col2[q + 32 * u];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double a = P::lo(x[u]), b = P::hi(x[u]);
        const int r = 2 * (q + 32 * u);
        if (MOMENTS) {
          s += a;
          ss = fma(a, a, ss);
          s += b;
          ss = fma(b, b, ss);
        }
#pragma unroll
        for (int c = 0; c < MB; ++c)
          if (c < nb) {
            const double2 v = *reinterpret_cast<const double2*>(vs + r + c * rc);
            acc[c] = fma(a, v.x, acc[c]);
            acc[c] = fma(b, v.y, acc[c]);
          }
      }
    }
    for (; q < pairs; q += 32) {
      const T2 x = col2[q];
      const double a = P::lo(x), b = P::hi(x);
      const int r = 2 * q;
      if (MOMENTS) {
        s += a;
        ss = fma(a, a, ss);
        s += b;
        ss = fma(b, b, ss);
      }
#pragma unroll
      for (int c = 0; c < MB; ++c)
        if (c < nb) {
          const double2 v = *reinterpret_cast<const double2*>(vs + r + c * rc);
          acc[c] = fma(a, v.x, acc[c]);
          acc[c] = fma(b, v.y, acc[c]);
        }
    }
    if ((rows & 1) && lane == 0) {  // odd last row of the final chunk
      const int r = rows - 1;
      const double a = as_f64(col[r]);
      if (MOMENTS) {
        s += a;
        ss = fma(a, a, ss);
      }
#pragma unroll
      for (int c = 0; c < MB; ++c)
        if (c < nb) acc[c] = fma(a, vs[r + c * rc], acc[c]);
    }
    double* out = partial + ((long)chunk * p + j) * slots;
#pragma unroll
    for (int c = 0; c < MB; ++c) {
      if (c < nb) {
        const double v = warp_sum(acc[c]);
        if (lane == 0) out[c] = v;
      }
    }
    if (MOMENTS) {
      s = warp_sum(s);
      ss = warp_sum(ss);
      if (lane == 0) {
        out[nb] = s;
        out[nb + 1] = ss;
      }
    }
  }
}

// Sum the per-chunk partials: out_c[j] (+ c*ldo) for each slot c < nb, and
// the moment slots into sum/sumsq.
__global__ void xtv_finish(const double* __restrict__ partial, int chunks,
                           int p, int nb, int slots, double* out, long ldo,
                           double* sum, double* sumsq) {
  const long total = (long)p * slots;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int j = (int)(idx / slots), c = (int)(idx % slots);
    double v = 0.0;
    for (int k = 0; k < chunks; ++k) v += partial[((long)k * p + j) * slots + c];
    if (c < nb) out[j + (long)c * ldo] = v;
    else if (c == nb) sum[j] = v;
    else sumsq[j] = v;
  }
}

template <class T, int MB, bool MOMENTS>
void xtv_launch(const T* X, int n, int p, long ld, const double* V, long ldv,
                int nb, double* out, long ldo, double* sum, double* sumsq,
                DeviceArray<double>& scratch, cudaStream_t stream) {
  // rows per chunk: keep the staged V block <= 64 KB and give the grid
  // enough blocks to cover every SM several times.
  int rc = 2048;
  if (nb > 0) rc = std::min(rc, std::max(128, (64 * 1024 / 8) / nb / 64 * 64));
  const int col_tiles = (int)ceil_div(p, 32);
  int chunks = (int)ceil_div(n, rc);
  const int want = 6 * num_sms();
  if (col_tiles * chunks < want && n > 256) {
    const int target = std::min((int)ceil_div(n, 256), (int)ceil_div(want, col_tiles));
    if (target > chunks) {
      rc = std::max(256, (int)ceil_div(n, target));
      rc = (rc + 127) / 128 * 128;
      chunks = (int)ceil_div(n, rc);
    }
  }
  const int slots = nb + (MOMENTS ? 2 : 0);
  scratch.reserve((size_t)chunks * p * slots, stream);
  const size_t smem = (size_t)rc * std::max(nb, 1) * sizeof(double);
  if (pair_aligned(X, ld)) {
    if (smem > 48 * 1024)
      FPLS_CHECK(cudaFuncSetAttribute(xtv_pair_kernel<T, MB, MOMENTS>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    xtv_pair_kernel<T, MB, MOMENTS><<<dim3(col_tiles, chunks), kThreads, smem, stream>>>(
        X, n, p, ld, V, ldv, nb, rc, scratch.get());
  } else {
    if (smem > 48 * 1024)
      FPLS_CHECK(cudaFuncSetAttribute(xtv_kernel<T, MB, MOMENTS>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    xtv_kernel<T, MB, MOMENTS><<<dim3(col_tiles, chunks), kThreads, smem, stream>>>(
        X, n, p, ld, V, ldv, nb, rc, scratch.get());
  }
  count_launch();
  FPLS_LAUNCH("xtv_kernel");
  const long total = (long)p * slots;
  const unsigned blocks = (unsigned)std::min<long>((total + 255) / 256, 8L * num_sms());
  xtv_finish<<<blocks, 256, 0, stream>>>(scratch.get(), chunks, p, nb, slots,
                                         out, ldo, sum, sumsq);
  count_launch();
  FPLS_LAUNCH("xtv_finish");
}

template <class T, bool MOMENTS>
void xtv_dispatch(const T* X, int n, int p, long ld, const double* V, long ldv,
                  int nb, double* out, long ldo, double* sum, double* sumsq,
                  DeviceArray<double>& scratch, cudaStream_t stream) {
  if (nb == 0) xtv_launch<T, 0, MOMENTS>(X, n, p, ld, V, ldv, nb, out, ldo, sum, sumsq, scratch, stream);
  else if (nb <= 1) xtv_launch<T, 1, MOMENTS>(X, n, p, ld, V, ldv, nb, out, ldo, sum, sumsq, scratch, stream);
  else if (nb <= 4) xtv_launch<T, 4, MOMENTS>(X, n, p, ld, V, ldv, nb, out, ldo, sum, sumsq, scratch, stream);
  else if (nb <= 8) xtv_launch<T, 8, MOMENTS>(X, n, p, ld, V, ldv, nb, out, ldo, sum, sumsq, scratch, stream);
  else if (nb <= 16) xtv_launch<T, 16, MOMENTS>(X, n, p, ld, V, ldv, nb, out, ldo, sum, sumsq, scratch, stream);
  else xtv_launch<T, 32, MOMENTS>(X, n, p, ld, V, ldv, nb, out, ldo, sum, sumsq, scratch, stream);
}

// ---------------------------------------------------------------------------
// X R - offset: thread per row pair, block over 512 rows x a column chunk.
// partial layout: [chunk][c][row] (column-major per chunk, ld = n).
// ---------------------------------------------------------------------------
template <class T, int NB>
__global__ void __launch_bounds__(kThreads)
    xr_kernel(const T* __restrict__ X, int n, int p, long ld,
              const double* __restrict__ R, long ldr, int nb, int cc,
              double* __restrict__ partial) {
  extern __shared__ double rs[];  // cc x NB
  const int chunk = blockIdx.y;
  const int c0 = chunk * cc;
  const int cols = min(cc, p - c0);
  for (int idx = threadIdx.x; idx < cols * NB; idx += blockDim.x) {
    const int j = idx / NB, c = idx % NB;
    rs[idx] = c < nb ? R[(c0 + j) + (long)c * ldr] : 0.0;
  }
  __syncthreads();
  const int i0 = blockIdx.x * (2 * kThreads) + threadIdx.x;
  const int i1 = i0 + kThreads;
  double a0[NB], a1[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) a0[c] = a1[c] = 0.0;
  const bool v0 = i0 < n, v1 = i1 < n;
  const T* base = X + (long)c0 * ld;
  int j = 0;
  for (; j + 3 < cols; j += 4) {
    double x0[4], x1[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x0[u] = v0 ? as_f64(base[i0 + (long)(j + u) * ld]) : 0.0;
      x1[u] = v1 ? as_f64(base[i1 + (long)(j + u) * ld]) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        const double r = rs[(j + u) * NB + c];
        a0[c] = fma(x0[u], r, a0[c]);
        a1[c] = fma(x1[u], r, a1[c]);
      }
  }
  for (; j < cols; ++j) {
    const double x0 = v0 ? as_f64(base[i0 + (long)j * ld]) : 0.0;
    const double x1 = v1 ? as_f64(base[i1 + (long)j * ld]) : 0.0;
#pragma unroll
    for (int c = 0; c < NB; ++c) {
      const double r = rs[j * NB + c];
      a0[c] = fma(x0, r, a0[c]);
      a1[c] = fma(x1, r, a1[c]);
    }
  }
  double* out = partial + (long)chunk * n * nb;
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    if (c < nb) {
      if (v0) out[i0 + (long)c * n] = a0[c];
      if (v1) out[i1 + (long)c * n] = a1[c];
    }
  }
}

// X R with 16-byte row vectors: thread t of a 256 x V row tile takes rows
// V t .. V t + V - 1 (V = 16 / sizeof(T): 8 BF16, 4 FP32, 2 FP64 rows) with
// one 16-byte load per column, 4 columns per step. Needs a column stride
// that is a multiple of 8 elements and a 16-byte aligned X. Each row's sum
// runs over the chunk's columns in order, exactly as in xr_kernel.
template <class T>
struct Vec16 {
  static constexpr int V = 16 / sizeof(T);
  static __device__ __forceinline__ void unpack(const uint4& raw, double (&x)[V]) {
    const T* v = reinterpret_cast<const T*>(&raw);
#pragma unroll
    for (int e = 0; e < V; ++e) x[e] = as_f64(v[e]);
  }
};

template <class T, int NB>
__global__ void __launch_bounds__(kThreads)
    xr_vec_kernel(const T* __restrict__ X, int n, int p, long ld,
                  const double* __restrict__ R, long ldr, int nb, int cc,
                  double* __restrict__ partial) {
  constexpr int V = Vec16<T>::V;
  extern __shared__ double rs[];  // cc x NB
  const int chunk = blockIdx.y;
  const int c0 = chunk * cc;
  const int cols = min(cc, p - c0);
  for (int idx = threadIdx.x; idx < cols * NB; idx += blockDim.x) {
    const int j = idx / NB, c = idx % NB;
    rs[idx] = c < nb ? R[(c0 + j) + (long)c * ldr] : 0.0;
  }
  __syncthreads();
  const int r0 = blockIdx.x * (kThreads * V) + threadIdx.x * V;
  if (r0 >= n) return;
  double acc[V][NB];
#pragma unroll
  for (int e = 0; e < V; ++e)
#pragma unroll
    for (int c = 0; c < NB; ++c) acc[e][c] = 0.0;
  const T* base = X + (long)c0 * ld + r0;
  if (r0 + V <= n) {
    int j = 0;
    for (; j + 3 < cols; j += 4) {
      uint4 raw[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        raw[u] = __ldcs(reinterpret_cast<const uint4*>(base + (long)(j + u) * ld));
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        double x[V];
        Vec16<T>::unpack(raw[u], x);
#pragma unroll
        for (int c = 0; c < NB; ++c) {
          const double r = rs[(j + u) * NB + c];
#pragma unroll
          for (int e = 0; e < V; ++e) acc[e][c] = fma(x[e], r, acc[e][c]);
        }
      }
    }
    for (; j < cols; ++j) {
      double x[V];
      Vec16<T>::unpack(__ldcs(reinterpret_cast<const uint4*>(base + (long)j * ld)), x);
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        const double r = rs[j * NB + c];
#pragma unroll
        for (int e = 0; e < V; ++e) acc[e][c] = fma(x[e], r, acc[e][c]);
      }
    }
  } else {  // ragged last rows: element loads
    for (int j = 0; j < cols; ++j) {
#pragma unroll
      for (int e = 0; e < V; ++e) {
        if (r0 + e >= n) break;
        const double x = as_f64(base[(long)j * ld + e]);
#pragma unroll
        for (int c = 0; c < NB; ++c) acc[e][c] = fma(x, rs[j * NB + c], acc[e][c]);
      }
    }
  }
  double* out = partial + (long)chunk * n * nb;
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    if (c < nb) {
#pragma unroll
      for (int e = 0; e < V; ++e)
        if (r0 + e < n) out[r0 + e + (long)c * n] = acc[e][c];
    }
  }
}

__global__ void xr_finish(const double* __restrict__ partial, int chunks, int n,
                          int nb, const double* offset, double* out, long ldo) {
  const long total = (long)n * nb;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), c = (int)(idx / n);
    double v = 0.0;
    for (int k = 0; k < chunks; ++k) v += partial[(long)k * n * nb + idx];
    if (offset) v -= offset[c];
    out[i + (long)c * ldo] = v;
  }
}

template <class T, int NB>
void xr_launch(const T* X, int n, int p, long ld, const double* R, long ldr,
               int nb, const double* offset, double* out, long ldo,
               DeviceArray<double>& scratch, cudaStream_t stream) {
  // 16-byte row vectors for the one- and two-column products (HBM-bound);
  // wider products are FP64-issue-bound and keep two rows per thread. The
  // column chunks depend on n and p only (a nominal 1024-row tile), so every
  // storage type and both kernels sum each row in the same order.
  const bool vec = NB <= 2 && ld % 8 == 0 && reinterpret_cast<uintptr_t>(X) % 16 == 0;
  const int nominal_tiles = (int)ceil_div(n, 1024);
  const int want = 16 * num_sms();
  int chunks = std::max(1, std::min((int)ceil_div(want, nominal_tiles), (int)ceil_div(p, 64)));
  int cc = (int)ceil_div(p, chunks);
  cc = std::min(cc, (48 * 1024 / 8) / NB);
  chunks = (int)ceil_div(p, cc);
  scratch.reserve((size_t)chunks * n * nb, stream);
  const size_t smem = (size_t)cc * NB * sizeof(double);
  bool launched = false;
  if constexpr (NB <= 2) {
    if (vec) {
      xr_vec_kernel<T, NB><<<dim3(ceil_div(n, kThreads * Vec16<T>::V), chunks), kThreads, smem,
                             stream>>>(X, n, p, ld, R, ldr, nb, cc, scratch.get());
      launched = true;
    }
  }
  if (!launched)
    xr_kernel<T, NB><<<dim3(ceil_div(n, 2 * kThreads), chunks), kThreads, smem, stream>>>(
        X, n, p, ld, R, ldr, nb, cc, scratch.get());
  count_launch();
  FPLS_LAUNCH("xr_kernel");
  const long total = (long)n * nb;
  const unsigned blocks = (unsigned)std::min<long>((total + 255) / 256, 8L * num_sms());
  xr_finish<<<blocks, 256, 0, stream>>>(scratch.get(), chunks, n, nb, offset, out, ldo);
  count_launch();
  FPLS_LAUNCH("xr_finish");
}

template <class T>
__global__ void gather_rows_kernel(const T* __restrict__ src, long ld_src,
                                   int cols, const int* __restrict__ idx,
                                   int count, T* __restrict__ dst, long ld_dst) {
  const long total = (long)count * cols;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total;
       k += (long)gridDim.x * blockDim.x) {
    const int r = (int)(k % count);
    const long c = k / count;
    dst[r + c * ld_dst] = src[idx[r] + c * ld_src];
  }
}

__global__ void topk_kernel(const double* __restrict__ v, int rows, int classes,
                            int top, int* __restrict__ out, long ldo) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  // repeated strict-'>' scans: the lowest index wins ties, ranks are distinct
  unsigned long long used_lo = 0ull;
  for (int k = 0; k < top; ++k) {
    int best = -1;
    double bv = 0.0;
    for (int c = 0; c < classes; ++c) {
      if (c < 64 && ((used_lo >> c) & 1ull)) continue;
      if (c >= 64) {
        bool taken = false;
        for (int q = 0; q < k; ++q)
          if (out[r + (long)q * ldo] == c + 1) taken = true;
        if (taken) continue;
      }
      const double x = v[r + (long)c * rows];
      if (best < 0 || x > bv) {
        best = c;
        bv = x;
      }
    }
    if (best < 64 && best >= 0) used_lo |= 1ull << best;
    out[r + (long)k * ldo] = best + 1;
  }
}

}  // namespace

template <class T>
void column_moments(const T* X, int n, int p, long ld, const double* Yc, int m,
                    double* sum, double* sumsq, double* cross,
                    DeviceArray<double>& scratch, cudaStream_t stream) {
  // the first pass carries the column sums and sums of squares with up to 32
  // response columns; further columns go in passes of 32 without them
  const int w0 = std::min(m, 32);
  xtv_dispatch<T, true>(X, n, p, ld, Yc, n, w0, cross, p, sum, sumsq, scratch,
                        stream);
  for (int c0 = 32; c0 < m; c0 += 32) {
    const int w = std::min(32, m - c0);
    xtv_dispatch<T, false>(X, n, p, ld, Yc + (long)c0 * n, n, w,
                           cross + (long)c0 * p, p, nullptr, nullptr, scratch,
                           stream);
  }
}

// ---------------------------------------------------------------------------
// Column moments with one-based class labels (classification): per column
// the sum, the sum of squares and the per-class sums, in one pass over X.
// Block = 8 warps over a 32-column tile and a chunk of rows whose labels are
// staged in shared memory; each lane keeps its own class accumulators in
// shared memory (acc[warp][class][lane]), so an element costs one add into
// its class's slot instead of m products with staged responses. partial
// layout: [chunk][j][slot], slots = classes, sum, sumsq.
template <class T>
__global__ void __launch_bounds__(kThreads)
    class_moments_kernel(const T* __restrict__ X, int n, int p, long ld,
                         const int* __restrict__ labels, int m, int rc,
                         double* __restrict__ partial) {
  extern __shared__ double csm[];
  int* lab = reinterpret_cast<int*>(csm);                  // rc labels
  double* acc = csm + (rc + 1) / 2;                        // 8 x m x 32
  const int chunk = blockIdx.y;
  const int r0 = chunk * rc;
  const int rows = min(rc, n - r0);
  for (int r = threadIdx.x; r < rows; r += blockDim.x) lab[r] = labels[r0 + r] - 1;
  __syncthreads();
  const int slots = m + 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* my = acc + (long)warp * m * 32;
  for (int jj = warp; jj < 32; jj += kThreads / 32) {
    const int j = blockIdx.x * 32 + jj;
    if (j >= p) break;
    for (int c = 0; c < m; ++c) my[c * 32 + lane] = 0.0;
    __syncwarp();
    const T* col = X + (long)j * ld + r0;
    double s = 0.0, ss = 0.0;
    int r = lane;
    for (; r + 96 < rows; r += 128) {
      double x[4];
      int l[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        x[u] = as_f64(col[r + 32 * u]);
        l[u] = lab[r + 32 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        s += x[u];
        ss = fma(x[u], x[u], ss);
        if (l[u] >= 0 && l[u] < m) my[l[u] * 32 + lane] += x[u];
      }
    }
    for (; r < rows; r += 32) {
      const double x = as_f64(col[r]);
      const int l = lab[r];
      s += x;
      ss = fma(x, x, ss);
      if (l >= 0 && l < m) my[l * 32 + lane] += x;
    }
    __syncwarp();
    double* out = partial + ((long)chunk * p + j) * slots;
    for (int c = 0; c < m; ++c) {
      const double v = warp_sum(my[c * 32 + lane]);
      if (lane == 0) out[c] = v;
    }
    s = warp_sum(s);
    ss = warp_sum(ss);
    if (lane == 0) {
      out[m] = s;
      out[m + 1] = ss;
    }
    __syncwarp();
  }
}

// cross[j + c p] = classsum[j, c] - prior[c] * colsum[j] (= X^T (onehot -
// prior)), sum and sumsq, from the per-chunk partials.
__global__ void class_moments_finish(const double* __restrict__ partial, int chunks, int p,
                                     int m, const double* __restrict__ prior, double* sum,
                                     double* sumsq, double* cross) {
  const int slots = m + 2;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x) {
    double s = 0.0, ss = 0.0;
    for (int k = 0; k < chunks; ++k) {
      s += partial[((long)k * p + j) * slots + m];
      ss += partial[((long)k * p + j) * slots + m + 1];
    }
    sum[j] = s;
    sumsq[j] = ss;
    for (int c = 0; c < m; ++c) {
      double v = 0.0;
      for (int k = 0; k < chunks; ++k) v += partial[((long)k * p + j) * slots + c];
      cross[j + (long)c * p] = v - prior[c] * s;
    }
  }
}

template <class T>
void class_moments(const T* X, int n, int p, long ld, const int* labels, int m,
                   const double* prior, double* sum, double* sumsq, double* cross,
                   DeviceArray<double>& scratch, cudaStream_t stream) {
  // rows per chunk: enough blocks to cover every SM several times
  const int col_tiles = (int)ceil_div(p, 32);
  int rc = 2048;
  int chunks = (int)ceil_div(n, rc);
  const int want = 6 * num_sms();
  if (col_tiles * chunks < want && n > 256) {
    const int target = std::min((int)ceil_div(n, 256), (int)ceil_div(want, col_tiles));
    if (target > chunks) {
      rc = std::max(256, (int)ceil_div(n, target));
      rc = (rc + 127) / 128 * 128;
      chunks = (int)ceil_div(n, rc);
    }
  }
  const int slots = m + 2;
  scratch.reserve((size_t)chunks * p * slots, stream);
  const size_t smem = (size_t)(rc + 1) / 2 * sizeof(double) + (size_t)8 * m * 32 * sizeof(double);
  static const bool configured = [] {
    FPLS_CHECK(cudaFuncSetAttribute(class_moments_kernel<T>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (2048 / 2 + 8 * kClassMomentsMaxClasses * 32) * 8));
    return true;
  }();
  (void)configured;
  class_moments_kernel<T><<<dim3(col_tiles, chunks), kThreads, smem, stream>>>(
      X, n, p, ld, labels, m, rc, scratch.get());
  count_launch();
  FPLS_LAUNCH("class_moments_kernel");
  class_moments_finish<<<std::min<unsigned>(ceil_div(p, 256), 8 * num_sms()), 256, 0, stream>>>(
      scratch.get(), chunks, p, m, prior, sum, sumsq, cross);
  count_launch();
  FPLS_LAUNCH("class_moments_finish");
}

template <class T>
void xtv_product(const T* X, int n, int p, long ld, const double* V, long ldv,
                 int nb, double* out, long ldo, DeviceArray<double>& scratch,
                 cudaStream_t stream) {
  for (int c0 = 0; c0 < nb; c0 += 32) {
    const int w = std::min(32, nb - c0);
    xtv_dispatch<T, false>(X, n, p, ld, V + (long)c0 * ldv, ldv, w,
                           out + (long)c0 * ldo, ldo, nullptr, nullptr,
                           scratch, stream);
  }
}

template <class T>
void xr_product(const T* X, int n, int p, long ld, const double* R, long ldr,
                int nb, const double* offset, double* out, long ldo,
                DeviceArray<double>& scratch, cudaStream_t stream, int* flag) {
  // 3..16 columns of a large X: one pass over X on bulk-copy stages instead
  // of a pass per 8 columns
  if (nb >= 3 && nb <= 16 && (long)n * p >= (1L << 24) &&
      xr_ring<T>(X, n, p, ld, R, ldr, nb, offset, out, ldo, flag, stream))
    return;
  for (int c0 = 0; c0 < nb; c0 += 8) {
    const int w = std::min(8, nb - c0);
    const double* off = offset ? offset + c0 : nullptr;
    if (w == 1)
      xr_launch<T, 1>(X, n, p, ld, R + (long)c0 * ldr, ldr, w, off, out + (long)c0 * ldo, ldo, scratch, stream);
    else if (w <= 2)
      xr_launch<T, 2>(X, n, p, ld, R + (long)c0 * ldr, ldr, w, off, out + (long)c0 * ldo, ldo, scratch, stream);
    else if (w <= 4)
      xr_launch<T, 4>(X, n, p, ld, R + (long)c0 * ldr, ldr, w, off, out + (long)c0 * ldo, ldo, scratch, stream);
    else
      xr_launch<T, 8>(X, n, p, ld, R + (long)c0 * ldr, ldr, w, off, out + (long)c0 * ldo, ldo, scratch, stream);
  }
}

template <class T>
void gather_rows(const T* src, long ld_src, int cols, const int* idx, int count,
                 T* dst, long ld_dst, cudaStream_t stream) {
  if (count <= 0 || cols <= 0) return;
  const long total = (long)count * cols;
  const unsigned blocks = (unsigned)std::min<long>((total + 255) / 256, 16L * num_sms());
  gather_rows_kernel<T><<<blocks, 256, 0, stream>>>(src, ld_src, cols, idx, count, dst, ld_dst);
  count_launch();
  FPLS_LAUNCH("gather_rows");
}

void topk_rows(const double* values, int rows, int classes, int top, int* out,
               long ldo, cudaStream_t stream) {
  if (rows <= 0) return;
  topk_kernel<<<ceil_div(rows, 128), 128, 0, stream>>>(values, rows, classes, top, out, ldo);
  count_launch();
  FPLS_LAUNCH("topk_rows");
}

#define FPLS_INSTANTIATE(T)                                                   \
  template void class_moments<T>(const T*, int, int, long, const int*, int,  \
                                 const double*, double*, double*, double*,   \
                                 DeviceArray<double>&, cudaStream_t);        \
  template void column_moments<T>(const T*, int, int, long, const double*,    \
                                  int, double*, double*, double*,             \
                                  DeviceArray<double>&, cudaStream_t);        \
  template void xtv_product<T>(const T*, int, int, long, const double*, long, \
                               int, double*, long, DeviceArray<double>&,      \
                               cudaStream_t);                                 \
  template void xr_product<T>(const T*, int, int, long, const double*, long,  \
                              int, const double*, double*, long,              \
                              DeviceArray<double>&, cudaStream_t, int*);      \
  template void gather_rows<T>(const T*, long, int, const int*, int, T*,      \
                               long, cudaStream_t);
FPLS_INSTANTIATE(float)
FPLS_INSTANTIATE(double)
FPLS_INSTANTIATE(bf16)
template void gather_rows<int>(const int*, long, int, const int*, int, int*,
                               long, cudaStream_t);
#undef FPLS_INSTANTIATE

}  // namespace fpls
