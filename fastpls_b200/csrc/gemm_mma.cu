// FP64 GEMM on the FP64 tensor-core path (DMMA, mma.sync m8n8k4 f64).
//
//   C[M x N] = alpha * A[M x K] * op(B) (+ beta C), all FP64, column-major;
//   op(B) = B (K x N, ld >= K) or B^T (B stored N x K, ld >= N).
//
// B200 has no tcgen05 kind for FP64; its FP64 tensor path is the warp-level
// DMMA instruction (same peak as DFMA, ~37 TFLOP/s, but one instruction does
// 256 FMAs from register fragments, so shared-memory and issue bandwidth stop
// being the limit of a SIMT register-tiled kernel).
//
// Block tile 128 x 128 x 16, 8 warps (2 x 4) each owning a 64 x 32 tile
// (8 x 4 DMMA tiles, 64 FP64 accumulators per thread). Operand slabs stream
// through a 3-stage cp.async ring (16-byte copies, zero-filled outside the
// matrix). Shared layouts are padded so the fragment loads are conflict-free:
// k-major [16][136] for operands contiguous along M/N, n-major [128][20] for
// B contiguous along K. `lower` restricts the grid to the lower triangle of
// block tiles (symmetric products such as the Gram X X^T); the caller mirrors.
#include "common.cuh"
#include "kernels.cuh"

#include <algorithm>

namespace fpls {

namespace {

constexpr int TM = 128, TN = 128, TK = 16, STAGES = 3, NT = 256;
constexpr int LDA_S = TM + 8;   // k-major stride (doubles)
constexpr int LDBN_S = TK + 4;  // n-major stride (doubles)

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int bytes = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// B_T: op(B) = B^T (B stored N x K, contiguous along N)
template <bool B_T>
__global__ void __launch_bounds__(NT, 1)
    dgemm_mma(int M, int N, int K, const double* __restrict__ A, long lda,
              const double* __restrict__ B, long ldb, double alpha, double beta,
              double* __restrict__ C, long ldc, long split_stride,
              int k_per_split, int lower) {
  extern __shared__ __align__(16) double smem[];
  double* As = smem;                                  // STAGES x TK x LDA_S
  double* Bs = smem + STAGES * TK * LDA_S;            // STAGES x (TK x LDA_S | TN x LDBN_S)
  constexpr int B_STAGE = B_T ? TK * LDA_S : TN * LDBN_S;

  int bm, bn;
  if (lower) {
    // blockIdx.x enumerates lower-triangular tile pairs (bm >= bn)
    const int t = blockIdx.x;
    bm = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while (bm * (bm + 1) / 2 > t) --bm;
    while ((bm + 1) * (bm + 2) / 2 <= t) ++bm;
    bn = t - bm * (bm + 1) / 2;
  } else {
    bn = blockIdx.x;
    bm = blockIdx.y;
  }
  const int m0 = bm * TM, n0 = bn * TN;
  const int kbeg = blockIdx.z * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  const int ktiles = kend > kbeg ? (kend - kbeg + TK - 1) / TK : 0;
  double* Cz = C + (long)blockIdx.z * split_stride;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps

  auto load_stage = [&](int stage, int kt) {
    const int k0 = kbeg + kt * TK;
    double* as = As + stage * TK * LDA_S;
    double* bs = Bs + stage * B_STAGE;
    // A: TK rows (k) of 128 contiguous m -> 16 x 64 chunks of 2 doubles
#pragma unroll
    for (int it = 0; it < (TK * TM / 2) / NT; ++it) {
      const int c = tid + it * NT;
      const int kk = c / (TM / 2), mm = (c % (TM / 2)) * 2;
      const int gm = m0 + mm, gk = k0 + kk;
      const bool ok = gm < M && gk < kend;
      cp_async16(as + kk * LDA_S + mm, ok ? A + gm + (long)gk * lda : A, ok);
    }
    if (B_T) {
      // op(B)(k, n) = B[n + k*ldb]: contiguous along n, stored k-major
#pragma unroll
      for (int it = 0; it < (TK * TN / 2) / NT; ++it) {
        const int c = tid + it * NT;
        const int kk = c / (TN / 2), nn = (c % (TN / 2)) * 2;
        const int gn = n0 + nn, gk = k0 + kk;
        const bool ok = gn < N && gk < kend;
        cp_async16(bs + kk * LDA_S + nn, ok ? B + gn + (long)gk * ldb : B, ok);
      }
    } else {
      // op(B)(k, n) = B[k + n*ldb]: contiguous along k, stored n-major
#pragma unroll
      for (int it = 0; it < (TK * TN / 2) / NT; ++it) {
        const int c = tid + it * NT;
        const int nn = c / (TK / 2), kk = (c % (TK / 2)) * 2;
        const int gn = n0 + nn, gk = k0 + kk;
        const bool ok = gn < N && gk < kend;
        cp_async16(bs + nn * LDBN_S + kk, ok ? B + gk + (long)gn * ldb : B, ok);
      }
    }
  };

  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_commit();
  }
  const int g = lane >> 2, tg = lane & 3;
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    const int pre = kt + STAGES - 1;
    if (pre < ktiles) load_stage(pre % STAGES, pre);
    cp_commit();
    const double* as = As + (kt % STAGES) * TK * LDA_S;
    const double* bs = Bs + (kt % STAGES) * B_STAGE;
#pragma unroll
    for (int kk = 0; kk < TK; kk += 4) {
      double af[8], bf[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) af[i] = as[(kk + tg) * LDA_S + wm * 64 + i * 8 + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int nn = wn * 32 + j * 8 + g;
        bf[j] = B_T ? bs[(kk + tg) * LDA_S + nn] : bs[nn * LDBN_S + kk + tg];
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_wait<0>();

#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int row = m0 + wm * 64 + i * 8 + g;
    if (row >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int col = n0 + wn * 32 + j * 8 + tg * 2 + h;
        if (col >= N) continue;
        double* dst = Cz + row + (long)col * ldc;
        const double v = alpha * acc[i][j][h];
        *dst = beta != 0.0 ? fma(beta, *dst, v) : v;
      }
    }
  }
}

__global__ void mirror_lower(double* C, int n, long ldc) {
  const long total = (long)n * n;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % n), c = (int)(idx / n);
    if (r < c) C[r + (long)c * ldc] = C[c + (long)r * ldc];
  }
}

size_t smem_bytes(bool b_t) {
  const size_t a = (size_t)STAGES * TK * LDA_S;
  const size_t b = (size_t)STAGES * (b_t ? TK * LDA_S : TN * LDBN_S);
  return (a + b) * sizeof(double);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

bool gemm_mma_supported(const GemmArgs& g) {
  if (g.a_f32 || g.b_f32 || g.trans_a || g.kscale) return false;
  if (!aligned16(g.A) || !aligned16(g.B)) return false;
  if ((g.lda & 1) || (g.ldb & 1)) return false;
  if (g.M & 1) return false;
  if (!g.trans_b && (g.K & 1)) return false;
  if (g.trans_b && (g.N & 1)) return false;
  return true;
}

void gemm_mma_launch(const GemmArgs& g, bool lower, cudaStream_t stream) {
  const size_t smem = smem_bytes(g.trans_b);
  static bool configured[2] = {false, false};
  if (!configured[g.trans_b]) {
    if (g.trans_b)
      FPLS_CHECK(cudaFuncSetAttribute(dgemm_mma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
      FPLS_CHECK(cudaFuncSetAttribute(dgemm_mma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured[g.trans_b] = true;
  }
  const int kps = ((g.K + g.splits - 1) / g.splits + TK - 1) / TK * TK;
  dim3 grid;
  if (lower) {
    const unsigned tiles = ceil_div(g.M, TM);
    grid = dim3(tiles * (tiles + 1) / 2, 1, g.splits);
  } else {
    grid = dim3(ceil_div(g.N, TN), ceil_div(g.M, TM), g.splits);
  }
  if (g.trans_b)
    dgemm_mma<true><<<grid, NT, smem, stream>>>(g.M, g.N, g.K, static_cast<const double*>(g.A), g.lda,
                                                static_cast<const double*>(g.B), g.ldb, g.alpha, g.beta,
                                                g.C, g.ldc, g.split_stride, kps, lower ? 1 : 0);
  else
    dgemm_mma<false><<<grid, NT, smem, stream>>>(g.M, g.N, g.K, static_cast<const double*>(g.A), g.lda,
                                                 static_cast<const double*>(g.B), g.ldb, g.alpha, g.beta,
                                                 g.C, g.ldc, g.split_stride, kps, lower ? 1 : 0);
  count_launch();
  FPLS_LAUNCH("dgemm_mma");
}

void mirror_lower_triangle(double* C, int n, long ldc, cudaStream_t stream) {
  const long total = (long)n * n;
  mirror_lower<<<(unsigned)std::min<long>((total + 255) / 256, 16L * num_sms()), 256, 0, stream>>>(C, n, ldc);
  count_launch();
  FPLS_LAUNCH("mirror_lower");
}

}  // namespace fpls
