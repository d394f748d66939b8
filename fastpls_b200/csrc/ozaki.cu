// FP64-accurate GEMM on the int8 tensor cores (tcgen05.mma kind::i8, TMEM
// accumulators, TMA-fed shared memory), by the digit split described in
// ozaki.cuh.
//
// Kernel layout (one CTA per 128 x 128 output tile, 320 threads):
//   warp 0, lane 0   bulk-copy producer: per k-block of 32 bytes, the digit
//                    planes 0..ns-1 of the A rows and of the B rows of the
//                    tile (4 KB each, stored pre-tiled so that they are one
//                    contiguous run per operand) by two cp.async.bulk copies
//                    (TMA engine) into a ring of stages.
//   warp 1, lane 0   MMA issuer: for every diagonal d of the pass and every
//                    digit pair (s, d - s), one tcgen05.mma (K = 32) into the
//                    TMEM accumulator of d (128 lanes x 128 int32 columns);
//                    tcgen05.commit releases the stage.
//   warps 2..9       epilogue: tcgen05.ld of the accumulators (lane quarter
//                    = warp % 4, column half = (warp - 2) / 4), exact int32 ->
//                    FP64, weighted sum over the diagonals, power-of-two row
//                    scales, one store to C.
// TMEM holds four 128-column accumulators, so the S diagonals run in passes
// of four (S = 6: diagonals 0-3, then 4-5); the epilogue keeps the first
// pass's 64 partial sums per thread in registers while the second pass runs.
// Every wait on an mbarrier is bounded: on expiry the kernel sets flag = 4,
// stops issuing, waits (bounded) for its copies and MMAs in flight, frees TMEM
// and returns.
#include "ozaki.cuh"
#include "kernels.cuh"


#include <algorithm>
#include <cmath>
#include <cstdlib>

namespace fpls {

int& ozaki_slices() {
  static int slices = 6;
  return slices;
}

OzakiWaitTest& ozaki_wait_test() {
  static OzakiWaitTest t;
  return t;
}

// MMA issue order of the int8 product within a stage: 0 = diagonal-major
// (default: each diagonal's MMAs back to back into its accumulator), 1 =
// digit-major (consecutive MMAs alternate between the accumulators).
// Bit-identical results either way; digit-major measured 14% slower on the
// benchmark's products (1.37 against 1.59 POP/s). The environment variable
// FASTPLS_B200_INT8_ORDER (0 or 1) selects the order.
int ozaki_mma_order() {
  static const int order = [] {
    const char* e = std::getenv("FASTPLS_B200_INT8_ORDER");
    return (e && e[0] == '1') ? 1 : 0;
  }();
  return order;
}

namespace {

constexpr int OZ_BM = 128;                 // A rows per tile (TMEM lanes)
constexpr int OZ_BK = 32;                  // k bytes per stage
constexpr int OZ_KPAD = 64;                // k padding of the digit planes
constexpr int OZ_ROWPAD = 64;              // row padding of the digit planes
constexpr int OZ_TAIL = 256 * OZ_BK;       // bytes past the last plane a tile may read
constexpr int OZ_A_PLANE = OZ_BM * OZ_BK;  // one A digit plane block: 4 KB
constexpr int OZ_DATA = 222 * 1024;        // bytes of stages
constexpr int OZ_MAX_STAGES = 8;
constexpr int OZ_EPI_WARPS = 8;
constexpr int OZ_THREADS = 64 + 32 * OZ_EPI_WARPS;
constexpr int OZ_TMEM_COLS = 512;
constexpr long long OZ_WAIT_CYCLES = 4000000000LL;  // about 2 s

// Tile shapes: BN output columns (B rows) per tile. TMEM holds 512 int32
// columns: four 128-column accumulators (diagonals per pass) for BN = 128,
// two for BN = 192 and 256.
template <int BN>
struct OzShape {
  static constexpr int ACC = BN == 128 ? 4 : 2;
  static constexpr int B_PLANE = BN * OZ_BK;
  // s32 accumulator, signed int8 A and B, both K-major, N = BN (bits 17-22:
  // N / 8), M = 128 (bits 24-28: M / 16)
  static constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) |
                                    ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(OZ_BM >> 4) << 24);
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256 && ACC * BN <= OZ_TMEM_COLS, "tile");
};

struct OzArgs {
  int M, N;          // valid rows of A (output rows) and of B (output columns)
  int tiles_n;       // column tiles (rectangular grid)
  int kb0, kblocks;  // k-block range of this launch
  int rows_pa, rows_pb;  // padded rows of the digit layouts of A and B
  int slices, stages, lower, accumulate;
  int interleave;    // MMA order within a stage (1: digit-major across diagonals)
  int skip_last;     // test of the bounded waits: withhold each tile's last stage
  long long wait_cycles;  // bound of the MMA issuer's wait for a stage
  long ldc;
  double* C;
  const double* scale_a;
  const double* scale_b;
  int* flag;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the phase of the given parity. Gives up when another
// thread of the CTA gave up (abort set, unless ignore_abort) or after
// OZ_WAIT_CYCLES; a timeout sets the CTA abort flag and the error flag.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort,
                          int* flag, bool ignore_abort = false,
                          long long limit = OZ_WAIT_CYCLES) {
  const long long start = clock64();
  while (!mbar_test(bar, parity)) {
    if (!ignore_abort && *abort) return false;
    if (clock64() - start > limit) {
      *abort = 1;
      flag_error(flag, 4);
      return false;
    }
  }
  return true;
}

// One contiguous global -> shared copy on the TMA engine, completing on an
// mbarrier (addresses 16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, no swizzle. A plane block holds
// row groups of 2 k-chunks x 8 x 16-byte core matrices: k-adjacent core
// matrices 128 bytes apart (leading offset), row groups 256 bytes apart
// (stride offset); descriptor version 1.
__device__ __forceinline__ uint64_t core_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(256 >> 4) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t a, uint32_t b, uint32_t c,
                                         uint32_t d) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr),
               "r"(a), "r"(b), "r"(c), "r"(d)
               : "memory");
}

__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// 1 / (127^2 254^d): the weight of diagonal d (254^d exact for d < 7)
constexpr double oz_weight(int d) {
  double p = 1.0;
  for (int i = 0; i < d; ++i) p *= 254.0;
  return 1.0 / (16129.0 * p);
}
__constant__ double kOzWeight[kOzakiMaxSlices] = {oz_weight(0), oz_weight(1), oz_weight(2),
                                                  oz_weight(3), oz_weight(4), oz_weight(5),
                                                  oz_weight(6)};

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Weighted sum over the nd accumulators of a pass for 4 columns of this
// thread's TMEM lane, smallest weight first (exact int32 -> FP64).
template <int ACC, int BN>
__device__ __forceinline__ void pass_sum4(uint32_t addr, int nd, const double (&w)[ACC],
                                          double (&v)[4]) {
  uint32_t r[ACC][4];
#pragma unroll
  for (int a = 0; a < ACC; ++a)
    if (a < nd) tmem_ld4(addr + (uint32_t)(a * BN), r[a]);
  tmem_wait_ld();
#pragma unroll
  for (int j = 0; j < 4; ++j) v[j] = 0.0;
#pragma unroll
  for (int a = ACC - 1; a >= 0; --a)
    if (a < nd) {
#pragma unroll
      for (int j = 0; j < 4; ++j) v[j] = __dadd_rn(v[j], __dmul_rn(w[a], (double)(int)r[a][j]));
    }
}

template <int BN>
__global__ void __launch_bounds__(OZ_THREADS, 1)
    ozaki_gemm_kernel(const int8_t* __restrict__ digits_a, const int8_t* __restrict__ digits_b,
                      const OzArgs args) {
  using Shape = OzShape<BN>;
  constexpr int ACC = Shape::ACC;
  extern __shared__ uint8_t oz_smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[OZ_MAX_STAGES];
  __shared__ __align__(8) uint64_t empty_bar[OZ_MAX_STAGES];
  __shared__ __align__(8) uint64_t acc_full, acc_empty, drain_bar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int abort_s;
  volatile int* abort = &abort_s;

  uint8_t* smem = oz_smem_raw + ((1024 - (smem_u32(oz_smem_raw) & 1023)) & 1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int tm, tn;
  if (args.lower) {
    // blockIdx.x = tm (tm + 1) / 2 + tn, tn <= tm (BN == OZ_BM)
    const int t = blockIdx.x;
    int r = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    while (r * (r + 1) / 2 > t) --r;
    tm = r;
    tn = t - r * (r + 1) / 2;
  } else {
    tm = blockIdx.x / args.tiles_n;
    tn = blockIdx.x % args.tiles_n;
  }
  const int S = args.slices;
  const int stages = args.stages;
  const int stage_bytes = S * (OZ_A_PLANE + Shape::B_PLANE);
  const int npass = (S + ACC - 1) / ACC;

  if (threadIdx.x == 0) {
    for (int i = 0; i < stages; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    mbar_init(&acc_full, 1);
    mbar_init(&acc_empty, 32 * OZ_EPI_WARPS);
    mbar_init(&drain_bar, 1);
    abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(OZ_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------------------------------------------------- producer
      uint32_t it = 0;
      bool ok = true;
      for (int pass = 0; pass < npass && ok; ++pass) {
        const int dhi = min(S - 1, pass * ACC + ACC - 1);
        const int ns = min(S, dhi + 1);
        // a stage has S plane slots of A and of B: a pass that needs ns < S
        // digit planes packs S / ns k-blocks into each stage
        const int kbs = S / ns;
        for (int kb = 0; kb < args.kblocks; kb += kbs) {
          const int nk = min(kbs, args.kblocks - kb);
          const int st = it % stages;
          if (args.skip_last && pass + 1 == npass && kb + kbs >= args.kblocks) {
            ok = false;  // the stage is never issued: the MMA issuer's wait runs out
            break;
          }
          if (it >= (uint32_t)stages &&
              !mbar_wait(&empty_bar[st], ((it / stages) - 1) & 1, abort, args.flag)) {
            ok = false;
            break;
          }
          uint8_t* a_dst = smem + st * stage_bytes;
          uint8_t* b_dst = a_dst + S * OZ_A_PLANE;
          mbar_expect_tx(&full_bar[st], (uint32_t)(nk * ns) * (OZ_A_PLANE + Shape::B_PLANE));
          for (int q = 0; q < nk; ++q) {
            const long slab = (long)(args.kb0 + kb + q) * S;
            for (int j = 0; j < ns; ++j) {
              bulk_load(a_dst + (q * ns + j) * OZ_A_PLANE,
                        digits_a + ((slab + j) * args.rows_pa + (long)tm * OZ_BM) * OZ_BK,
                        (uint32_t)OZ_A_PLANE, &full_bar[st]);
              bulk_load(b_dst + (q * ns + j) * Shape::B_PLANE,
                        digits_b + ((slab + j) * args.rows_pb + (long)tn * BN) * OZ_BK,
                        (uint32_t)Shape::B_PLANE, &full_bar[st]);
            }
          }
          ++it;
        }
      }
      // copies still in flight land before the CTA leaves (no-op when every
      // stage was consumed)
      for (uint32_t j = it > (uint32_t)stages ? it - stages : 0; j < it; ++j)
        mbar_wait(&full_bar[j % stages], (j / stages) & 1, abort, args.flag, true);
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      // -------------------------------------------------------- MMA issuer
      uint32_t it = 0;
      bool ok = true;
      for (int pass = 0; pass < npass && ok; ++pass) {
        const int dlo = pass * ACC, dhi = min(S - 1, dlo + ACC - 1);
        if (pass > 0) {
          if (!mbar_wait(&acc_empty, (pass - 1) & 1, abort, args.flag)) break;
          tc_fence_after();
        }
        const int ns = min(S, dhi + 1);
        const int kbs = S / ns;
        for (int kb = 0; kb < args.kblocks; kb += kbs) {
          const int nk = min(kbs, args.kblocks - kb);
          const int st = it % stages;
          if (!mbar_wait(&full_bar[st], (it / stages) & 1, abort, args.flag, false,
                         args.wait_cycles)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(smem + st * stage_bytes);
          const uint32_t b0 = a0 + S * OZ_A_PLANE;
          for (int q = 0; q < nk; ++q) {
            if (args.interleave) {
              // digit s outer, diagonal inner: consecutive MMAs write
              // different accumulators (the int32 sums are exact, so the
              // order does not change any result)
              for (int s = 0; s <= dhi; ++s)
                for (int d = max(dlo, s); d <= dhi; ++d) {
                  const uint64_t ad = core_desc(a0 + (q * ns + s) * OZ_A_PLANE);
                  const uint64_t bd = core_desc(b0 + (q * ns + d - s) * Shape::B_PLANE);
                  const uint32_t acc = (kb + q > 0 || s > 0) ? 1u : 0u;
                  tc_mma_i8(tmem + (uint32_t)((d - dlo) * BN), ad, bd, Shape::IDESC, acc);
                }
            } else {
              for (int d = dlo; d <= dhi; ++d)
                for (int s = 0; s <= d; ++s) {
                  const uint64_t ad = core_desc(a0 + (q * ns + s) * OZ_A_PLANE);
                  const uint64_t bd = core_desc(b0 + (q * ns + d - s) * Shape::B_PLANE);
                  const uint32_t acc = (kb + q > 0 || s > 0) ? 1u : 0u;
                  tc_mma_i8(tmem + (uint32_t)((d - dlo) * BN), ad, bd, Shape::IDESC, acc);
                }
            }
          }
          tc_commit(&empty_bar[st]);
          ++it;
        }
        if (ok) tc_commit(&acc_full);
      }
      // every MMA issued has completed before TMEM is freed
      tc_commit(&drain_bar);
      mbar_wait(&drain_bar, 0, abort, args.flag, true);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue
    // Two epilogue warps per TMEM lane quarter, each owning BN / 2 columns of
    // every accumulator. For BN = 128 with two passes whose second pass needs
    // at most two accumulators, the first pass's FP64 sums are parked in
    // TMEM, in this thread's own (already read) columns of accumulators 2
    // and 3; otherwise each pass after the first adds to C.
    constexpr int HALF = BN / 2;
    const int quarter = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = tm * OZ_BM + quarter * 32 + lane;
    const bool row_ok = row < args.M;
    const double sa = row_ok ? args.scale_a[row] : 0.0;
    const uint32_t mine = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * HALF);
    const int col0 = tn * BN + half * HALF;
    const int nd_last = S - (npass - 1) * ACC;
    const bool park = ACC == 4 && npass == 2 && nd_last <= 2;
    for (int pass = 0; pass < npass; ++pass) {
      const int dlo = pass * ACC, dhi = min(S - 1, dlo + ACC - 1);
      const int nd = dhi - dlo + 1;
      const bool last = pass + 1 == npass;
      int ready = 0;
      if (lane == 0) ready = mbar_wait(&acc_full, pass & 1, abort, args.flag) ? 1 : 0;
      ready = __shfl_sync(0xffffffffu, ready, 0);
      if (!ready) break;
      tc_fence_after();
      double w[ACC];
#pragma unroll
      for (int a = 0; a < ACC; ++a) w[a] = a < nd ? kOzWeight[dlo + a] : 0.0;
#pragma unroll 2
      for (int c = 0; c < HALF / 4; ++c) {
        const uint32_t at = mine + (uint32_t)(c * 4);
        double v[4];
        if (last && park) {
          uint32_t p0[4], p1[4];
          tmem_ld4(at + 2 * BN, p0);
          tmem_ld4(at + 3 * BN, p1);
          pass_sum4<ACC, BN>(at, nd, w, v);  // waits for all loads of this thread
          const double first[4] = {__hiloint2double((int)p0[1], (int)p0[0]),
                                   __hiloint2double((int)p0[3], (int)p0[2]),
                                   __hiloint2double((int)p1[1], (int)p1[0]),
                                   __hiloint2double((int)p1[3], (int)p1[2])};
          if (row_ok) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int col = col0 + c * 4 + j;
              if (col < args.N) {
                const double sb = args.scale_b[col];
                double* dst = args.C + row + (long)col * args.ldc;
                const double f = __dmul_rn(__dmul_rn(first[j], sa), sb);
                const double val = __dmul_rn(__dmul_rn(v[j], sa), sb);
                *dst = args.accumulate ? __dadd_rn(__dadd_rn(*dst, f), val) : __dadd_rn(f, val);
              }
            }
          }
        } else {
          pass_sum4<ACC, BN>(at, nd, w, v);
          if (!last && park) {
            tmem_st4(at + 2 * BN, (uint32_t)__double2loint(v[0]), (uint32_t)__double2hiint(v[0]),
                     (uint32_t)__double2loint(v[1]), (uint32_t)__double2hiint(v[1]));
            tmem_st4(at + 3 * BN, (uint32_t)__double2loint(v[2]), (uint32_t)__double2hiint(v[2]),
                     (uint32_t)__double2loint(v[3]), (uint32_t)__double2hiint(v[3]));
          } else if (row_ok) {
            const bool add = pass > 0 || args.accumulate;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int col = col0 + c * 4 + j;
              if (col < args.N) {
                double* dst = args.C + row + (long)col * args.ldc;
                const double val = __dmul_rn(__dmul_rn(v[j], sa), args.scale_b[col]);
                *dst = add ? __dadd_rn(*dst, val) : val;
              }
            }
          }
        }
      }
      if (!last) {
        if (park) tmem_wait_st();
        tc_fence_before();
        mbar_arrive(&acc_empty);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(OZ_TMEM_COLS)
                 : "memory");
  }
}

// ---------------------------------------------------------- CTA-pair helpers
__device__ __forceinline__ bool mbar_test_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait with cluster-scope acquire (for phases completed by arrivals
// from the other CTA of the pair).
__device__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, volatile int* abort, int* flag) {
  const long long start = clock64();
  while (!mbar_test_cluster(bar, parity)) {
    if (*abort) return false;
    if (clock64() - start > OZ_WAIT_CYCLES) {
      *abort = 1;
      flag_error(flag, 4);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// Shared::cluster address of the same shared variable in CTA `rank`.
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}

__device__ __forceinline__ void mbar_arrive_remote(uint32_t addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(addr) : "memory");
}

// Every thread of both CTAs of the pair.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}

__device__ __forceinline__ void tc_mma_i8_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                               uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrives (once the pair's MMAs issued so far complete) on the barrier at
// this address in both CTAs of the pair.
__device__ __forceinline__ void tc_commit_pair(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(smem_u32(bar)),
      "h"((uint16_t)3)
      : "memory");
}

// CTA-pair form (tcgen05 cta_group::2): a cluster of two CTAs computes a
// 256 x BN tile. CTA r of the pair holds A rows 128 r .. 128 r + 127 and
// B rows (BN / 2) r .. (BN / 2) (r + 1) - 1 of the tile in its own shared
// memory; the leader (r = 0) issues M = 256 MMAs that read both CTAs' halves
// and accumulate each CTA's 128 rows x BN columns in that CTA's TMEM, so each
// SM reads only half of B from shared memory per MMA. Each CTA's producer
// completes its copies on its own full barrier; in the second CTA a relay
// thread forwards each completed stage to the leader (peer_full). The
// leader frees both CTAs' stages, and signals both epilogues, with
// multicast commits; both epilogues release the accumulators to the
// leader's acc_empty. Waits are bounded as in the single-CTA kernel; every
// thread of both CTAs reaches the final cluster barrier.
template <int BN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(OZ_THREADS, 1)
    ozaki_gemm_pair_kernel(const int8_t* __restrict__ digits_a,
                           const int8_t* __restrict__ digits_b, const OzArgs args) {
  using Shape = OzShape<BN>;
  constexpr int ACC = Shape::ACC;
  constexpr int B_HALF = (BN / 2) * OZ_BK;  // this CTA's B plane block
  // s32 accumulator, signed int8 A and B, K-major, N = BN, M = 256
  constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                             ((uint32_t)(256 >> 4) << 24);
  static_assert(BN % 32 == 0, "each CTA holds a multiple of 16 B rows");
  extern __shared__ uint8_t oz_smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[OZ_MAX_STAGES];
  __shared__ __align__(8) uint64_t empty_bar[OZ_MAX_STAGES];
  __shared__ __align__(8) uint64_t peer_full[OZ_MAX_STAGES];
  __shared__ __align__(8) uint64_t acc_full, acc_empty, drain_bar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int abort_s;
  volatile int* abort = &abort_s;

  uint8_t* smem = oz_smem_raw + ((1024 - (smem_u32(oz_smem_raw) & 1023)) & 1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const int pair = blockIdx.x >> 1;
  const int tm = pair / args.tiles_n, tn = pair % args.tiles_n;
  const int S = args.slices;
  const int stages = args.stages;
  const int stage_bytes = S * (OZ_A_PLANE + B_HALF);
  const int npass = (S + ACC - 1) / ACC;

  if (threadIdx.x == 0) {
    for (int i = 0; i < stages; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
      mbar_init(&peer_full[i], 1);
    }
    mbar_init(&acc_full, 1);
    mbar_init(&acc_empty, 2 * 32 * OZ_EPI_WARPS);
    mbar_init(&drain_bar, 1);
    abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(OZ_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  cluster_sync_all();  // barriers of both CTAs initialised before any remote arrival
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------------------------------------------------- producer
      uint32_t it = 0;
      bool ok = true;
      const long a_row = (long)tm * 256 + rank * OZ_BM;
      const long b_row = (long)tn * BN + rank * (BN / 2);
      for (int pass = 0; pass < npass && ok; ++pass) {
        const int dhi = min(S - 1, pass * ACC + ACC - 1);
        const int ns = min(S, dhi + 1);
        const uint32_t bytes = (uint32_t)ns * (OZ_A_PLANE + B_HALF);
        for (int kb = 0; kb < args.kblocks; ++kb) {
          const int st = it % stages;
          if (it >= (uint32_t)stages &&
              !mbar_wait(&empty_bar[st], ((it / stages) - 1) & 1, abort, args.flag)) {
            ok = false;
            break;
          }
          uint8_t* a_dst = smem + st * stage_bytes;
          uint8_t* b_dst = a_dst + S * OZ_A_PLANE;
          mbar_expect_tx(&full_bar[st], bytes);
          const long slab = (long)(args.kb0 + kb) * S;
          for (int j = 0; j < ns; ++j) {
            bulk_load(a_dst + j * OZ_A_PLANE, digits_a + ((slab + j) * args.rows_pa + a_row) * OZ_BK,
                      (uint32_t)OZ_A_PLANE, &full_bar[st]);
            bulk_load(b_dst + j * B_HALF, digits_b + ((slab + j) * args.rows_pb + b_row) * OZ_BK,
                      (uint32_t)B_HALF, &full_bar[st]);
          }
          ++it;
        }
      }
      for (uint32_t j = it > (uint32_t)stages ? it - stages : 0; j < it; ++j)
        mbar_wait(&full_bar[j % stages], (j / stages) & 1, abort, args.flag, true);
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0 && leader) {
      // -------------------------------------------------- MMA issuer (leader)
      uint32_t it = 0;
      bool ok = true;
      for (int pass = 0; pass < npass && ok; ++pass) {
        const int dlo = pass * ACC, dhi = min(S - 1, dlo + ACC - 1);
        if (pass > 0) {
          if (!mbar_wait_cluster(&acc_empty, (pass - 1) & 1, abort, args.flag)) break;
          tc_fence_after();
        }
        for (int kb = 0; kb < args.kblocks; ++kb) {
          const int st = it % stages;
          const uint32_t ph = (it / stages) & 1;
          if (!mbar_wait(&full_bar[st], ph, abort, args.flag) ||
              !mbar_wait_cluster(&peer_full[st], ph, abort, args.flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(smem + st * stage_bytes);
          const uint32_t b0 = a0 + S * OZ_A_PLANE;
          for (int d = dlo; d <= dhi; ++d)
            for (int s = 0; s <= d; ++s) {
              const uint64_t ad = core_desc(a0 + s * OZ_A_PLANE);
              const uint64_t bd = core_desc(b0 + (d - s) * B_HALF);
              const uint32_t acc = (kb > 0 || s > 0) ? 1u : 0u;
              tc_mma_i8_pair(tmem + (uint32_t)((d - dlo) * BN), ad, bd, IDESC, acc);
            }
          tc_commit_pair(&empty_bar[st]);
          ++it;
        }
        if (ok) tc_commit_pair(&acc_full);
      }
      tc_commit_pair(&drain_bar);
      mbar_wait(&drain_bar, 0, abort, args.flag, true);
    } else if (lane == 0) {
      // ------------------------------------------ relay (second CTA of the pair)
      const uint32_t leader_peer_full = cluster_addr(&peer_full[0], 0);
      uint32_t it = 0;
      bool ok = true;
      for (int pass = 0; pass < npass && ok; ++pass)
        for (int kb = 0; kb < args.kblocks; ++kb) {
          const int st = it % stages;
          if (!mbar_wait(&full_bar[st], (it / stages) & 1, abort, args.flag)) {
            ok = false;
            break;
          }
          mbar_arrive_remote(leader_peer_full + (uint32_t)(st * sizeof(uint64_t)));
          ++it;
        }
      // the leader's MMAs write this CTA's TMEM: wait for them before it is freed
      mbar_wait(&drain_bar, 0, abort, args.flag, true);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue
    constexpr int HALF = BN / 2;
    const int quarter = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = tm * 256 + (int)rank * OZ_BM + quarter * 32 + lane;
    const bool row_ok = row < args.M;
    const double sa = row_ok ? args.scale_a[row] : 0.0;
    const uint32_t mine = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * HALF);
    const int col0 = tn * BN + half * HALF;
    const uint32_t leader_acc_empty = cluster_addr(&acc_empty, 0);
    for (int pass = 0; pass < npass; ++pass) {
      const int dlo = pass * ACC, dhi = min(S - 1, dlo + ACC - 1);
      const int nd = dhi - dlo + 1;
      const bool last = pass + 1 == npass;
      int ready = 0;
      if (lane == 0) ready = mbar_wait_cluster(&acc_full, pass & 1, abort, args.flag) ? 1 : 0;
      ready = __shfl_sync(0xffffffffu, ready, 0);
      if (!ready) break;
      tc_fence_after();
      double w[ACC];
#pragma unroll
      for (int a = 0; a < ACC; ++a) w[a] = a < nd ? kOzWeight[dlo + a] : 0.0;
#pragma unroll 2
      for (int c = 0; c < HALF / 4; ++c) {
        double v[4];
        pass_sum4<ACC, BN>(mine + (uint32_t)(c * 4), nd, w, v);
        if (row_ok) {
          const bool add = pass > 0 || args.accumulate;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int col = col0 + c * 4 + j;
            if (col < args.N) {
              double* dst = args.C + row + (long)col * args.ldc;
              const double val = __dmul_rn(__dmul_rn(v[j], sa), args.scale_b[col]);
              *dst = add ? __dadd_rn(*dst, val) : val;
            }
          }
        }
      }
      if (!last) {
        tc_fence_before();
        mbar_arrive_remote(leader_acc_empty);
      }
    }
  }

  tc_fence_before();
  cluster_sync_all();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(OZ_TMEM_COLS)
                 : "memory");
  }
}

// ------------------------------------------------------------------ split
// Byte offset of (row, k) in plane s of the tiled digit layout (k % 4 == 0
// keeps a 4-byte group, k % 16 == 0 a 16-byte group, inside one core row).
__device__ __forceinline__ size_t digit_offset(int row, int k, int s, int slices, int rows_p) {
  return ((size_t)((k >> 5) * slices + s) * rows_p + (row & ~7)) * OZ_BK +
         (size_t)(((k & 31) >> 4) * 128 + (row & 7) * 16 + (k & 15));
}
// x = 2^e (d0 + d1/254 + ...)/127: scaled by 2^-e (exact) and 127, then
// rounded to nearest digit by digit.
__device__ __forceinline__ void split_value(double x, double inv, int slices, int (&d)[kOzakiMaxSlices]) {
  double v = __dmul_rn(__dmul_rn(x, inv), 127.0);
#pragma unroll
  for (int s = 0; s < kOzakiMaxSlices; ++s) {
    if (s < slices) {
      const double r = rint(v);
      d[s] = (int)r;
      v = __dmul_rn(__dsub_rn(v, r), 254.0);
    } else {
      d[s] = 0;
    }
  }
}

__device__ __forceinline__ void row_exponent(double mx, double* inv, double* scale) {
  if (mx > 0.0 && isfinite(mx)) {
    int e = 0;
    frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1): 2^e > mx
    *inv = ldexp(1.0, -e);
    *scale = ldexp(1.0, e);
  } else {
    *inv = 0.0;
    *scale = 1.0;
  }
}

// Block per row; rows stored contiguously (row r at src + r * ld). Each
// thread digitises 16 consecutive values per step and stores one 16-byte
// core-matrix row per digit plane.
constexpr int OZ_SPLIT_THREADS = 128;

__global__ void __launch_bounds__(OZ_SPLIT_THREADS)
    split_rows_kernel(const double* __restrict__ src, long ld, int rows, int k, int k_p,
                      int slices, int8_t* __restrict__ digits, double* __restrict__ scale,
                      int* flag) {
  __shared__ double red[OZ_SPLIT_THREADS / 32];
  const int row = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool live = row < rows;
  const double* x = src + (long)row * ld;
  double mx = 0.0;
  bool bad = false;
  if (live)
    for (int c = threadIdx.x; c < k; c += OZ_SPLIT_THREADS) {
      const double v = x[c];
      bad |= !isfinite(v);
      mx = fmax(mx, fabs(v));
    }
#pragma unroll
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) red[warp] = mx;
  if (__syncthreads_or(bad) && threadIdx.x == 0) flag_error(flag, 1);
  mx = red[0];
#pragma unroll
  for (int w = 1; w < OZ_SPLIT_THREADS / 32; ++w) mx = fmax(mx, red[w]);
  double inv, sc;
  row_exponent(mx, &inv, &sc);
  if (threadIdx.x == 0) scale[row] = sc;
  const int rows_p = gridDim.x;
  for (int c16 = threadIdx.x * 16; c16 < k_p; c16 += OZ_SPLIT_THREADS * 16) {
    uint32_t pk[kOzakiMaxSlices][4];
#pragma unroll
    for (int s = 0; s < kOzakiMaxSlices; ++s) pk[s][0] = pk[s][1] = pk[s][2] = pk[s][3] = 0u;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int c = c16 + j;
      const double v = (live && c < k) ? x[c] : 0.0;
      int d[kOzakiMaxSlices];
      split_value(isfinite(v) ? v : 0.0, inv, slices, d);
#pragma unroll
      for (int s = 0; s < kOzakiMaxSlices; ++s)
        pk[s][j >> 2] |= (uint32_t)(uint8_t)(int8_t)d[s] << (8 * (j & 3));
    }
#pragma unroll
    for (int s = 0; s < kOzakiMaxSlices; ++s)
      if (s < slices)
        *reinterpret_cast<int4*>(digits + digit_offset(row, c16, s, slices, rows_p)) =
            make_int4((int)pk[s][0], (int)pk[s][1], (int)pk[s][2], (int)pk[s][3]);
  }
}

// Row maxima of a scaled column-major matrix (non-negative doubles order as
// their bit patterns, so an integer atomic max is exact and deterministic).
template <class T>
__global__ void colmajor_rowmax(const T* __restrict__ X, int n, int p, long ld,
                                const double* __restrict__ kscale, int cols_per_block,
                                unsigned long long* rowmax, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j0 = blockIdx.y * cols_per_block, j1 = min(p, j0 + cols_per_block);
  double mx = 0.0;
  bool bad = false;
  for (int j = j0; j < j1; ++j) {
    double v = as_f64(X[i + (long)j * ld]);
    if (kscale) v = v * sqrt(kscale[j]);
    bad |= !isfinite(v);
    mx = fmax(mx, fabs(v));
  }
  if (bad) flag_error(flag, 1);
  atomicMax(rowmax + i, (unsigned long long)__double_as_longlong(mx));
}

// 64 x 64 tile: read along rows (coalesced in the column-major source),
// write each row's 16-digit groups per plane into the tiled layout.
template <class T>
__global__ void colmajor_split(const T* __restrict__ X, int n, int p, long ld,
                               const double* __restrict__ kscale,
                               const unsigned long long* __restrict__ rowmax, int rows_p,
                               int k_p, int slices, int8_t* __restrict__ digits,
                               double* __restrict__ scale) {
  __shared__ double tile[64][65];
  const int i0 = blockIdx.x * 64, k0 = blockIdx.y * 64;
  {
    const int ii = threadIdx.x & 63;
    const int i = i0 + ii;
    for (int kk = threadIdx.x >> 6; kk < 64; kk += 4) {
      const int c = k0 + kk;
      double v = 0.0;
      if (i < n && c < p) {
        v = as_f64(X[i + (long)c * ld]);
        if (kscale) v = v * sqrt(kscale[c]);
        if (!isfinite(v)) v = 0.0;
      }
      tile[kk][ii] = v;
    }
  }
  __syncthreads();
  const int ii = threadIdx.x >> 2, kg = (threadIdx.x & 3) * 16;
  const int i = i0 + ii;
  double inv = 0.0, sc = 1.0;
  if (i < n) row_exponent(__longlong_as_double((long long)rowmax[i]), &inv, &sc);
  if (blockIdx.y == 0 && (threadIdx.x & 3) == 0) scale[i] = sc;
  alignas(16) signed char out[kOzakiMaxSlices][16];
#pragma unroll 4
  for (int j = 0; j < 16; ++j) {
    int d[kOzakiMaxSlices];
    split_value(tile[kg + j][ii], inv, slices, d);
#pragma unroll
    for (int s = 0; s < kOzakiMaxSlices; ++s) out[s][j] = (signed char)d[s];
  }
  for (int s = 0; s < slices; ++s)
    *reinterpret_cast<int4*>(digits + digit_offset(i, k0 + kg, s, slices, rows_p)) =
        *reinterpret_cast<const int4*>(out[s]);
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

void prepare(OzakiOperand& out, int rows, int k, int slices, cudaStream_t s) {
  require(slices >= 1 && slices <= kOzakiMaxSlices, "int8 split: 1..7 digits");
  require(rows >= 0 && k >= 0, "int8 split: invalid shape");
  out.rows = rows;
  out.k = k;
  out.rows_p = std::max(OZ_ROWPAD, round_up(rows, OZ_ROWPAD));
  out.k_p = std::max(OZ_KPAD, round_up(k, OZ_KPAD));
  out.slices = slices;
  // a tile may run up to OZ_TAIL bytes past the last plane (rows beyond the
  // padded ones only feed outputs that are never stored)
  const size_t body = (size_t)slices * out.rows_p * out.k_p;
  out.digits.reserve(body + OZ_TAIL, s);
  FPLS_CHECK(cudaMemsetAsync(out.digits.get() + body, 0, OZ_TAIL, s));
  out.scale.reserve((size_t)out.rows_p, s);
}

// Tile shape for a rectangular product: waves of tiles over the SMs (pairs
// over SM pairs) times the measured time of one MMA step of the tile in this
// kernel (B200, 6 digits, k = 5000; clocks per 128 x BN x 32 step, per pair
// step for 256-row CTA-pair tiles). The CTA-pair form measured slower than
// single-CTA tiles at every shape tried, so it runs only when asked for.
struct TileChoice {
  int bn;
  bool pair;
};

TileChoice pick_tile(int M, int N, int tile_n, int pair) {
  struct Cand {
    int bn;
    bool pair;
    double step_clk;
  };
  const Cand cands[] = {{128, false, 177.0}, {192, false, 276.0}, {256, false, 288.0},
                        {192, true, 327.0},  {256, true, 342.0}};
  TileChoice best{128, false};
  double best_cost = -1.0;
  const int sms = num_sms();
  for (const Cand& c : cands) {
    if (c.pair != (pair == 1)) continue;  // pair < 0 (automatic): single-CTA tiles
    if (tile_n > 0 && c.bn != tile_n) continue;
    const long tiles = (long)ceil_div(M, c.pair ? 2 * OZ_BM : OZ_BM) * ceil_div(N, c.bn);
    const long slots = c.pair ? sms / 2 : sms;
    const double cost = (double)((tiles + slots - 1) / slots) * c.step_clk;
    if (best_cost < 0.0 || cost < best_cost) {
      best = {c.bn, c.pair};
      best_cost = cost;
    }
  }
  return best;
}

template <int BN>
bool configure_gemm() {
  static const bool configured = [] {
    FPLS_CHECK(cudaFuncSetAttribute(ozaki_gemm_kernel<BN>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_DATA + 1024));
    return true;
  }();
  return configured;
}

template <int BN>
void launch_gemm(const OzakiOperand& a, const OzakiOperand& b, OzArgs args, long tiles,
                 cudaStream_t stream) {
  const int S = a.slices;
  const int stage_bytes = S * (OZ_A_PLANE + OzShape<BN>::B_PLANE);
  args.stages = std::min(OZ_MAX_STAGES, OZ_DATA / stage_bytes);
  require(args.stages >= 2, "int8 split product: stages do not fit shared memory");
  const size_t smem = (size_t)args.stages * stage_bytes + 1024;
  configure_gemm<BN>();
  // int32 accumulators stay exact while (digit pairs on a diagonal) x k x 127^2 < 2^31
  const int kb_total = a.k_p / OZ_BK;
  const int seg_bytes = std::max(OZ_KPAD, (int)((2147483647LL / (16129LL * S)) / OZ_KPAD * OZ_KPAD));
  const int kb_seg = seg_bytes / OZ_BK;
  for (int kb0 = 0; kb0 < kb_total; kb0 += kb_seg) {
    args.kb0 = kb0;
    args.kblocks = std::min(kb_seg, kb_total - kb0);
    args.accumulate = kb0 > 0 ? 1 : 0;
    ozaki_gemm_kernel<BN><<<(unsigned)tiles, OZ_THREADS, smem, stream>>>(a.digits.get(),
                                                                         b.digits.get(), args);
    count_launch();
    FPLS_LAUNCH("ozaki_gemm_kernel");
  }
}


struct OzTiming {
  bool enabled = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
  std::vector<double> ops;
};
OzTiming& oz_timing() {
  static OzTiming t;
  return t;
}

template <int BN>
void launch_gemm_pair(const OzakiOperand& a, const OzakiOperand& b, OzArgs args, long pairs,
                      cudaStream_t stream) {
  const int S = a.slices;
  const int stage_bytes = S * (OZ_A_PLANE + (BN / 2) * OZ_BK);
  args.stages = std::min(OZ_MAX_STAGES, OZ_DATA / stage_bytes);
  require(args.stages >= 2, "int8 split product: stages do not fit shared memory");
  const size_t smem = (size_t)args.stages * stage_bytes + 1024;
  static const bool configured = [] {
    FPLS_CHECK(cudaFuncSetAttribute(ozaki_gemm_pair_kernel<BN>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_DATA + 1024));
    return true;
  }();
  (void)configured;
  const int kb_total = a.k_p / OZ_BK;
  const int seg_bytes = std::max(OZ_KPAD, (int)((2147483647LL / (16129LL * S)) / OZ_KPAD * OZ_KPAD));
  const int kb_seg = seg_bytes / OZ_BK;
  for (int kb0 = 0; kb0 < kb_total; kb0 += kb_seg) {
    args.kb0 = kb0;
    args.kblocks = std::min(kb_seg, kb_total - kb0);
    args.accumulate = kb0 > 0 ? 1 : 0;
    ozaki_gemm_pair_kernel<BN><<<(unsigned)(2 * pairs), OZ_THREADS, smem, stream>>>(
        a.digits.get(), b.digits.get(), args);
    count_launch();
    FPLS_LAUNCH("ozaki_gemm_pair_kernel");
  }
}

}  // namespace

void ozaki_configure_kernels() {
  configure_gemm<128>();
  configure_gemm<192>();
  configure_gemm<256>();
}

void ozaki_profile_enable(bool on) { oz_timing().enabled = on; }

bool ozaki_profile_enabled() { return oz_timing().enabled; }

void ozaki_reserve(OzakiOperand& out, int rows, int k, int slices, cudaStream_t stream) {
  prepare(out, rows, k, slices, stream);
}

int ozaki_wide_tile(int a_rows, int b_rows) {
  // waves of tiles x the measured clocks of one 128 x BN x 32 step (the
  // single-CTA candidates of pick_tile)
  const int sms = num_sms();
  auto cost = [&](int bn, double step_clk) {
    const long tiles = (long)ceil_div(a_rows, OZ_BM) * ceil_div(b_rows, bn);
    return (double)((tiles + sms - 1) / sms) * step_clk;
  };
  return cost(256, 288.0) <= cost(192, 276.0) ? 256 : 192;
}

void ozaki_profile_read(double* ms, double* int8_ops, unsigned long long* launches) {
  OzTiming& t = oz_timing();
  double total_ms = 0.0, total_ops = 0.0;
  for (size_t k = 0; k < t.events.size(); ++k) {
    float e = 0.f;
    cudaEventSynchronize(t.events[k].second);
    cudaEventElapsedTime(&e, t.events[k].first, t.events[k].second);
    total_ms += e;
    total_ops += t.ops[k];
    cudaEventDestroy(t.events[k].first);
    cudaEventDestroy(t.events[k].second);
  }
  if (ms) *ms = total_ms;
  if (int8_ops) *int8_ops = total_ops;
  if (launches) *launches = t.events.size();
  t.events.clear();
  t.ops.clear();
}

void ozaki_split_rows(const double* src, long ld, int rows, int k, int slices,
                      OzakiOperand& out, int* flag, cudaStream_t stream) {
  prepare(out, rows, k, slices, stream);
  split_rows_kernel<<<out.rows_p, OZ_SPLIT_THREADS, 0, stream>>>(
      src, ld, rows, k, out.k_p, slices, out.digits.get(), out.scale.get(), flag);
  count_launch();
  FPLS_LAUNCH("split_rows_kernel");
}

template <class T>
void ozaki_split_colmajor(const T* X, int n, int p, long ld, const double* kscale,
                          int slices, OzakiOperand& out, int* flag, cudaStream_t stream) {
  prepare(out, n, p, slices, stream);
  DeviceArray<unsigned long long> rowmax((size_t)out.rows_p, stream);
  rowmax.zero(stream);
  const int cols_per_block = 128;
  dim3 g1(ceil_div(std::max(n, 1), 256), ceil_div(std::max(p, 1), cols_per_block));
  colmajor_rowmax<T><<<g1, 256, 0, stream>>>(X, n, p, ld, kscale, cols_per_block, rowmax.get(), flag);
  dim3 g2(out.rows_p / 64, out.k_p / 64);
  colmajor_split<T><<<g2, 256, 0, stream>>>(X, n, p, ld, kscale, rowmax.get(), out.rows_p,
                                           out.k_p, slices, out.digits.get(), out.scale.get());
  count_launch(2);
  FPLS_LAUNCH("colmajor_split");
}

template void ozaki_split_colmajor<float>(const float*, int, int, long, const double*, int,
                                          OzakiOperand&, int*, cudaStream_t);
template void ozaki_split_colmajor<double>(const double*, int, int, long, const double*, int,
                                           OzakiOperand&, int*, cudaStream_t);

void ozaki_gemm(const OzakiOperand& a, const OzakiOperand& b, double* C, long ldc, bool lower,
                int* flag, cudaStream_t stream, int tile_n, int pair) {
  require(a.slices == b.slices && a.slices >= 1 && a.slices <= kOzakiMaxSlices,
          "int8 split product: operands need the same digit count (1..7)");
  require(a.k == b.k && a.k_p == b.k_p, "int8 split product: operands need the same k");
  require(!lower || (&a == &b), "symmetric int8 split product needs one operand");
  require(ldc >= std::max(a.rows, 1), "int8 split product: ldc < rows");
  if (a.rows == 0 || b.rows == 0) return;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (oz_timing().enabled) {
    FPLS_CHECK(cudaEventCreate(&ev0));
    FPLS_CHECK(cudaEventCreate(&ev1));
    FPLS_CHECK(cudaEventRecord(ev0, stream));
  }
  const int S = a.slices;
  require(tile_n == 0 || tile_n == 128 || tile_n == 192 || tile_n == 256,
          "int8 split product: tile width 128, 192 or 256");
  require(!(pair == 1 && ozaki_wait_test().skip_last),
          "int8 split product: the bounded-wait test runs on single-CTA tiles");
  require(!(pair == 1 && (lower || tile_n == 128)),
          "int8 split product: CTA pairs need a rectangular product with 192 or 256 columns");
  const TileChoice tc = lower ? TileChoice{128, false} : pick_tile(a.rows, b.rows, tile_n, pair);
  const int bn = tc.bn;
  OzArgs args{};
  args.M = a.rows;
  args.N = b.rows;
  args.slices = S;
  args.lower = lower ? 1 : 0;
  args.ldc = ldc;
  args.C = C;
  args.scale_a = a.scale.get();
  args.scale_b = b.scale.get();
  args.flag = flag;
  args.rows_pa = a.rows_p;
  args.rows_pb = b.rows_p;
  args.interleave = ozaki_mma_order();
  args.skip_last = ozaki_wait_test().skip_last;
  args.wait_cycles = ozaki_wait_test().cycles > 0 ? ozaki_wait_test().cycles : OZ_WAIT_CYCLES;
  const int tiles_n = ceil_div(b.rows, bn);
  args.tiles_n = tiles_n;
  if (tc.pair) {
    const long pairs = (long)ceil_div(a.rows, 2 * OZ_BM) * tiles_n;
    if (bn == 192)
      launch_gemm_pair<192>(a, b, args, pairs, stream);
    else
      launch_gemm_pair<256>(a, b, args, pairs, stream);
  } else {
    const int tiles_m = ceil_div(a.rows, OZ_BM);
    const long tiles = lower ? (long)tiles_m * (tiles_m + 1) / 2 : (long)tiles_m * tiles_n;
    if (bn == 128)
      launch_gemm<128>(a, b, args, tiles, stream);
    else if (bn == 192)
      launch_gemm<192>(a, b, args, tiles, stream);
    else
      launch_gemm<256>(a, b, args, tiles, stream);
  }
  if (lower) mirror_lower_triangle(C, a.rows, ldc, stream);
  if (ev0) {
    FPLS_CHECK(cudaEventRecord(ev1, stream));
    oz_timing().events.emplace_back(ev0, ev1);
    const double pairs = S * (S + 1) / 2.0;
    oz_timing().ops.push_back(pairs * (lower ? (double)a.rows * (a.rows + 1.0) * a.k
                                             : 2.0 * a.rows * (double)b.rows * a.k));
  }
}

}  // namespace fpls
