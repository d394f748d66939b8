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
constexpr int SC_H = 104;          // V^T p (a)

using Fit = PersistentFit;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Arrival: releases this CTA's earlier writes (ordered before it by the CTA
// barrier) and acquires those released by earlier arrivals, in one atomic.
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void red_add_release(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Barrier of the fit's CTAs with a deterministic reduction of their
// partials (slots 0 .. count-1 of each CTA's row of cpart). Every thread of
// the CTA calls it after writing its partials; the reducing CTA calls
// store(k, sum) in the thread of slot k, then (after a CTA barrier) after(),
// and releases everyone. Returns false when a wait ran out (flag set to 5);
// the caller returns.
//
// Up to kFlatSlots slots: every CTA arrives at one counter and the last one
// reduces, Q = PT / count threads per slot, thread q of slot k summing CTAs
// q, q + Q, ... in order, then the Q sums in order. Wider reductions arrive
// in groups of kBarGroup CTAs: the last CTA of a group sums the group's
// partials (thread k: slot k, the group's CTAs in order) into its row of
// gpart and arrives at the top counter; the last group's reducer sums the
// group rows in order.
constexpr int kBarGroup = 32;
constexpr int kFlatSlots = 64;
template <class S, class A>
__device__ bool group_sync(const Fit& f, int* flag, unsigned& epoch, int count, S&& store, A&& after) {
  __shared__ int role_s, ok_s;  // role: 0 waits, 1 reduced its group, 2 reduces all
  // per-thread sums of the flat reduction: dynamic shared memory past psm and
  // hs (the ring is idle at barriers; a static array would be duplicated per
  // instantiation)
  extern __shared__ __align__(16) double dyn_smem[];
  double* const part_s = dyn_smem + kSmemDoubles + kPersistMaxComponents;
  const bool flat = count <= kFlatSlots;
  const int cta = (int)blockIdx.x - f.cta0;
  const int g = cta / kBarGroup;
  const int ngroups = (f.C + kBarGroup - 1) / kBarGroup;
  const int gsize = min(kBarGroup, f.C - g * kBarGroup);
  // the generation after this barrier (every CTA passes the same barriers)
  const unsigned target = epoch + 1u;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok_s = 1;
    if (flat) role_s = atom_add_acq_rel(f.bar, 1u) == (unsigned)f.C - 1u ? 2 : 0;
    else role_s = atom_add_acq_rel(f.bar + 2 + g, 1u) == (unsigned)gsize - 1u ? 1 : 0;
  }
  __syncthreads();
  if (role_s == 1) {
    for (int k = threadIdx.x; k < count; k += PT) {
      const double* src = f.cpart + (long)g * kBarGroup * f.cslots + k;
      double sum = 0.0;
#pragma unroll 8
      for (int c = 0; c < gsize; ++c) sum += __ldcg(src + (long)c * f.cslots);
      f.gpart[(long)g * f.cslots + k] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      st_relaxed(f.bar + 2 + g, 0u);
      if (atom_add_acq_rel(f.bar, 1u) == (unsigned)ngroups - 1u) role_s = 2;
    }
    __syncthreads();
  }
  if (role_s == 2) {
    if (flat) {
      if (count > 0) {
        const int Q = PT / count;
        const int t = threadIdx.x;
        if (t < Q * count) {
          const int k = t % count, q = t / count;
          double sum = 0.0;
#pragma unroll 8
          for (int c = q; c < f.C; c += Q) sum += __ldcg(f.cpart + (long)c * f.cslots + k);
          part_s[t] = sum;
        }
        __syncthreads();
        for (int k = t; k < count; k += PT) {
          double sum = 0.0;
          for (int q = 0; q < Q; ++q) sum += part_s[q * count + k];
          store(k, sum);
        }
      }
    } else {
      for (int k = threadIdx.x; k < count; k += PT) {
        double sum = 0.0;
        for (int q = 0; q < ngroups; ++q) sum += __ldcg(f.gpart + (long)q * f.cslots + k);
        store(k, sum);
      }
    }
    __syncthreads();
    after();
    __syncthreads();
    if (threadIdx.x == 0) {
      st_relaxed(f.bar, 0u);
      red_add_release(f.bar + 1, 1u);
    }
  } else if (threadIdx.x == 0) {
    const long long t0 = clock64();
    while ((int)(ld_acquire(f.bar + 1) - target) < 0) {
      if (clock64() - t0 > f.barrier_cycles) {
        flag_error(flag, 5);
        ok_s = 0;
        break;
      }
      __nanosleep(32);
    }
  }
  __syncthreads();
  epoch = target;
  return ok_s != 0;
}

// Barrier without partials.
__device__ __forceinline__ bool group_sync(const Fit& f, int* flag, unsigned& epoch) {
  return group_sync(f, flag, epoch, 0, [](int, double) {}, [] {});
}

// CTA-level sum; every thread receives it.
__device__ __forceinline__ double cta_sum(double v, double* red) { return block_sum(v, red); }

// Contiguous column range [j0, j1) of CTA `c` out of C over p columns.
__device__ __forceinline__ void col_range(int p, int C, int c, int& j0, int& j1) {
  const int per = (p + C - 1) / C;
  j0 = min(p, c * per);
  j1 = min(p, j0 + per);
}

// ---------------------------------------------------------------------------
// Streaming passes over X. Each CTA owns a region of X: a row block of
// f.rb rows (block rbk = cta % Cr) times a column range of f.pc columns
// (range crg = cta / Cr). A pass streams the region through a ring of
// shared-memory stages of Ring<T>::kCols column segments, one cp.async.bulk
// copy per segment (its 16-byte aligned cover, or for the segments at the
// two ends of X its aligned interior, the rows outside it read from global
// memory by the consumers) completing on the stage's mbarrier. Warps consume
// the stages independently; the last warp done with a stage refills its
// slot. The scores pass walks the region's columns forward, the loading
// pass backward, so the stages read last by one pass are read first by the
// next while they are still in L2. The partition and the order of every sum
// depend on (n, p) only: every storage type sums in the same order.

constexpr int kBlockRows = 512;   // largest row block (rows of a segment)
constexpr int kAuxDoubles = 1024; // rt of the region's columns / t of its rows

// Stage geometry per storage type: kCols column segments of kBlockRows
// rows, kStages stages, about 100 KB of ring per CTA so that two CTAs fit
// an SM. Each stage carries 8192 elements (16 per thread, 4096 for FP64)
// so that the per-stage handshake is small beside the consume work.
// EXTRA: bytes a stage carries after its column segments (the projection's
// slice of R; 0 for the fit).
template <class T, int EXTRA = 0>
struct Ring {
  static constexpr int kColStride = kBlockRows * (int)sizeof(T) + 16;
  static constexpr int kCols = sizeof(T) == 8 ? 8 : 16;
  static constexpr int kStageBytes = kCols * kColStride + EXTRA;
  static constexpr int kStages = sizeof(T) == 2 ? 5 : 3;
  static constexpr int kBytes = kStages * kStageBytes;
  static constexpr int kDynBytes = kBytes + kAuxDoubles * (int)sizeof(double);
};
// No extra copy per stage.
struct NoExtra {
  __device__ void operator()(int, const void*& src, unsigned& bytes) const {
    src = nullptr;
    bytes = 0;
  }
};
constexpr int kMaxRingStages = 8;
static_assert(kBlockRows == 2 * PT, "the scores pass gives each thread two rows of a block");
static_assert(Ring<bf16>::kBytes >= (kSmemDoubles + kPersistMaxComponents + PT) * 8 &&
                  Ring<float>::kBytes >= (kSmemDoubles + kPersistMaxComponents + PT) * 8 &&
                  Ring<double>::kBytes >= (kSmemDoubles + kPersistMaxComponents + PT) * 8,
              "the vector phases and barriers use the first kSmemDoubles + kPersistMaxComponents + PT "
              "doubles of the ring");
static_assert(Ring<bf16>::kCols <= 32 && Ring<float>::kCols <= 32 && Ring<double>::kCols <= 32 &&
                  Ring<float>::kCols % (PT / 32) == 0 && Ring<double>::kCols % (PT / 32) == 0 &&
                  Ring<bf16>::kCols % (PT / 32) == 0,
              "one lane per column segment when issuing; whole columns per warp when loading");

inline int round_up(long v, long m) { return (int)((v + m - 1) / m * m); }

__device__ __forceinline__ uint32_t smem_u32(const void* ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void ring_bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void ring_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// One try of the wait; the thread may sleep up to 20 us in it (the
// suspend-time hint) until the phase completes, instead of spinning.
__device__ __forceinline__ bool ring_try(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
      : "memory");
  return done != 0;
}
// Bounded wait for the phase of `parity` to complete (false on expiry).
__device__ __forceinline__ bool ring_wait(uint64_t* bar, unsigned parity) {
  if (ring_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!ring_try(bar, parity))
    if (clock64() - t0 > kBarrierCycles) return false;
  return true;
}
__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <class T>
__device__ __forceinline__ T tzero() {
  return T(0);
}
template <>
__device__ __forceinline__ bf16 tzero<bf16>() {
  return __ushort_as_bfloat16((unsigned short)0);
}

// The region of this CTA.
struct Region {
  long r0;   // first row
  int rows;  // rows of the row block
  int rbk;   // row block
  int c0;    // first column
  int cols;  // columns of the range (0 for an empty trailing range)
  int crg;   // column range
  int nst;   // stages per pass
  int off0;  // byte offset mod 16 of (row r0, column 0) of X
  int offc;  // byte offset mod 16 added per column
  bool ends; // holds the first or the last segment of X (plain-loaded rows)
  // byte offset mod 16 of the region's segment of column col
  __device__ __forceinline__ int off(int col) const { return (off0 + col * offc) & 15; }
};

template <class T>
__device__ __forceinline__ Region region_of(const Fit& f, int cta) {
  Region g;
  g.rbk = cta % f.Cr;
  g.crg = cta / f.Cr;
  g.r0 = (long)g.rbk * f.rb;
  g.rows = (int)min((long)f.rb, (long)f.n - g.r0);
  g.c0 = min(f.p, g.crg * f.pc);
  g.cols = min(f.pc, f.p - g.c0);
  g.nst = (g.cols + Ring<T>::kCols - 1) / Ring<T>::kCols;
  const int es = f.elem;
  g.off0 = (int)((reinterpret_cast<uintptr_t>(f.X) + (uintptr_t)g.r0 * es) & 15);
  g.offc = (int)(((uintptr_t)f.ld * es) & 15);
  // whether an aligned cover leaves X: the region's segments ascend with
  // the column, so its first and last segments decide
  g.ends = false;
  if (g.cols > 0) {
    const uintptr_t x0 = reinterpret_cast<uintptr_t>(f.X);
    const uintptr_t x1 = x0 + ((uintptr_t)(f.p - 1) * f.ld + f.n) * es;
    const uintptr_t first = x0 + ((uintptr_t)g.c0 * f.ld + g.r0) * es;
    const uintptr_t last = x0 + ((uintptr_t)(g.c0 + g.cols - 1) * f.ld + g.r0 + g.rows) * es;
    g.ends = (first & ~(uintptr_t)15) < x0 || ((last + 15) & ~(uintptr_t)15) > x1;
  }
  return g;
}

// Byte geometry of one column segment (rows r0 .. r0 + rows - 1 of column
// col, element r at byte off + r * sizeof(T) of its slot). The copy is the
// segment's 16-byte aligned cover [lo, hi) when that lies inside X (the
// neighbouring bytes belong to other columns or row blocks and are not
// used); otherwise (the first and last segments of X, at most) the aligned
// interior [lo, hi) plus plain loads of the rows [0, head) and [tail0, rows).
struct Segment {
  uintptr_t g, lo, hi;
  int off;
  int head, tail0;
};

template <class T>
__device__ __forceinline__ Segment segment(const Fit& f, const T* X, const Region& g, int col) {
  Segment sg;
  sg.g = reinterpret_cast<uintptr_t>(X + (long)col * f.ld + g.r0);
  const uintptr_t end = sg.g + (uintptr_t)g.rows * sizeof(T);
  sg.off = (int)(sg.g & 15);
  const uintptr_t x0 = reinterpret_cast<uintptr_t>(X);
  const uintptr_t x1 = reinterpret_cast<uintptr_t>(X + (long)(f.p - 1) * f.ld + f.n);
  sg.lo = sg.g & ~(uintptr_t)15;
  sg.hi = (end + 15) & ~(uintptr_t)15;
  if (sg.lo >= x0 && sg.hi <= x1) {
    sg.head = 0;
    sg.tail0 = g.rows;
  } else {
    sg.lo = (sg.g + 15) & ~(uintptr_t)15;
    sg.hi = end & ~(uintptr_t)15;
    sg.head = (int)min((uintptr_t)g.rows, (sg.lo - sg.g) / sizeof(T));
    sg.tail0 = sg.hi > sg.lo ? (int)((sg.hi - sg.g) / sizeof(T)) : sg.head;
  }
  return sg;
}

// Whether stage st holds a segment whose cover leaves X (the region's
// first or last segments only; the same test as Region::ends per stage).
template <class T>
__device__ __forceinline__ bool stage_ends(const Fit& f, const T* X, const Region& g, int st) {
  if (!g.ends) return false;
  const int cb = g.c0 + st * Ring<T>::kCols;
  const int ce = min(g.c0 + g.cols, cb + Ring<T>::kCols) - 1;
  const uintptr_t x0 = reinterpret_cast<uintptr_t>(X);
  const uintptr_t x1 = reinterpret_cast<uintptr_t>(X + (long)(f.p - 1) * f.ld + f.n);
  const uintptr_t first = reinterpret_cast<uintptr_t>(X + (long)cb * f.ld + g.r0);
  const uintptr_t last = reinterpret_cast<uintptr_t>(X + (long)ce * f.ld + g.r0 + g.rows);
  return (first & ~(uintptr_t)15) < x0 || ((last + 15) & ~(uintptr_t)15) > x1;
}

// Warp 0: the bulk copies of stage `st` into `slot`, one lane per column,
// completing on `bar`; lane G::kCols copies the stage's extra bytes, if any,
// behind the segments.
template <class G, class T, class E = NoExtra>
__device__ void issue_stage(const Fit& f, const T* X, const Region& g, int st, unsigned char* slot,
                            uint64_t* bar, const E& extra = E()) {
  const int lane = threadIdx.x & 31;
  const int nc = min(G::kCols, g.cols - st * G::kCols);
  Segment sg;
  unsigned bytes = 0;
  const void* xsrc = nullptr;
  if (lane < nc) {
    sg = segment(f, X, g, g.c0 + st * G::kCols + lane);
    if (sg.hi > sg.lo) bytes = (unsigned)(sg.hi - sg.lo);
  } else if (lane == G::kCols) {
    extra(st, xsrc, bytes);
  }
  unsigned total = bytes;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
  if (lane == 0) ring_expect(bar, total);
  __syncwarp();
  if (bytes > 0) {
    if (lane < nc)
      bulk_to_smem(slot + lane * G::kColStride + sg.off + ((long)sg.lo - (long)sg.g),
                   reinterpret_cast<const void*>(sg.lo), bytes, bar);
    else
      bulk_to_smem(slot + G::kCols * G::kColStride, xsrc, bytes, bar);
  }
}

// Streams the region's stages through the ring: issues the first stages,
// runs prepare() (whole CTA) while they are in flight, then calls
// consume(stage, slot) in every warp for each stage in order (forward or
// backward). Warps run
// through the stages independently: the last warp done with a stage
// refills its slot with the stage kStages ahead (done[slot] counts the
// warps, reset by that warp). `seq` numbers the CTA's stages across passes
// (slot seq % stages, mbarrier parity (seq / stages) & 1). Returns false
// when a stage never arrived (flag 5 set, the copies in flight waited for).
template <class G, class T, class P, class F, class E = NoExtra>
__device__ bool stream_region(const Fit& f, const T* X, const Region& g, bool backward,
                              unsigned& seq, unsigned char* ring, uint64_t* bars, unsigned* done,
                              unsigned* issued, int* flag, P&& prepare, F&& consume,
                              const E& extra = E()) {
  constexpr int NS = G::kStages;
  constexpr unsigned kWarps = PT / 32;
  const int nst = g.nst;
  const int lane = threadIdx.x & 31;
  auto stage_of = [&](int k) { return backward ? nst - 1 - k : k; };
  auto slot_of = [&](int k) { return ring + (size_t)((seq + k) % NS) * G::kStageBytes; };
  __syncthreads();  // the ring is free (earlier passes and phases are done with it)
  if (threadIdx.x < 32) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    for (int k = 0; k < min(NS, nst); ++k)
      issue_stage<G>(f, X, g, stage_of(k), slot_of(k), bars + (seq + k) % NS, extra);
    if (lane == 0) *issued = (unsigned)min(NS, nst);
  }
  prepare();  // (whole CTA) while the first stages are in flight
  __syncthreads();
  bool ok = true;
  for (int k = 0; k < nst; ++k) {
    const unsigned sl = (seq + k) % NS;
    ok = __all_sync(0xffffffffu, ring_wait(bars + sl, ((seq + k) / NS) & 1u));
    if (!ok) break;
    consume(stage_of(k), (const unsigned char*)slot_of(k));
    __syncwarp();
    unsigned prev = 0;
    if (lane == 0) {
      __threadfence_block();
      prev = atomicAdd(done + sl, 1u);
    }
    prev = __shfl_sync(0xffffffffu, prev, 0);
    if (prev == kWarps - 1) {
      // every warp is done with the slot: refill it
      __threadfence_block();
      if (lane == 0) done[sl] = 0u;
      if (k + NS < nst) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_stage<G>(f, X, g, stage_of(k + NS), slot_of(k), bars + sl, extra);
        if (lane == 0) atomicAdd(issued, 1u);
      }
    }
  }
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) {
      flag_error(flag, 5);
      // the last stages issued may still be in flight
      const int last = (int)*issued;
      for (int j = max(0, last - NS); j < last; ++j) ring_wait(bars + (seq + j) % NS, ((seq + j) / NS) & 1u);
      for (int j = 0; j < NS; ++j) done[j] = 0u;
    }
    return false;
  }
  seq += (unsigned)nst;
  return true;
}

// Dominant eigenpair of the m x m Gram in A (shared, symmetric; whole CTA;
// B, C, v shared scratch): scal[SC_Z..] = s z / sqrt(lambda), sign fixed so
// the largest |z| entry is positive (as direction_kernel), and
// scal[SC_C] = z . u with u (shared, m) = S^T (mean / scale).
__device__ void direction_step(const Fit& f, const double* A, double* B, double* C, double* v,
                               const double* u, int* flag) {
  const int m = f.m;
  double lam = 0.0;
  const bool found = dominant_pair(A, B, C, v, m, lam);
  if (threadIdx.x == 0) {
    const bool ok = found && lam > 0.0 && isfinite(lam);
    if (!ok) flag_error(flag, 1);
    const double inv = ok ? 1.0 / sqrt(lam) : 0.0;
    int arg = 0;
    if (found)
      for (int k = 1; k < m; ++k)
        if (fabs(v[k]) > fabs(v[arg])) arg = k;
    const double sgn = found && v[arg] < 0.0 ? -1.0 : 1.0;
    double cz = 0.0;
    for (int k = 0; k < m; ++k) {
      const double zk = found ? sgn * v[k] * inv : 0.0;
      f.scal[SC_Z + k] = zk;
      cz = fma(zk, u[k], cz);
    }
    f.scal[SC_C] = cz;
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
__global__ void __launch_bounds__(PT, 2)
    persistent_simpls(const Fit* __restrict__ fits, int nfits) {
  // dynamic: the ring of the streaming passes, then kAuxDoubles (rt / t);
  // the vector phases use its first kSmemDoubles doubles as psm
  extern __shared__ __align__(16) double psm[];
  __shared__ __align__(8) uint64_t ring_bars[kMaxRingStages];
  __shared__ unsigned ring_done[kMaxRingStages], ring_issued;
  __shared__ double red[32];
  __shared__ double zs[kPersistMaxResponses];
  __shared__ double sv[kPersistMaxResponses];
  __shared__ double scal_s[4];
  int fi = 0;
  while (fi + 1 < nfits && (int)blockIdx.x >= fits[fi + 1].cta0) ++fi;
  const Fit& f = fits[fi];  // read through the read-only path as needed (fewer live registers)
  int* const flag = f.flag;
  const int cta = (int)blockIdx.x - f.cta0;
  if (cta == f.absent_cta) return;  // bounded-wait test only
  const T* X = static_cast<const T*>(f.X);
  const int n = f.n, p = f.p, m = f.m, C = f.C;
  const int tid = threadIdx.x;
  int j0, j1;
  col_range(p, C, cta, j0, j1);

  unsigned char* const ring = reinterpret_cast<unsigned char*>(psm);
  double* const aux = reinterpret_cast<double*>(ring + Ring<T>::kBytes);
  const Region rg = region_of<T>(f, cta);
  unsigned seq = 0;  // stages streamed by this CTA so far
  unsigned bar_epoch = 0;  // group barriers passed
  if (tid == 0) {
    for (int k = 0; k < Ring<T>::kStages; ++k) {
      ring_bar_init(ring_bars + k);
      ring_done[k] = 0u;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  const int G = m * (m + 1) / 2;
  // partials of the Gram of S and of u = S^T (mean / scale) over this CTA's
  // columns, before the first component (S = S0)
  gram_u_partials(f, cta, j0, j1, -1, 0.0, sv, psm);
  for (int a = 0; a < f.a; ++a) {
    // B0: Gram and u of the (deflated) S, the direction z / sqrt(lambda), and
    // the score offset c = mean . (S z / scale) = z . u
    {
      double* A = psm;               // m x m Gram
      double* B = A + m * m;         // squaring scratch
      double* Cs = B + m * m;        // m^2 + 1
      double* vd = Cs + m * m + 1;   // dominant eigenvector (m + 1)
      double* us = vd + m + 1;       // u
      auto store = [&](int k, double v) {
        if (k < G) {
          int c = (int)((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
          while (c * (c + 1) / 2 > k) --c;
          while ((c + 1) * (c + 2) / 2 <= k) ++c;
          const int d = k - c * (c + 1) / 2;
          A[c + d * m] = v;
          A[d + c * m] = v;
          f.gpk[k] = v;
        } else {
          us[k - G] = v;
        }
      };
      if (!group_sync(f, flag, bar_epoch, G + m, store, [&] { direction_step(f, A, B, Cs, vd, us, flag); })) return;
    }
    for (int c = tid; c < m; c += PT) zs[c] = __ldcg(f.scal + SC_Z + c);
    __syncthreads();
    // P2: score partials of the region, t_part[crg][rows] = X[rows, cols] rt[cols]
    // with rt = (S z) / scale (S is not deflated until P7)
    {
      // thread rows tid and tid + 256 of the row block (kBlockRows = 2 PT);
      // each row's sum over the region's columns runs as four interleaved
      // sums (column j into sum j % 4) added at the end, a fixed order
      constexpr int SC = Ring<T>::kCols;
      double acc0[4] = {0.0, 0.0, 0.0, 0.0}, acc1[4] = {0.0, 0.0, 0.0, 0.0};
      const int r1 = tid + PT;
      const bool in0 = tid < rg.rows, in1 = r1 < rg.rows;
      auto rt = [&] {
        for (int j = tid; j < rg.cols; j += PT) {
          double rv = 0.0;
          for (int c = 0; c < m; ++c) rv = fma(__ldcg(f.S + rg.c0 + j + (long)c * p), zs[c], rv);
          aux[j] = rv / f.scale[rg.c0 + j];
        }
      };
      const bool ok = stream_region<Ring<T>>(f, X, rg, false, seq, ring, ring_bars, ring_done, &ring_issued, flag, rt,
                                    [&](int st, const unsigned char* slot) {
        const int nc = min(SC, rg.cols - st * SC);
        const double* w = aux + st * SC;
        const int cb = rg.c0 + st * SC;
        if (nc == SC && !stage_ends(f, X, rg, st)) {
          // the stage's values kept in the storage type (fewer registers,
          // all loads ahead of the FMAs); rows past the block read stale
          // shared memory and their sums are never stored
          T x0[SC], x1[SC];
#pragma unroll
          for (int c = 0; c < SC; ++c) {
            const T* col = reinterpret_cast<const T*>(slot + c * Ring<T>::kColStride + rg.off(cb + c));
            x0[c] = col[tid];
            x1[c] = col[r1];
          }
#pragma unroll
          for (int c = 0; c < SC; ++c) {
            const double wc = w[c];
            acc0[c & 3] = fma(as_f64(x0[c]), wc, acc0[c & 3]);
            acc1[c & 3] = fma(as_f64(x1[c]), wc, acc1[c & 3]);
          }
        } else {
          for (int c4 = 0; c4 < nc; c4 += 4) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int c = c4 + u;
              if (c >= nc) break;
              const T* col = reinterpret_cast<const T*>(slot + c * Ring<T>::kColStride + rg.off(cb + c));
              const Segment sg = segment(f, X, rg, cb + c);
              const T* gcol = X + (long)(cb + c) * f.ld + rg.r0;  // rows outside the copy
              const double wc = w[c];
              if (in0) acc0[u] = fma(as_f64(tid < sg.head || tid >= sg.tail0 ? gcol[tid] : col[tid]), wc, acc0[u]);
              if (in1) acc1[u] = fma(as_f64(r1 < sg.head || r1 >= sg.tail0 ? gcol[r1] : col[r1]), wc, acc1[u]);
            }
          }
        }
      });
      if (!ok) return;
      double* out = f.tpart + (long)rg.crg * n + rg.r0;
      if (tid < rg.rows) out[tid] = (acc0[0] + acc0[1]) + (acc0[2] + acc0[3]);
      if (r1 < rg.rows) out[r1] = (acc1[0] + acc1[1]) + (acc1[2] + acc1[3]);
    }
    if (!group_sync(f, flag, bar_epoch)) return;
    // P4: loading partials of the region, p_part[rbk][cols] = X[rows, cols]^T t[rows],
    // the stages backward. While the first stages are in flight each CTA
    // forms t for its row block: t = sum of the column ranges' partials - c
    // (the CTAs of column range 0 also store T[:, a] and the |t|^2, sum t
    // partials of their block).
    {
      const double cc = __ldcg(f.scal + SC_C);
      double* tcol = f.T + (long)a * n + rg.r0;
      auto tv = [&] {
        double s2 = 0.0, s1 = 0.0;
        for (int r = tid; r < rg.rows; r += PT) {
          const long i = rg.r0 + r;
          // eight interleaved partial sums (more loads in flight), fixed order
          double q[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) q[u] = 0.0;
          int k = 0;
          for (; k + 7 < f.Cc; k += 8) {
#pragma unroll
            for (int u = 0; u < 8; ++u) q[u] += __ldcg(f.tpart + (long)(k + u) * n + i);
          }
          for (; k < f.Cc; ++k) q[0] += __ldcg(f.tpart + (long)k * n + i);
          const double t = (((q[0] + q[1]) + (q[2] + q[3])) + ((q[4] + q[5]) + (q[6] + q[7]))) - cc;
          aux[r] = t;
          if (rg.crg == 0) {
            tcol[r] = t;
            s2 = fma(t, t, s2);
            s1 += t;
          }
        }
        for (int r = rg.rows + tid; r < kBlockRows; r += PT) aux[r] = 0.0;
        if (rg.crg == 0) {
          s2 = cta_sum(s2, red);
          s1 = cta_sum(s1, red);
        }
        if (tid == 0) {
          f.cpart[(long)cta * f.cslots] = rg.crg == 0 ? s2 : 0.0;
          f.cpart[(long)cta * f.cslots + 1] = rg.crg == 0 ? s1 : 0.0;
        }
      };
      const int lane = tid & 31, warp = tid >> 5;
      // each warp takes CPW columns of the stage; per column four
      // interleaved sums over the rows in a fixed order, then the warp tree
      constexpr int SC = Ring<T>::kCols;
      constexpr int CPW = SC / (PT / 32);
      const bool ok = stream_region<Ring<T>>(f, X, rg, true, seq, ring, ring_bars, ring_done, &ring_issued, flag, tv,
                                    [&](int st, const unsigned char* slot) {
        const int nc = min(SC, rg.cols - st * SC);
        const int cb = rg.c0 + st * SC;
        double q[CPW][4];
        const T* col[CPW];
#pragma unroll
        for (int j = 0; j < CPW; ++j) {
          const int cl = warp * CPW + j;
          col[j] = reinterpret_cast<const T*>(slot + cl * Ring<T>::kColStride + rg.off(cb + cl));
#pragma unroll
          for (int u = 0; u < 4; ++u) q[j][u] = 0.0;
        }
        // rows lane + 32 u + 128 i (i < kBlockRows / 128) into sum u of each
        // column, a fixed order; past the block's rows t is staged as zero
        // and x selected as zero, so those terms add exactly nothing
        constexpr int RI = kBlockRows / 128;
        if (!stage_ends(f, X, rg, st)) {
#pragma unroll
          for (int i = 0; i < RI; ++i) {
            double tv[4];
            T xr[CPW][4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int r = lane + 128 * i + 32 * u;
              tv[u] = aux[r];
#pragma unroll
              for (int j = 0; j < CPW; ++j) xr[j][u] = r < rg.rows ? col[j][r] : tzero<T>();
            }
#pragma unroll
            for (int j = 0; j < CPW; ++j)
#pragma unroll
              for (int u = 0; u < 4; ++u) q[j][u] = fma(as_f64(xr[j][u]), tv[u], q[j][u]);
          }
        } else {
#pragma unroll
          for (int j = 0; j < CPW; ++j) {
            const int cl = warp * CPW + j;
            if (cl >= nc) continue;
            const Segment sg = segment(f, X, rg, cb + cl);
            const T* gcol = X + (long)(cb + cl) * f.ld + rg.r0;  // rows outside the copy
#pragma unroll
            for (int i = 0; i < RI; ++i)
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int r = lane + 128 * i + 32 * u;
                const double x =
                    r < rg.rows ? as_f64(r < sg.head || r >= sg.tail0 ? gcol[r] : col[j][r]) : 0.0;
                q[j][u] = fma(x, aux[r], q[j][u]);
              }
          }
        }
#pragma unroll
        for (int j = 0; j < CPW; ++j) {
          const int cl = warp * CPW + j;
          const double v = warp_sum((q[j][0] + q[j][1]) + (q[j][2] + q[j][3]));
          if (lane == 0 && cl < nc) f.ppart[(long)rg.rbk * p + cb + cl] = v;
        }
      });
      if (!ok) return;
    }
    if (!group_sync(f, flag, bar_epoch, 2, [&](int k, double v) { f.scal[k == 0 ? SC_T2 : SC_ST] = v; }, [] {}))
      return;
    // P5: p, R[:, a] = (S z) / |t|; partial V^T p (a) and S0^T R[:, a] (m).
    // The column partials are loaded while thread 0 fetches |t|^2 and sum t.
    if (tid == 0) {
      scal_s[0] = __ldcg(f.scal + SC_T2);
      scal_s[1] = __ldcg(f.scal + SC_ST);
    }
    double* ps = psm;          // p values of this CTA's columns (<= 2048)
    double* rs = psm + 2048;   // R values
    for (int jl = tid; jl < j1 - j0; jl += PT) {
      const int j = j0 + jl;
      // sum u takes the row blocks k = u (mod 4) in order; eight loads per step
      double q0 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0;
      int k = 0;
      for (; k + 7 < f.Cr; k += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldcg(f.ppart + (long)(k + u) * p + j);
        q0 += v[0];
        q1 += v[1];
        q2 += v[2];
        q3 += v[3];
        q0 += v[4];
        q1 += v[5];
        q2 += v[6];
        q3 += v[7];
      }
      for (; k + 3 < f.Cr; k += 4) {
        q0 += __ldcg(f.ppart + (long)k * p + j);
        q1 += __ldcg(f.ppart + (long)(k + 1) * p + j);
        q2 += __ldcg(f.ppart + (long)(k + 2) * p + j);
        q3 += __ldcg(f.ppart + (long)(k + 3) * p + j);
      }
      for (; k < f.Cr; ++k) q0 += __ldcg(f.ppart + (long)k * p + j);
      double rv = 0.0;
      for (int c = 0; c < m; ++c) rv = fma(__ldcg(f.S + j + (long)c * p), zs[c], rv);
      ps[jl] = (q0 + q1) + (q2 + q3);
      rs[jl] = rv;
    }
    __syncthreads();
    if (tid == 0) {
      const double tn = sqrt(scal_s[0]);
      const bool ok = tn > 0.0 && isfinite(tn);
      if (!ok && cta == 0) flag_error(flag, 1);
      scal_s[2] = ok ? 1.0 / tn : 0.0;
    }
    __syncthreads();
    const double inv_t = scal_s[2], sum_t = scal_s[1];
    for (int jl = tid; jl < j1 - j0; jl += PT) {
      const int j = j0 + jl;
      const double pj = (ps[jl] - f.mean[j] * sum_t) / f.scale[j] * inv_t;
      const double rj = rs[jl] * inv_t;
      f.pv[j] = pj;
      f.R[j + (long)a * p] = rj;
      ps[jl] = pj;
      rs[jl] = rj;
    }
    __syncthreads();
    {
      // three of a warp's dot products at once (their loads in flight
      // together); each is the lane-strided sum then the warp tree
      const int lane = tid & 31, warp = tid >> 5;
      const int cols = j1 - j0;
      constexpr int W = PT / 32;
      for (int kb = warp; kb < a + m; kb += 3 * W) {
        double sd[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          const int k = kb + e * W;
          if (k >= a + m) continue;
          const double* src = k < a ? f.V + (long)k * p + j0 : f.S0 + (long)(k - a) * p + j0;
          const double* w = k < a ? ps : rs;
          for (int jl = lane; jl < cols; jl += 32) sd[e] = fma(__ldcg(src + jl), w[jl], sd[e]);
        }
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          const int k = kb + e * W;
          const double v = warp_sum(sd[e]);
          if (lane == 0 && k < a + m) f.cpart[(long)cta * f.cslots + k] = v;
        }
      }
    }
    if (!group_sync(f, flag, bar_epoch, a + m,
                    [&](int k, double v) {
                      if (k < a) {
                        f.scal[SC_H + k] = v;
                      } else {
                        f.scal[SC_Q + k - a] = v;
                        f.Q[(k - a) + (long)a * m] = v;
                      }
                    },
                    [] {}))
      return;
    // P6: v = p - V h; partial v.v and S^T v
    double* const hs = psm + kSmemDoubles;  // V^T p (a), beside psm in the idle ring
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
    if (!group_sync(f, flag, bar_epoch, 1 + m,
                    [&](int k, double v) {
                      if (k == 0) f.scal[SC_VV] = v;
                      else f.scal[SC_SV + k - 1] = v;
                    },
                    [] {}))
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

// ---------------------------------------------------------------------------
// Projection X R (n x p times p x nb, nb <= NB <= 16) in one pass over X: the
// regions and ring of the fit's scores pass, each stage also carrying the
// matching rows of Rt (R row-major, NB doubles per row, zero past nb) behind
// its column segments. Each thread keeps its two rows' NB sums over the
// region's columns in order; part[(range * nb + b) * n + row] receives them
// (the column ranges are summed in order afterwards). A normal launch: CTAs
// never wait on each other.
constexpr int kRSlice = 16 * 16 * 8;  // bytes of Rt a stage can carry (16 rows x 16)

template <class T, int NB>
__global__ void __launch_bounds__(PT, 2)
    xr_ring_kernel(const Fit f, const double* __restrict__ Rt, int nb, double* __restrict__ part) {
  using G = Ring<T, kRSlice>;
  constexpr int SC = G::kCols;
  static_assert(NB % 2 == 0 && NB <= 16 && SC * NB * 8 <= kRSlice, "Rt slice of a stage");
  extern __shared__ __align__(16) double psm[];
  __shared__ __align__(8) uint64_t ring_bars[kMaxRingStages];
  __shared__ unsigned ring_done[kMaxRingStages], ring_issued;
  const T* X = static_cast<const T*>(f.X);
  const int tid = threadIdx.x;
  unsigned char* const ring = reinterpret_cast<unsigned char*>(psm);
  const Region rg = region_of<T>(f, blockIdx.x);
  if (tid == 0) {
    for (int k = 0; k < G::kStages; ++k) {
      ring_bar_init(ring_bars + k);
      ring_done[k] = 0u;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  unsigned seq = 0;
  double acc0[NB], acc1[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) acc0[b] = acc1[b] = 0.0;
  const int r1 = tid + PT;
  const bool in0 = tid < rg.rows, in1 = r1 < rg.rows;
  auto extra = [&](int st, const void*& src, unsigned& bytes) {
    const int cb = rg.c0 + st * SC;
    const int nc = min(SC, rg.cols - st * SC);
    src = Rt + (long)cb * NB;
    bytes = (unsigned)(nc * NB * (int)sizeof(double));
  };
  const bool ok = stream_region<G>(f, X, rg, false, seq, ring, ring_bars, ring_done, &ring_issued, f.flag,
                                   [] {}, [&](int st, const unsigned char* slot) {
    const int nc = min(SC, rg.cols - st * SC);
    const int cb = rg.c0 + st * SC;
    const double* rs = reinterpret_cast<const double*>(slot + SC * G::kColStride);
    if (nc == SC && !stage_ends(f, X, rg, st)) {
      // rows past the block read stale shared memory; their sums are never stored
#pragma unroll 2
      for (int c = 0; c < SC; ++c) {
        const T* col = reinterpret_cast<const T*>(slot + c * G::kColStride + rg.off(cb + c));
        const double x0 = as_f64(col[tid]), x1 = as_f64(col[r1]);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const double w = rs[c * NB + b];
          acc0[b] = fma(x0, w, acc0[b]);
          acc1[b] = fma(x1, w, acc1[b]);
        }
      }
    } else {
      for (int c = 0; c < nc; ++c) {
        const T* col = reinterpret_cast<const T*>(slot + c * G::kColStride + rg.off(cb + c));
        const Segment sg = segment(f, X, rg, cb + c);
        const T* gcol = X + (long)(cb + c) * f.ld + rg.r0;  // rows outside the copy
        const double x0 = in0 ? as_f64(tid < sg.head || tid >= sg.tail0 ? gcol[tid] : col[tid]) : 0.0;
        const double x1 = in1 ? as_f64(r1 < sg.head || r1 >= sg.tail0 ? gcol[r1] : col[r1]) : 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const double w = rs[c * NB + b];
          acc0[b] = fma(x0, w, acc0[b]);
          acc1[b] = fma(x1, w, acc1[b]);
        }
      }
    }
  }, extra);
  if (!ok) return;
  double* out = part + (long)rg.crg * nb * f.n + rg.r0;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    if (b < nb) {
      if (in0) out[(long)b * f.n + tid] = acc0[b];
      if (in1) out[(long)b * f.n + r1] = acc1[b];
    }
  }
}

// Rt[j * NB + b] = R[j + b * ldr] for b < nb, 0 for nb <= b < NB.
__global__ void transpose_rows(const double* __restrict__ R, long ldr, int p, int nb, int NB,
                               double* __restrict__ Rt) {
  const long total = (long)p * NB;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < total; k += (long)gridDim.x * blockDim.x) {
    const int j = (int)(k / NB), b = (int)(k % NB);
    Rt[k] = b < nb ? R[j + (long)b * ldr] : 0.0;
  }
}

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

namespace {

// Regions of a fit of n x p: Cr row blocks of rb rows times Cc column ranges
// of pc columns (a function of the shape only); false when the shape does
// not fit the persistent launch.
bool persistent_grid(int n, int p, int& Cr, int& Cc, int& rb, int& pc) {
  const long elems = (long)n * p;
  // about 2^15 elements per CTA: one CTA streams a few tens of GB/s, so
  // even small fits spread over many SMs (the barriers cost little more)
  const int c0 = (int)std::max(1L, std::min<long>(2L * num_sms(), (elems + (1L << 15) - 1) >> 15));
  Cr = (n + kBlockRows - 1) / kBlockRows;
  rb = round_up((n + Cr - 1) / Cr, 8);
  Cr = (n + rb - 1) / rb;
  Cc = std::max(c0 / Cr, (p + kAuxDoubles - 1) / kAuxDoubles);
  pc = (p + Cc - 1) / Cc;
  return (long)Cr * Cc <= 2L * num_sms();
}

}  // namespace

int persistent_ctas(int n, int p) {
  int Cr, Cc, rb, pc;
  return persistent_grid(n, p, Cr, Cc, rb, pc) ? Cr * Cc : 0;
}

namespace {

template <class T>
int capacity_of() {
  static const int cap = [] {
    int v = 0, coop = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
        cudaFuncSetAttribute(persistent_simpls<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Ring<T>::kDynBytes) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, persistent_simpls<T>, PT,
                                                      Ring<T>::kDynBytes) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    return v >= 2 ? v * num_sms() : 0;
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
  int Cr, Cc, rb, pc;
  if (!persistent_grid(n, p, Cr, Cc, rb, pc)) return false;
  const int C = Cr * Cc;
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
  f.Cr = Cr;
  f.Cc = Cc;
  f.rb = rb;
  f.pc = pc;
  f.cslots = std::max(a + m, std::max(1 + m, m * (m + 1) / 2 + m));
  const PersistentWaitTest& wt = persistent_wait_test();
  f.barrier_cycles = wt.cycles > 0 ? wt.cycles : kBarrierCycles;
  f.absent_cta = wt.absent ? 0 : -1;

  // scratch of this fit (stream-ordered, freed behind the launch); the
  // kernel forms the Gram of S itself (into gpk) before the first component
  plan.elem = (int)sizeof(T);
  f.elem = (int)sizeof(T);
  plan.S = std::move(S);
  f.S = plan.S.get();
  plan.part.allocate((size_t)Cc * n + (size_t)Cr * p, stream);
  f.tpart = plan.part.get();
  f.ppart = f.tpart + (size_t)Cc * n;
  const int ngroups = (C + kBarGroup - 1) / kBarGroup;
  plan.cpart.allocate((size_t)(C + ngroups) * f.cslots, stream);
  plan.scal.allocate((size_t)SC_H + kPersistMaxComponents + 8, stream);
  plan.bar.allocate(2 + ngroups, stream);
  plan.bar.zero(stream);
  f.cpart = plan.cpart.get();
  f.gpart = f.cpart + (size_t)C * f.cslots;
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
  const int dyn = elem == 2 ? Ring<bf16>::kDynBytes
                : elem == 4 ? Ring<float>::kDynBytes
                            : Ring<double>::kDynBytes;
  FPLS_CHECK(cudaLaunchCooperativeKernel(fn, dim3(total), dim3(PT), args, (size_t)dyn, stream));
  count_launch();
  FPLS_LAUNCH("persistent_simpls");
  // the descriptors are freed stream-ordered, behind the launch
}

namespace {

// out[i + b ldo] = sum over the column ranges k (in order) of
// part[(k nb + b) n + i] - offset[b].
__global__ void ring_finish(const double* __restrict__ part, int ranges, int n, int nb,
                            const double* offset, double* out, long ldo) {
  const long total = (long)n * nb;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % n), b = (int)(idx / n);
    double v = 0.0;
    for (int k = 0; k < ranges; ++k) v += part[((long)k * nb + b) * n + i];
    if (offset) v -= offset[b];
    out[i + (long)b * ldo] = v;
  }
}

template <class T, int NB>
void launch_xr_ring(const Fit& f, const double* Rt, int nb, double* part, cudaStream_t s) {
  const int dyn = Ring<T, kRSlice>::kBytes;
  static const bool configured = [dyn] {
    FPLS_CHECK(cudaFuncSetAttribute(xr_ring_kernel<T, NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    return true;
  }();
  (void)configured;
  xr_ring_kernel<T, NB><<<f.C, PT, dyn, s>>>(f, Rt, nb, part);
  count_launch();
  FPLS_LAUNCH("xr_ring_kernel");
}

}  // namespace

template <class T>
bool xr_ring(const T* X, int n, int p, long ld, const double* R, long ldr, int nb,
             const double* offset, double* out, long ldo, int* flag, cudaStream_t s) {
  if (nb < 3 || nb > 16 || n < 1 || p < 1) return false;
  const int NB = nb <= 4 ? 4 : nb <= 8 ? 8 : nb <= 10 ? 10 : nb <= 12 ? 12 : 16;
  // row blocks of at most kBlockRows rows, about one wave of two CTAs per SM
  int Cr = (n + kBlockRows - 1) / kBlockRows;
  const int rb = round_up((n + Cr - 1) / Cr, 8);
  Cr = (n + rb - 1) / rb;
  const int Cc = std::max(1, 2 * num_sms() / Cr);
  Fit f{};
  f.X = X;
  f.ld = ld;
  f.n = n;
  f.p = p;
  f.Cr = Cr;
  f.rb = rb;
  f.Cc = Cc;
  f.pc = (p + Cc - 1) / Cc;
  f.C = Cr * Cc;
  f.elem = (int)sizeof(T);
  f.flag = flag;
  DeviceArray<double> Rt((size_t)p * NB, s), part((size_t)Cc * nb * n, s);
  const long tot = (long)p * NB;
  transpose_rows<<<(unsigned)std::min<long>((tot + 255) / 256, 8L * num_sms()), 256, 0, s>>>(R, ldr, p, nb, NB,
                                                                                            Rt.get());
  count_launch();
  FPLS_LAUNCH("transpose_rows");
  switch (NB) {
    case 4: launch_xr_ring<T, 4>(f, Rt.get(), nb, part.get(), s); break;
    case 8: launch_xr_ring<T, 8>(f, Rt.get(), nb, part.get(), s); break;
    case 10: launch_xr_ring<T, 10>(f, Rt.get(), nb, part.get(), s); break;
    case 12: launch_xr_ring<T, 12>(f, Rt.get(), nb, part.get(), s); break;
    default: launch_xr_ring<T, 16>(f, Rt.get(), nb, part.get(), s); break;
  }
  const long total = (long)n * nb;
  ring_finish<<<(unsigned)std::min<long>((total + 255) / 256, 8L * num_sms()), 256, 0, s>>>(
      part.get(), Cc, n, nb, offset, out, ldo);
  count_launch();
  FPLS_LAUNCH("ring_finish");
  return true;
}

template bool xr_ring<float>(const float*, int, int, long, const double*, long, int, const double*,
                             double*, long, int*, cudaStream_t);
template bool xr_ring<double>(const double*, int, int, long, const double*, long, int, const double*,
                              double*, long, int*, cudaStream_t);
template bool xr_ring<bf16>(const bf16*, int, int, long, const double*, long, int, const double*,
                            double*, long, int*, cudaStream_t);

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
