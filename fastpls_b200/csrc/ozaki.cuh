// FP64-accurate products on the int8 tensor cores (tcgen05, kind::i8).
//
// Each FP64 operand row is scaled by a power of two 2^e >= max|row| and
// written as S signed 8-bit digits with round-to-nearest:
//     v0 = x 2^-e 127,  d_s = rint(v_s),  v_{s+1} = (v_s - d_s) 254
// so x = 2^e (d_0 + d_1/254 + ... + d_{S-1}/254^{S-1} + r) / 127 with
// |r| <= 1/(2 254^{S-1}). The product of two such rows is the sum over digit
// pairs (s, t); pairs on the same diagonal d = s + t share the weight
// 1 / (127^2 254^d) and are accumulated exactly in int32 by the tensor core
// (|sum| <= (d+1) K 127^2 < 2^31 for K below 2^17). Diagonals d <= S - 1 are
// kept (S (S + 1) / 2 int8 products); the FP64 epilogue combines the exact
// integer sums of the diagonals, smallest weight first, and applies the two
// power-of-two row scales. With S = 6 the product error is below 2^-47 of
// max|a_i| max|b_j| K, which keeps the batched SIMPLS path within 1e-5 of the
// FP64 path at 20 components.
#pragma once

#include "common.cuh"

namespace fpls {

constexpr int kOzakiMaxSlices = 7;

// One operand of the split product: int8 digits of rows_p (64-multiple) rows
// x k_p (64-multiple) columns, zero padded, for each of `slices` digit
// planes, plus one power-of-two scale per row. Layout, tiled for the tensor
// cores: slabs ordered [k-block (32 columns)][plane], each slab the rows_p / 8
// row groups of 2 k-chunks x 8 rows x 16 bytes (core matrices):
//   byte (r, k, s) = ((k/32 * slices + s) * rows_p + r - r%8) * 32
//                    + (k%32)/16 * 128 + (r%8) * 16 + k%16
// so any run of consecutive rows (from a multiple of 8) of one plane and
// k-block is one contiguous block of 32 bytes per row.
struct OzakiOperand {
  DeviceArray<int8_t> digits;
  DeviceArray<double> scale;
  int rows = 0, rows_p = 0, k = 0, k_p = 0, slices = 0;
};

// Rows stored contiguously: row r is src[r * ld + 0 .. k).
void ozaki_split_rows(const double* src, long ld, int rows, int k, int slices,
                      OzakiOperand& out, int* flag, cudaStream_t stream);

// Rows of a column-major n x p matrix X (leading dimension ld), each element
// scaled as X[i, j] * sqrt(kscale[j]) when kscale is given.
template <class T>
void ozaki_split_colmajor(const T* X, int n, int p, long ld,
                          const double* kscale, int slices, OzakiOperand& out,
                          int* flag, cudaStream_t stream);

// C (a.rows x b.rows, column-major, ldc) = A B^T over the split rows of a
// and b (same k, same slices). lower: only tiles on or below the diagonal
// are computed (a and b must be the same operand) and mirrored. tile_n: the
// tile width in columns of C (128, 192, 256; 0 picks one for the shape);
// pair: 1 runs 256-row tiles on CTA pairs (tcgen05 cta_group::2; widths 192
// and 256), 0 or -1 single-CTA 128-row tiles (-1: the automatic choice; the
// pair form measured slower, so it is never chosen automatically). The FP64
// summation order of the epilogue depends only on the width (diagonals are
// combined in passes of four for 128, of two otherwise).
void ozaki_gemm(const OzakiOperand& a, const OzakiOperand& b, double* C,
                long ldc, bool lower, int* flag, cudaStream_t stream, int tile_n = 0,
                int pair = -1);

// Sizes out's buffers for `rows` x k digits (as the split would), so that a
// later split of at most that many rows does not allocate (e.g. inside a
// captured CUDA graph).
void ozaki_reserve(OzakiOperand& out, int rows, int k, int slices, cudaStream_t stream);

// The tile width (192 or 256) of a rectangular product of a_rows x b_rows
// with the fewer waves of measured step cost. Both widths combine the digit
// diagonals in the same FP64 order, so the choice never changes results.
int ozaki_wide_tile(int a_rows, int b_rows);

// Digit count used by the batched CV engine for its products with the
// shared Gram (0 selects the FP64 DMMA path). Process-wide setting.
int& ozaki_slices();
int ozaki_mma_order();

// Test of the bounded waits of the int8 product (single-CTA tiles): with
// skip_last set, every tile's producer withholds its last stage, so the MMA
// issuer's wait for it runs out after `cycles` clocks; the kernel then sets
// its error flag (4), waits for the copies and MMAs it issued, frees TMEM and
// returns. cycles <= 0 keeps the default bound (about 2 s).
struct OzakiWaitTest {
  int skip_last = 0;
  long long cycles = 0;
};
OzakiWaitTest& ozaki_wait_test();

// Timing of the last ozaki_gemm launches (CUDA events), for benchmarks.
// Sets the kernels' launch attributes once (before any stream capture).
void ozaki_configure_kernels();

void ozaki_profile_enable(bool on);
bool ozaki_profile_enabled();
void ozaki_profile_read(double* ms, double* int8_ops, unsigned long long* launches);

}  // namespace fpls
