// sdft_gemm_oz.cuh -- FP64-accurate GEMM on INT8 tensor cores (Ozaki
// scheme) for the Kleinman-Bylander projection and back projection of the
// mixed-precision filter.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace sdft {

// A matrix of `rows` x K doubles in digit form: every row carries a
// power-of-two scale 2^E (E chosen so that all |x| < 2^E) and four signed
// 8-bit digits per value,
//     x ~= 2^E * 2^-27 * (d0 2^21 + d1 2^14 + d2 2^7 + d3),  d_s in [-64, 64],
// i.e. 28 bits relative to the row's largest element (the representation
// error is below 2^-28 of it).  Digits are stored slice-major:
// dig[s*rows*ld + row*ld + k], ld a multiple of 64, zero for k >= K.
constexpr int kOzSlices = 4;

// Digit formats.  OZ_7x4 (above): 4 signed 7-bit digits, 28 bits.  OZ_8x3:
// 3 digits of 8 bits, the first signed (floor of x 2^(7-E), in [-128, 127])
// and two unsigned (floor of the remainder times 2^8, in [0, 255]),
//     x ~= 2^E * 2^-23 * (d0 2^16 + d1 2^8 + d2),
// truncation below 2^-23 of the row's scale; products with s + t <= 2
// (6 of 9), int32 accumulation exact for K ranges up to 16384.  Used where
// the result is stored in FP32 (the back projection).
enum OzFmt : int { OZ_7x4 = 0, OZ_8x3 = 1 };
__host__ __device__ constexpr int oz_slices(int fmt) { return fmt == OZ_8x3 ? 3 : 4; }

// out[n*ldo + m] = sum_k A[m][k] B[n][k] over the digit products of the
// format (OZ_7x4: s + t <= 3, 10 of the 16; the rest lie below 2^-28 of
// the leading term).  Every product is an exact int8 x int8 -> int32
// tensor-core MMA; the digit orders are accumulated exactly in TMEM
// accumulators and combined exactly in 64-bit integers, so a K range
// contributes an exactly representable FP64 value and the only rounding is
// the FP64 sum of split-K partials.  A: M x K (M multiple of 128), B: N x K
// (N multiple of bn); only m < Mst, n < Nst are stored.
struct OzGemm {
  CUtensorMap tA, tB;
  int M, N, K, ldo, Mst, Nst;
  const double *sa, *sb;  // row scales 2^E of A (M) and B (N)
  int fmt = OZ_7x4;       // digit format of both operands
  int bn = 128;           // output columns per tile (128 or 64; tB's box height, N a multiple of it)
};

bool gemm_oz_available();
// tensor map of a digit array [oz_slices(fmt)][rows][ld] (int8, K-major)
// box_rows: the rows of one TMA box (128 for A operands, the tile width bn for B)
int make_tmap_oz(CUtensorMap *tm, const int8_t *dig, int rows, int ld, int fmt = OZ_7x4, int box_rows = 128);
// split == 1: out = result; split > 1: FP64 partial z at out + z*split_stride.
// The K tiles are dealt out evenly, which can leave fewer partials than
// asked for (e.g. 32 over 206 K tiles: 7 each, 30 partials); *split_used
// (nullable) receives the count written, the one a reduction must sum.
int run_gemm_oz(const OzGemm &g, int split, double *out, size_t split_stride, int *err, cudaStream_t st,
                int *split_used = nullptr);
// the same with FP32 output (rounded once from the exact FP64 tile value)
int run_gemm_oz(const OzGemm &g, int split, float *out, size_t split_stride, int *err, cudaStream_t st,
                int *split_used = nullptr);
// split count for `tiles` output tiles over `ktiles` K tiles (<= max_split)
int oz_choose_split(int tiles, int ktiles, int max_split);
// the fewest K splits that keep every K range within the format's exact
// int32 accumulation limit
int oz_min_split(int K, int fmt);
// Bounded-wait self-test: one thread waits on an mbarrier that nothing
// arrives at, through the GEMMs' mbar_wait capped at `polls` polls; it gives
// up and sets *err (the GEMMs' device error word).  polls <= kSelftestMaxPolls.
constexpr long long kSelftestMaxPolls = 1ll << 22;
void launch_selftest_wait(int *err, long long polls, cudaStream_t st);
// rowmax[r] = bits of max_k |x[r][k]| (zeroed first); rows x cols, pitch ldx
void launch_oz_rowmax(const double *x, int ldx, int rows, int cols, unsigned long long *rowmax, cudaStream_t st);
// digits (row pitch ld, slice pitch slice_stride bytes) + scales of rows x
// cols doubles under the row maxima in rowmax
void launch_oz_slice(const double *x, int ldx, int rows, int cols, const unsigned long long *rowmax, int8_t *dig,
                     int ld, size_t slice_stride, double *scale, cudaStream_t st, int fmt = OZ_7x4);
// the same two passes for the rows of i G_d c formed from c on the fly
// (v: rows of 2 ngp, re then im; gk: G_d per coefficient; 28-bit digits of
// 2 ngp columns), the vector whose projection is dZ/dR_d
// rowmax3[d rows + r] for d = x, y, z in one pass over c (gk: 3 ngp, G_x then G_y, G_z)
void launch_oz_rowmax_igc3(const double *v, const double *gk, int ngp, int ncoef, int rows,
                           unsigned long long *rowmax3, cudaStream_t st);
void launch_oz_slice_igc(const double *v, const double *gk, int ngp, int ncoef, int rows,
                         const unsigned long long *rowmax, int8_t *dig, int ld, size_t slice_stride, double *scale,
                         cudaStream_t st);
// both of the above
void launch_oz_slice_rows(const double *x, int ldx, int rows, int cols, unsigned long long *rowmax, int8_t *dig,
                          int ld, size_t slice_stride, double *scale, cudaStream_t st, int fmt = OZ_7x4);
// out[n*ldo+m] = sum_z part[z*stride + n*ldo + m] (m < Mst, else 0) for
// n < Nst, plus the digit form of each row n (ld = ldo, slice pitch
// dig_stride bytes).  zero_rowmax (nullable): words [0, Nst) set to 0.
void launch_oz_reduce_slice(const double *part, int split, size_t stride, int ldo, int Mst, int Nst, double *out,
                            int8_t *dig, size_t dig_stride, double *scale, unsigned long long *zero_rowmax,
                            cudaStream_t st, int fmt = OZ_7x4);

}  // namespace sdft
