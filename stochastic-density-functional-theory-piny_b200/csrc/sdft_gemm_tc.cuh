// sdft_gemm_tc.cuh -- TF32x3 tcgen05 GEMM interface (mixed precision KB term).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>

namespace sdft {
// out[n*ldo + m] = sum_k A[m][k] B[n][k]; A: M x K (M multiple of 128),
// B: N x K (N multiple of bn), K multiple of 32; A/B given as TF32 hi/lo
// FP32 tensor maps.  Only m < Mst, n < Nst are stored.
struct TcGemm {
  CUtensorMap tAh, tAl, tBh, tBl;
  int M, N, K, ldo, Mst, Nst, bn;
};
bool gemm_tf32x3_available();
int make_tmap(CUtensorMap *tm, const float *base, int rows, int K, int ld, int box_rows);
// split > 1 or out_hi != nullptr: partials in `part`, FP64 reduction into
// out64 (+ TF32 hi/lo of the result into out_hi/out_lo).
int run_gemm_tf32x3(const TcGemm &gm, int split, float *part, size_t part_elems, double *out64, float *out_hi,
                    float *out_lo, int *err, cudaStream_t st);
void launch_split_tf32(const double *src, int lds, float *hi, float *lo, int ldd, int rows, int cols,
                       cudaStream_t st);
}  // namespace sdft
