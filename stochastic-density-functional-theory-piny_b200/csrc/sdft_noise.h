// sdft_noise.h -- device generation of the gaussran2 sign sequence.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace sdft {

// Pairs whose phi lies within 1e-9 of a sign change, listed per launch for
// the host to decide; more than this falls back to the host generator.
constexpr int kNoiseMarginCap = 4096;

// Device bytes device_gauss_signs needs as scratch.
size_t noise_scratch_bytes();

// neg[i] = 1 if the i-th value of gaussran2(nran, qseed) is negative, written
// to device memory; *qseed is left where gaussran2 leaves it.  Identical to
// gauss_signs; synchronises `st`.  kernel_launches (may be null) counts the
// kernels issued.
int device_gauss_signs(long long nran, double *qseed, unsigned char *d_neg, void *d_scratch, cudaStream_t st,
                       int *kernel_launches);

}  // namespace sdft
