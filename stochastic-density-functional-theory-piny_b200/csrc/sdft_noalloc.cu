// sdft_noalloc.cu -- sdft_half_dots_noalloc: per-orbital half-sphere inner
// products computed without allocating any memory.
//
// Who needs it: a host that has already handed the whole device to its own
// memory pool (or runs with a fixed, pre-reserved footprint) cannot let a
// library call cudaMalloc in the middle of its loop, and cannot afford the
// per-call allocations of a context either.  This entry point works on
// device arrays the caller already owns, writes only the caller's output
// array and one static scratch array compiled into this library, and never
// calls an allocating routine.
//
// The sums are the ones the Chebyshev moments path forms in the epilogue of
// its last FFT stage (the reference takes them with ddot over the half
// sphere, stodft/filter.c:492-496 and calc-chempot-chebyshev.c:725-729):
// for orbital s, over all ncoef stored coefficients,
//     out[s] = 2 sum_G (a_re b_re + a_im b_im) - a_re(G0) b_re(G0),
// G0 being the last coefficient of each orbital.  The G0 imaginary parts
// enter the doubled sum as they stand (PINY keeps them at zero).
//
// Scratch: g_partials below holds one partial sum per (orbital, slice of
// the coefficient range).  Every slot a call reads was written earlier in
// the same call, so nothing in it has to start at zero.  Because the array
// is one per device, two calls whose kernels may overlap on one device
// (different streams, or different host threads without ordering) race on
// it and may return wrong sums; order such calls on one stream.
#include <cuda_runtime.h>
#include <mutex>
#include "sdft_internal.h"

namespace {

constexpr int kSlices = 8;             // partial sums per orbital
constexpr int kMaxStates = 1024;       // orbitals per call
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

// 1024 x 8 doubles = 64 KB per device
static __device__ __align__(256) double g_partials[kMaxStates * kSlices];

__global__ void __launch_bounds__(kThreads)
k_half_dot_partials(const double *__restrict__ ar, const double *__restrict__ ai, const double *__restrict__ br,
                    const double *__restrict__ bi, int ncoef, double *__restrict__ part) {
  const int s = blockIdx.y, slice = blockIdx.x;
  const size_t base = (size_t)s * ncoef;
  double acc = 0.0;
  for (int g = slice * kThreads + threadIdx.x; g < ncoef; g += kSlices * kThreads) {
    const double wr = (g == ncoef - 1) ? 1.0 : 2.0;
    acc += wr * ar[base + g] * br[base + g] + 2.0 * ai[base + g] * bi[base + g];
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  __shared__ double red[kThreads / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; w++) t += red[w];
    part[s * kSlices + slice] = t;
  }
}

// fixed summation order: the result does not depend on timing
__global__ void k_half_dot_finish(const double *__restrict__ part, int nstate, double *__restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nstate) return;
  double t = 0.0;
  for (int k = 0; k < kSlices; k++) t += part[s * kSlices + k];
  out[s] = t;
}

std::mutex g_setup_mu;
bool g_loaded[kMaxDevices] = {};

// Device address of g_partials in the current device's context.  The first
// call on a device also loads this file's kernels there (the module load
// that the first lookup may trigger), so that first call should come before
// any stream capture the caller starts.  The address itself is looked up on
// every call, not cached: it belongs to the context current now, and a host
// that reset the device, or calls from another context, gets the address
// that is valid there.  The lookup is a host-side query, not a stream
// operation.
int scratch_for(int dev, double **p) {
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_loaded[dev]) {
      cudaFuncAttributes fa;
      cudaError_t e;
      if ((e = cudaFuncGetAttributes(&fa, k_half_dot_partials)) != cudaSuccess ||
          (e = cudaFuncGetAttributes(&fa, k_half_dot_finish)) != cudaSuccess)
        return sdft::set_error(SDFT_ERR_CUDA, cudaGetErrorString(e));
      g_loaded[dev] = true;
    }
  }
  double *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_partials);
  if (e != cudaSuccess) return sdft::set_error(SDFT_ERR_CUDA, cudaGetErrorString(e));
  *p = ptr;
  return SDFT_OK;
}

}  // namespace

extern "C" int sdft_half_dots_noalloc(const double *a_re, const double *a_im, const double *b_re, const double *b_im,
                                      int ncoef, int nstate, double *out, void *stream) {
  if (!a_re || !a_im || !b_re || !b_im || !out) return sdft::set_error(SDFT_ERR_ARG, "half_dots_noalloc: null pointer");
  if (ncoef < 1 || nstate < 1) return sdft::set_error(SDFT_ERR_ARG, "half_dots_noalloc: ncoef and nstate must be >= 1");
  if (nstate > kMaxStates)
    return sdft::set_error(SDFT_ERR_ARG,
                           "half_dots_noalloc: nstate > 1024 (the static scratch holds 1024 orbitals; "
                           "split the call)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sdft::set_error(SDFT_ERR_NODEVICE, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return sdft::set_error(SDFT_ERR_UNSUPPORTED, "half_dots_noalloc: device index >= 64");
  double *part = nullptr;
  int r = scratch_for(dev, &part);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  k_half_dot_partials<<<dim3(kSlices, nstate), kThreads, 0, st>>>(a_re, a_im, b_re, b_im, ncoef, part);
  k_half_dot_finish<<<(nstate + 127) / 128, 128, 0, st>>>(part, nstate, out);
  if ((e = cudaGetLastError()) != cudaSuccess) return sdft::set_error(SDFT_ERR_CUDA, cudaGetErrorString(e));
  return SDFT_OK;
}
