// sdft_xc.cu -- LDA exchange-correlation potential and energy on the
// real-space grid, the xc step of cpGetVksStodft
// (stodft/reduced-energy/cp-energy-ee-rho-stodft.c:838-870): excpot_pz_lda
// (Perdew-Zunger 1981, energy/cp/xc_functionals.c:268) and excpot_pw_lda
// (Perdew-Wang 1992, :378), spin-unpolarised, no LYP.
//
// Per grid point (rho clamped to 1e-10 where not positive):
//   rs = (3 / (4 pi rho))^(1/3),  x = -(3 rho / pi)^(1/3)  (exchange potential),
//   PZ81:  rs >= 1: c = g / (1 + b1 sqrt(rs) + b2 rs),
//                   mu = c (1 + 7/6 b1 sqrt(rs) + 4/3 b2 rs) / (1 + b1 sqrt(rs) + b2 rs);
//          rs <  1: c = a ln rs + b + c' rs ln rs + d rs,
//                   mu = a ln rs + (b - a/3) + 2/3 c' rs ln rs + (2 d - c')/3 rs;
//   PW92:  q1 = 2 A (b1 rs^1/2 + b2 rs + b3 rs^3/2 + b4 rs^2), L = ln(1 + 1/q1),
//          c = -2 A (1 + a1 rs) L,
//          mu = -2 A (1 + 2/3 a1 rs) L
//               - 2 A rs (1 + a1 rs) q1' / (3 q1 (1 + q1)),
//          q1' = 2 A (b1 / (2 sqrt rs) + b2 + 3/2 b3 sqrt rs + 2 b4 rs);
//   v_ks += x + mu;   E_xc = (3/4 sum x rho + sum c rho) vol / N,
//   mu_xc = sum (x + mu) rho vol / N.
// Grid sums are deterministic (fixed block partials, summed in block order).
#include <cuda_runtime.h>
#include <cmath>
#include "sdft_internal.h"

namespace sdft {
namespace {

constexpr int kXcBlocks = 296, kXcThreads = 256;

template <int KIND>
__global__ void __launch_bounds__(kXcThreads) k_xc_lda(const double *__restrict__ rho, double *__restrict__ vks,
                                                       long long n, double *__restrict__ part) {
  double sx = 0.0, sc = 0.0, sv = 0.0;
  const double pi = M_PI, third = 1.0 / 3.0;
  for (long long i = blockIdx.x * (long long)kXcThreads + threadIdx.x; i < n; i += (long long)kXcBlocks * kXcThreads) {
    double r = rho[i];
    if (r <= 0.0) r = 1.0e-10;
    const double rs = pow(3.0 / (4.0 * pi * r), third);
    const double sq = sqrt(rs);
    const double x = -pow(3.0 * r / pi, third);
    double c, mu;
    if (KIND == SDFT_XC_PZ_LDA) {
      const double g = -0.14230, b1 = 1.05290, b2 = 0.33340;
      const double a = 0.03110, b = -0.0480, cc = 0.00200, d = -0.01160;
      if (rs >= 1.0) {
        const double f1 = 1.0 + b1 * sq + b2 * rs;
        const double f2 = 1.0 + (7.0 / 6.0) * b1 * sq + (4.0 / 3.0) * b2 * rs;
        c = g / f1;
        mu = c * (f2 / f1);
      } else {
        const double l = log(rs);
        c = a * l + b + cc * rs * l + d * rs;
        mu = a * l + (b - third * a) + 2.0 * third * cc * rs * l + third * (2.0 * d - cc) * rs;
      }
    } else {
      const double A = 0.03109070, a1 = 0.213700, b1 = 7.59570, b2 = 3.58760, b3 = 1.63820, b4 = 0.492940;
      const double q1 = 2.0 * A * (b1 * sq + b2 * rs + b3 * pow(rs, 1.5) + b4 * rs * rs);
      const double dq = 2.0 * A * (0.5 * b1 / sq + b2 + 1.5 * b3 * sq + 2.0 * b4 * rs);
      const double lg = log(1.0 + 1.0 / q1);
      const double op = 1.0 + a1 * rs;
      c = -2.0 * A * op * lg;
      mu = -2.0 * A * (1.0 + 2.0 * a1 * rs / 3.0) * lg + (-2.0 * A) * rs * op / (3.0 * q1 * (1.0 + q1)) * dq;
    }
    vks[i] += x + mu;
    sx += x * r;
    sc += c * r;
    sv += (x + mu) * r;
  }
  __shared__ double sh[3][kXcThreads];
  sh[0][threadIdx.x] = sx;
  sh[1][threadIdx.x] = sc;
  sh[2][threadIdx.x] = sv;
  __syncthreads();
  for (int h = kXcThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
      for (int k = 0; k < 3; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[(size_t)threadIdx.x * kXcBlocks + blockIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_xc_sum(const double *__restrict__ part, double *__restrict__ out) {
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int b = 0; b < kXcBlocks; b++) s += part[(size_t)threadIdx.x * kXcBlocks + b];
    out[threadIdx.x] = s;
  }
}

}  // namespace
}  // namespace sdft

using namespace sdft;

extern "C" int sdft_xc_lda_dev(int kind, long long n, const double *rho, double *vks, double vol, double *exc,
                               double *muxc, void *stream) {
  if (n < 1 || !rho || !vks || (kind != SDFT_XC_PZ_LDA && kind != SDFT_XC_PW_LDA))
    return set_error(SDFT_ERR_ARG, "xc_lda_dev: bad argument");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(SDFT_ERR_NODEVICE, "xc_lda_dev: no device");
  void *buf = nullptr;
  int r = dev_alloc(dev, stream, &buf, (3 * kXcBlocks + 4) * sizeof(double));
  if (r) return r;
  double *part = static_cast<double *>(buf), *sums = part + 3 * kXcBlocks;
  if (kind == SDFT_XC_PZ_LDA)
    k_xc_lda<SDFT_XC_PZ_LDA><<<kXcBlocks, kXcThreads, 0, st>>>(rho, vks, n, part);
  else
    k_xc_lda<SDFT_XC_PW_LDA><<<kXcBlocks, kXcThreads, 0, st>>>(rho, vks, n, part);
  k_xc_sum<<<1, 32, 0, st>>>(part, sums);
  double h[3] = {0.0, 0.0, 0.0};
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, sums, sizeof h, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  dev_free(buf, stream);
  if (e != cudaSuccess) return set_error(SDFT_ERR_CUDA, cudaGetErrorString(e));
  const double scale = vol / (double)n;
  if (exc) *exc = (0.75 * h[0] + h[1]) * scale;
  if (muxc) *muxc = h[2] * scale;
  return SDFT_OK;
}
