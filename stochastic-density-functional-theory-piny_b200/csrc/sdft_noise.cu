// sdft_noise.cu -- signs of gaussran2 generated on the device.
//
// genNoiseOrbitalReal (stodft/gen-noise.c:256) draws nstate*N Gaussians with
// gaussran2 (mathlib/mathlib.c:118-165) from one DURAND sequence
// (mathlib/blas_wrappers.f:39-69) and keeps their signs.  DURAND is
// sequential and evaluated in FP64, but its state settles within a few
// hundred draws on the lattice q = Q/128 (Q integer): there every FP64
// operation of the step is exact, so the generator is the integer LCG
//   Q <- 16807 Q mod m,   m = 128 (2^31 - 1) = 2^38 - 2^7,
// the draw is x = fl((Q 2^-38) (1 + 2^-31)), and the state stays on the
// lattice until a draw finds q < 1 or q > 2147483646 (ran_essl's reseed,
// probability ~1e-9 per draw).  The LCG jumps ahead by multiplying with
// 16807^k mod m, so every thread starts its own run of pairs exactly.
//
// Host/device split (device_gauss_signs): the host runs the FP64 generator
// until the state is on the lattice, the kernel covers the remaining pairs;
// a draw that would reseed stops its thread and is reported (first pair),
// the host continues from the exact state there (jump-ahead), runs the
// reseed and the next lattice entry itself and relaunches.  Pairs whose phi
// lies within 1e-9 of a sign change of cos or sin are listed and decided on
// the host by the same libm call as gauss_signs; all other signs follow from
// comparisons of phi, identical on both sides.  The result is byte-for-byte
// gauss_signs.
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>
#include <algorithm>
#include "sdft_internal.h"
#include "sdft_noise.h"

namespace sdft {

namespace {
constexpr uint64_t kMod = (1ull << 38) - 128ull;  // 128 (2^31 - 1)
constexpr uint64_t kMask38 = (1ull << 38) - 1ull;
constexpr uint64_t kQLow = 128ull;                 // q >= 1
constexpr uint64_t kQHigh = 128ull * 2147483646ull;  // q <= 2147483646
constexpr int kChunk = 256;                        // pairs per thread (multiple of 8)
constexpr int kThreads = 256;
constexpr double kTwoM38 = 1.0 / 274877906944.0;  // 2^-38
constexpr double kOnePEp = 1.0000000004656612873077392578125;  // 1 + 2^-31

struct JumpTable {
  uint64_t pow2[48];  // 16807^(2 * 2^j) mod m: advance by 2^j pairs
};

__host__ __device__ inline uint64_t fold38(uint64_t r) {  // r < 2^46 -> r mod m
  r = (r & kMask38) + (r >> 38) * 128ull;                   // < 2^38 + 2^15
  return r >= kMod ? r - kMod : r;
}

__host__ __device__ inline uint64_t lcg_step(uint64_t q) {  // 16807 q mod m, q < m
  return fold38(16807ull * q);                               // product < 2^53
}

__host__ __device__ inline uint64_t mulmod(uint64_t a, uint64_t b) {  // a, b < m
  const unsigned __int128 x = (unsigned __int128)a * b;               // < 2^76
  const uint64_t lo = (uint64_t)x & kMask38, hi = (uint64_t)(x >> 38);  // hi < 2^38
  return fold38(lo + hi * 128ull);                                  // < 2^46
}

__host__ __device__ inline uint64_t jump(uint64_t q, unsigned long long pairs, const JumpTable &jt) {
  for (int j = 0; pairs && j < 48; ++j, pairs >>= 1)
    if (pairs & 1ull) q = mulmod(q, jt.pow2[j]);
  return q;
}

JumpTable make_jump_table() {
  JumpTable jt;
  uint64_t a = lcg_step(lcg_step(1ull));  // 16807^2
  for (int j = 0; j < 48; ++j) {
    jt.pow2[j] = a;
    a = mulmod(a, a);
  }
  return jt;
}

__device__ inline double draw(uint64_t q) {  // x of a DURAND step that produced state q
  return __dmul_rn(__ull2double_rn(q) * kTwoM38, kOnePEp);
}

// bytes of one pair from (r, phi); bit 2 set = phi near a sign change of cos/sin
__device__ inline unsigned pair_code(double r, double phi) {
  if (r >= 1.0) return 0u;  // r == 1 after clipping: al = 0, both values +0
  const double d = 1e-9;
  unsigned c;
  if (phi > 0.25 + d && phi < 0.75 - d) c = 1u;
  else if (phi < 0.25 - d || (phi > 0.75 + d && phi < 1.0 - d)) c = 0u;
  else return 4u;
  if (phi > 0.5 + d && phi < 1.0 - d) c |= 1u << 8;
  else if (!(phi > d && phi < 0.5 - d)) return 4u;
  return c;
}

// Pairs [p0, pend) of the sign sequence; thread t covers the aligned run of
// kChunk pairs (p0 / kChunk + t) * kChunk ... clipped to [p0, pend).  q0: the
// lattice state entering pair p0.  Group of 8 pairs = 16 bytes, stored as one
// vector when the whole group is inside the thread's range and below nran.
__global__ void __launch_bounds__(kThreads) k_noise_signs(uint64_t q0, long long p0, long long pend, long long nran,
                                                          JumpTable jt, unsigned char *__restrict__ neg, int vec_ok,
                                                          unsigned long long *__restrict__ stop,
                                                          int *__restrict__ nmargin, long long *__restrict__ mpair,
                                                          double *__restrict__ mphi, int mcap) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long a0 = (p0 / kChunk + t) * kChunk;
  const long long beg = a0 > p0 ? a0 : p0;
  const long long end = (a0 + kChunk) < pend ? (a0 + kChunk) : pend;
  if (beg >= end) return;
  uint64_t q = jump(q0, (unsigned long long)(beg - p0), jt);
  unsigned long long w0 = 0, w1 = 0;  // bytes of pairs 0..3 and 4..7 of the current group
  long long gbeg = beg;               // first pair of the current group held in w0/w1
  long long p = beg;
  for (; p < end; ++p) {
    if (q < kQLow || q > kQHigh) break;
    q = lcg_step(q);
    const double r = draw(q);
    if (q < kQLow || q > kQHigh) break;
    q = lcg_step(q);
    const double phi = draw(q);
    unsigned c = pair_code(r, phi);
    if (c & 4u) {
      const int k = atomicAdd(nmargin, 1);
      if (k < mcap) { mpair[k] = p; mphi[k] = phi; }
      c = 0u;
    }
    const int i = (int)(p & 7);
    if (i < 4) w0 |= (unsigned long long)c << (16 * i);
    else w1 |= (unsigned long long)c << (16 * (i - 4));
    if (i == 7 || p + 1 == end) {
      const long long g = p & ~7ll;
      if (vec_ok && gbeg == g && i == 7 && 2 * (g + 8) <= nran) {
        *reinterpret_cast<ulonglong2 *>(neg + 2 * g) = make_ulonglong2(w0, w1);
      } else {
        for (long long u = gbeg; u <= p; ++u) {
          const int j = (int)(u & 7);
          const unsigned v = (unsigned)(((j < 4 ? w0 : w1) >> (16 * (j & 3))) & 0xffffull);
          neg[2 * u] = (unsigned char)(v & 0xff);
          if (2 * u + 1 < nran) neg[2 * u + 1] = (unsigned char)(v >> 8);
        }
      }
      w0 = w1 = 0;
      gbeg = p + 1;
    }
  }
  if (p < end) {  // stopped before pair p: keep the finished pairs of the open group
    for (long long u = gbeg; u < p; ++u) {
      const int j = (int)(u & 7);
      const unsigned v = (unsigned)(((j < 4 ? w0 : w1) >> (16 * (j & 3))) & 0xffffull);
      neg[2 * u] = (unsigned char)(v & 0xff);
      if (2 * u + 1 < nran) neg[2 * u + 1] = (unsigned char)(v >> 8);
    }
    atomicMin(stop, (unsigned long long)p);
  }
}

#define NCK(call)                                                                  \
  do {                                                                             \
    cudaError_t e__ = (call);                                                      \
    if (e__ != cudaSuccess) return set_error(SDFT_ERR_CUDA, cudaGetErrorString(e__)); \
  } while (0)

int upload(unsigned char *dst, const unsigned char *src, size_t n, cudaStream_t st) {
  if (n) NCK(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st));
  return SDFT_OK;
}
}  // namespace

size_t noise_scratch_bytes() { return 256 + (size_t)kNoiseMarginCap * (sizeof(long long) + sizeof(double)); }

int device_gauss_signs(long long nran, double *qseed, unsigned char *d_neg, void *d_scratch, cudaStream_t st,
                       int *kernel_launches) {
  if (nran <= 0) return SDFT_OK;
  const long long npairs = (nran + 1) / 2;
  unsigned long long *d_stop = reinterpret_cast<unsigned long long *>(d_scratch);
  int *d_nm = reinterpret_cast<int *>(reinterpret_cast<char *>(d_scratch) + 8);
  long long *d_mpair = reinterpret_cast<long long *>(reinterpret_cast<char *>(d_scratch) + 256);
  double *d_mphi = reinterpret_cast<double *>(d_mpair + kNoiseMarginCap);
  const JumpTable jt = make_jump_table();
  const int vec_ok = (reinterpret_cast<uintptr_t>(d_neg) & 15u) == 0;
  std::vector<unsigned char> hb;
  std::vector<long long> mpair;
  std::vector<double> mphi;
  double q = *qseed;
  long long p = 0;
  while (p < npairs) {
    // host: FP64 generator until the state is on the lattice
    hb.assign((size_t)std::min<long long>(2 * (npairs - p), 1 << 20), 0);
    const long long lim = std::min<long long>(npairs, p + (long long)hb.size() / 2);
    const long long p1 = gauss_signs_to_lattice(nran, p, lim, &q, hb.data());
    int r = upload(d_neg + 2 * p, hb.data(), (size_t)(std::min(2 * p1, nran) - 2 * p), st);
    if (r) return r;
    p = p1;
    if (p >= npairs || !durand_on_lattice(q)) continue;
    // device: the rest of the sequence from the lattice state
    const uint64_t q0 = (uint64_t)(q * 128.0);
    NCK(cudaMemsetAsync(d_scratch, 0xff, 8, st));
    NCK(cudaMemsetAsync(d_nm, 0, sizeof(int), st));
    const long long nthreads = (npairs - 1) / kChunk - p / kChunk + 1;
    const unsigned nblk = (unsigned)((nthreads + kThreads - 1) / kThreads);
    k_noise_signs<<<nblk, kThreads, 0, st>>>(q0, p, npairs, nran, jt, d_neg, vec_ok, d_stop, d_nm, d_mpair, d_mphi,
                                              kNoiseMarginCap);
    NCK(cudaGetLastError());
    if (kernel_launches) ++*kernel_launches;
    unsigned long long stop = 0;
    int nm = 0;
    NCK(cudaMemcpyAsync(&stop, d_stop, 8, cudaMemcpyDeviceToHost, st));
    NCK(cudaMemcpyAsync(&nm, d_nm, sizeof(int), cudaMemcpyDeviceToHost, st));
    NCK(cudaStreamSynchronize(st));
    const long long pstop = stop == ~0ull ? npairs : (long long)stop;
    if (nm > kNoiseMarginCap) {
      // more phi values near a sign change than the list holds: finish on the host
      const long long rest = npairs - p;
      hb.assign((size_t)(2 * rest), 0);
      gauss_signs(nran - 2 * p, &q, hb.data());
      if ((r = upload(d_neg + 2 * p, hb.data(), (size_t)(nran - 2 * p), st))) return r;
      NCK(cudaStreamSynchronize(st));
      p = npairs;
      break;
    }
    if (nm > 0) {
      mpair.resize(nm);
      mphi.resize(nm);
      NCK(cudaMemcpyAsync(mpair.data(), d_mpair, nm * sizeof(long long), cudaMemcpyDeviceToHost, st));
      NCK(cudaMemcpyAsync(mphi.data(), d_mphi, nm * sizeof(double), cudaMemcpyDeviceToHost, st));
      NCK(cudaStreamSynchronize(st));
      hb.assign((size_t)(2 * nm), 0);
      for (int k = 0; k < nm; ++k) {
        if (mpair[k] >= pstop) continue;  // past the stop: regenerated below
        gauss_signs_from_phi(mphi[k], &hb[2 * k]);
        const size_t nb = (2 * mpair[k] + 1 < nran) ? 2 : 1;
        if ((r = upload(d_neg + 2 * mpair[k], &hb[2 * k], nb, st))) return r;
      }
    }
    // exact state entering pair pstop
    q = (double)jump(q0, (unsigned long long)(pstop - p), jt) / 128.0;
    p = pstop;
  }
  NCK(cudaStreamSynchronize(st));
  *qseed = q;
  return SDFT_OK;
}

}  // namespace sdft

extern "C" int sdft_gaussran2_signs_dev(long long nran, double *qseed, unsigned char *neg, void *stream) {
  using namespace sdft;
  if (nran < 0 || !qseed || (nran > 0 && !neg)) return set_error(SDFT_ERR_ARG, "gaussran2_signs_dev: bad argument");
  if (nran == 0) return SDFT_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(SDFT_ERR_CUDA, "gaussran2_signs_dev: no device");
  void *scratch = nullptr;
  int r = dev_alloc(dev, stream, &scratch, noise_scratch_bytes());
  if (r) return r;
  r = device_gauss_signs(nran, qseed, neg, scratch, st, nullptr);
  dev_free(scratch, stream);
  cudaStreamSynchronize(st);
  return r;
}
