// sdft_gemm_oz.cu -- FP64-accurate GEMM from INT8 tcgen05 tensor cores
// (Ozaki scheme: split each operand into int8 digits under a per-row
// power-of-two scale, multiply digit slices exactly, recombine exactly).
//
// CTA = 10 warps over one 128 x BN output tile (BN = 128, or 64 for orbital
// counts that a 128-wide tile would pad more) and one K range:
//   warp 0    TMA producer: per 64-wide K tile one 3-D box per operand
//             carrying all four digit slices (64 B rows, 64B swizzle),
//             three-stage ring of 64 KB stages;
//   warp 1    TMEM owner (four int32 accumulators of BN columns, one per
//             digit order q = s + t: 512 columns, or 256 at BN = 64) and single-thread
//             issuer of tcgen05.mma.kind::i8 (10 slice pairs x 2 K steps
//             of 32 per stage);
//   warps 2-9 epilogue (two per TMEM lane quadrant, one column half each):
//             tcgen05.ld 32x32b of the four accumulators,
//             exact int64 combination acc0 2^21 + acc1 2^14 + acc2 2^7 +
//             acc3, one conversion to FP64 (exact: |value| < 2^53 for K
//             ranges below 2^20), scaling by 2^(Ea+Eb-33), coalesced store.
// int32 accumulation cannot overflow while (K range) * 4 * 64^2 < 2^31,
// i.e. K ranges up to 131072 (checked on the host).  The OZ_8x3 instance
// (3 slices, 6 products, the unsigned lower digits multiplied as u8) has
// three accumulators, four pipeline stages of 48 KB, and K ranges up to
// 16384.
// All mbarrier waits are bounded (sdft_tc_common.cuh).  No TMA multicast.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>
#include "sdft_internal.h"
#include "sdft_tc_common.cuh"
#include "sdft_gemm_oz.cuh"

namespace sdft {

constexpr int OZ_BM = 128, OZ_BK = 64;
// split-1 GEMMs (the back projection) run as the persistent kernel: the
// next tile's loads overlap the epilogue (measured 4 % faster than one CTA
// per tile at 28-bit digits, 7 % at 24-bit)
constexpr bool kOzPersistent = true;

// per digit format: slices, digit bits, pipeline stages, K range limit and
// the power of two that turns the combined accumulators into the product
template <int FMT> struct OzF;
template <> struct OzF<OZ_7x4> {
  static constexpr int NS = 4, BITS = 7, STAGES = 3, MAX_KRANGE = 131072, SCALE_EXP = -33;
};
template <> struct OzF<OZ_8x3> {
  static constexpr int NS = 3, BITS = 8, STAGES = 4, MAX_KRANGE = 16384, SCALE_EXP = -30;
};

// BN: output columns (orbitals) per tile, 128 or 64.  The 64-wide tile
// pads small orbital counts less; its stages are smaller, so it keeps one
// more of them.
template <int FMT, int BN = 128> struct OzSmem {
  static constexpr int NS = OzF<FMT>::NS, OZ_STAGES = OzF<FMT>::STAGES + (BN == 64 ? 1 : 0);
  static constexpr int A_SLICE = OZ_BM * OZ_BK;          // 8 KB
  static constexpr int B_SLICE = BN * OZ_BK;             // 8 KB (BN = 128) or 4 KB
  static constexpr int A_BYTES = NS * A_SLICE;
  static constexpr int B_BYTES = NS * B_SLICE;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;  // 64 KB (7x4) or 48 KB (8x3)
  static constexpr int BAR_OFF = OZ_STAGES * STAGE_BYTES;
  static constexpr int TOTAL = BAR_OFF + 8 * (2 * OZ_STAGES + 2) + 16 + 1024;  // + alignment slack
  // NS accumulators of BN columns, rounded up to a power of two
  static constexpr int TMEM_COLS = NS * BN <= 256 ? 256 : 512;
};

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

constexpr int OZ_EPI_WARPS = 8;                 // two per TMEM lane quadrant
constexpr int OZ_THREADS = 32 * (2 + OZ_EPI_WARPS);

template <typename OutT, int FMT, int BN>
__global__ void __launch_bounds__(OZ_THREADS, 1)
k_gemm_oz8(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, int ktiles_total,
           int ktiles_per_split, const double *__restrict__ sa, const double *__restrict__ sb,
           OutT *__restrict__ out, size_t split_stride, int ldo, int Mst, int Nst, int *err) {
  using S = OzSmem<FMT, BN>;
  constexpr int NS = OzF<FMT>::NS, OZ_STAGES = S::OZ_STAGES, BITS = OzF<FMT>::BITS;
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bar_full = sbase + S::BAR_OFF;
  const uint32_t bar_empty = bar_full + 8 * OZ_STAGES;
  const uint32_t bar_tmem = bar_empty + 8 * OZ_STAGES;
  uint32_t *tmem_slot = (uint32_t *)(smem + S::BAR_OFF + 8 * (2 * OZ_STAGES + 1));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * OZ_BM;
  const int kt0 = blockIdx.z * ktiles_per_split;
  const int nkt = max(0, min(ktiles_total, kt0 + ktiles_per_split) - kt0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < OZ_STAGES; s++) {
      mbar_init(bar_full + 8 * s, 1);
      mbar_init(bar_empty + 8 * s, 1);
    }
    mbar_init(bar_tmem, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(S::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      for (int it = 0; it < nkt; it++) {
        const int s = it % OZ_STAGES;
        const uint32_t par = ((it / OZ_STAGES) & 1) ^ 1;
        if (!mbar_wait(bar_empty + 8 * s, par, err)) break;
        const uint32_t st = sbase + s * S::STAGE_BYTES;
        mbar_expect_tx(bar_full + 8 * s, S::STAGE_BYTES);
        const int kx = (kt0 + it) * OZ_BK;
        tma_load_3d(st, &tA, kx, m0, 0, bar_full + 8 * s);
        tma_load_3d(st + S::A_BYTES, &tB, kx, n0, 0, bar_full + 8 * s);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      // D = S32, A / B = signed (1) or unsigned (0) 8-bit, K-major, N = 128, M = 128;
      // OZ_8x3: digit 0 signed, digits 1 and 2 unsigned
      constexpr uint32_t idesc0 = (2u << 4) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(OZ_BM >> 4) << 24);
      uint32_t started = 0;  // bit q: accumulator q holds data
      for (int it = 0; it < nkt; it++) {
        const int s = it % OZ_STAGES;
        if (!mbar_wait(bar_full + 8 * s, (it / OZ_STAGES) & 1, err)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = sbase + s * S::STAGE_BYTES;
#pragma unroll
        for (int ks = 0; ks < OZ_BK / 32; ks++) {
#pragma unroll
          for (int sa_ = 0; sa_ < NS; sa_++) {
#pragma unroll
            for (int tb = 0; tb + sa_ < NS; tb++) {
              const int q = sa_ + tb;
              const bool as = FMT == OZ_7x4 || sa_ == 0, bs = FMT == OZ_7x4 || tb == 0;
              const uint32_t idesc = idesc0 | (as ? 1u << 7 : 0u) | (bs ? 1u << 10 : 0u);
              const uint64_t ad = smem_desc<64>(st + sa_ * S::A_SLICE + ks * 32);
              const uint64_t bd = smem_desc<64>(st + S::A_BYTES + tb * S::B_SLICE + ks * 32);
              mma_i8(tmem + (uint32_t)(q * BN), ad, bd, idesc, (started >> q) & 1u);
              started |= 1u << q;
            }
          }
        }
        mma_commit(bar_empty + 8 * s);  // stage free once these MMAs retire
      }
      mma_commit(bar_tmem);  // accumulators complete (also fires when nkt == 0)
    }
  } else {  // epilogue warps 2..9: TMEM lane quadrant = warp % 4, column half = (warp - 2) / 4
    const int qd = warp & 3;
    const int half = (warp - 2) >> 2;
    const bool ok = mbar_wait(bar_tmem, 0, err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int m = m0 + 32 * qd + lane;
    const bool row_ok = ok && m < Mst && nkt > 0;
    const double fa = row_ok ? ldexp(sa[m], OzF<FMT>::SCALE_EXP) : 0.0;
    const uint32_t tl = tmem + ((uint32_t)(32 * qd) << 16);
    constexpr int CH = BN / 16 / 2;  // 16-column chunks per epilogue warp
#pragma unroll 1
    for (int c = half * CH; c < (half + 1) * CH; c++) {
      uint32_t r0[16], r1[16], r2[16], r3[16];
      tmem_ld16(tl + 0 * BN + c * 16, r0);
      tmem_ld16(tl + 1 * BN + c * 16, r1);
      tmem_ld16(tl + 2 * BN + c * 16, r2);
      if constexpr (NS == 4) tmem_ld16(tl + 3 * BN + c * 16, r3);
      tmem_ld_wait();
      if (!(ok && m < Mst)) continue;
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const int n = n0 + c * 16 + j;
        if (n < Nst) {
          long long v;
          if constexpr (NS == 4)
            v = ((long long)(int)r0[j] << (3 * BITS)) + ((long long)(int)r1[j] << (2 * BITS)) +
                ((long long)(int)r2[j] << BITS) + (long long)(int)r3[j];
          else
            v = ((long long)(int)r0[j] << (2 * BITS)) + ((long long)(int)r1[j] << BITS) + (long long)(int)r2[j];
          out[(size_t)blockIdx.z * split_stride + (size_t)n * ldo + m] = (OutT)(row_ok ? (double)v * fa * sb[n] : 0.0);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TMEM_COLS));
  }
}

// Persistent form for split == 1 (the back projection, whose K range is
// short): one CTA per SM walks the output tiles t = blockIdx.x, +gridDim.x,
// ...; the stage ring and its phases run on across tiles, so the producer
// loads the next tile's first K tiles while the epilogue drains the
// accumulators, and a tmem_empty barrier (one arrive per epilogue warp) holds
// the next tile's MMAs until the accumulators have been read.  Sixteen
// epilogue warps (four per TMEM lane quadrant, two 16-column chunks each)
// drain a tile in half the rounds of eight, which shortens the time the
// MMAs wait between tiles.
constexpr int OZP_EPI_WARPS = 16;
constexpr int OZP_THREADS = 32 * (2 + OZP_EPI_WARPS);
template <typename OutT, int FMT, int BN>
__global__ void __launch_bounds__(OZP_THREADS, 1)
k_gemm_oz8p(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, int nkt, int ntn,
            int ntiles, const double *__restrict__ sa, const double *__restrict__ sb, OutT *__restrict__ out,
            int ldo, int Mst, int Nst, int *err) {
  using S = OzSmem<FMT, BN>;
  constexpr int NS = OzF<FMT>::NS, OZ_STAGES = S::OZ_STAGES, BITS = OzF<FMT>::BITS;
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bar_full = sbase + S::BAR_OFF;
  const uint32_t bar_empty = bar_full + 8 * OZ_STAGES;
  const uint32_t bar_tfull = bar_empty + 8 * OZ_STAGES;
  const uint32_t bar_tempty = bar_tfull + 8;
  uint32_t *tmem_slot = (uint32_t *)(smem + S::BAR_OFF + 8 * (2 * OZ_STAGES + 2));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < OZ_STAGES; s++) {
      mbar_init(bar_full + 8 * s, 1);
      mbar_init(bar_empty + 8 * s, 1);
    }
    mbar_init(bar_tfull, 1);
    mbar_init(bar_tempty, OZP_EPI_WARPS);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(S::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer, continuous over the CTA's tiles
      bool go = true;
      for (int tile = blockIdx.x, ti = 0; go && tile < ntiles; tile += gridDim.x, ti++) {
        const int n0 = (tile % ntn) * BN, m0 = (tile / ntn) * OZ_BM;
        for (int it = 0; it < nkt; it++) {
          const int g = ti * nkt + it, s = g % OZ_STAGES;
          if (!mbar_wait(bar_empty + 8 * s, ((g / OZ_STAGES) & 1) ^ 1, err)) { go = false; break; }
          const uint32_t st = sbase + s * S::STAGE_BYTES;
          mbar_expect_tx(bar_full + 8 * s, S::STAGE_BYTES);
          tma_load_3d(st, &tA, it * OZ_BK, m0, 0, bar_full + 8 * s);
          tma_load_3d(st + S::A_BYTES, &tB, it * OZ_BK, n0, 0, bar_full + 8 * s);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc0 = (2u << 4) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(OZ_BM >> 4) << 24);
      bool go = true;
      for (int tile = blockIdx.x, ti = 0; go && tile < ntiles; tile += gridDim.x, ti++) {
        if (ti > 0) {  // accumulators of the previous tile read out
          if (!mbar_wait(bar_tempty, (ti - 1) & 1, err)) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        uint32_t started = 0;
        for (int it = 0; it < nkt; it++) {
          const int g = ti * nkt + it, s = g % OZ_STAGES;
          if (!mbar_wait(bar_full + 8 * s, (g / OZ_STAGES) & 1, err)) { go = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t st = sbase + s * S::STAGE_BYTES;
#pragma unroll
          for (int ks = 0; ks < OZ_BK / 32; ks++) {
#pragma unroll
            for (int sa_ = 0; sa_ < NS; sa_++) {
#pragma unroll
              for (int tb = 0; tb + sa_ < NS; tb++) {
                const int q = sa_ + tb;
                const bool as = FMT == OZ_7x4 || sa_ == 0, bs = FMT == OZ_7x4 || tb == 0;
                const uint32_t idesc = idesc0 | (as ? 1u << 7 : 0u) | (bs ? 1u << 10 : 0u);
                const uint64_t ad = smem_desc<64>(st + sa_ * S::A_SLICE + ks * 32);
                const uint64_t bd = smem_desc<64>(st + S::A_BYTES + tb * S::B_SLICE + ks * 32);
                mma_i8(tmem + (uint32_t)(q * BN), ad, bd, idesc, (started >> q) & 1u);
                started |= 1u << q;
              }
            }
          }
          mma_commit(bar_empty + 8 * s);
        }
        mma_commit(bar_tfull);  // this tile's accumulators complete
      }
    }
  } else {  // epilogue warps 2..17: TMEM lane quadrant = warp % 4, column quarter = (warp - 2) / 4
    const int qd = warp & 3;
    const int part = (warp - 2) >> 2;
    for (int tile = blockIdx.x, ti = 0; tile < ntiles; tile += gridDim.x, ti++) {
      const int n0 = (tile % ntn) * BN, m0 = (tile / ntn) * OZ_BM;
      const bool ok = mbar_wait(bar_tfull, ti & 1, err);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int m = m0 + 32 * qd + lane;
      const bool row_ok = ok && m < Mst;
      const double fa = row_ok ? ldexp(sa[m], OzF<FMT>::SCALE_EXP) : 0.0;
      const uint32_t tl = tmem + ((uint32_t)(32 * qd) << 16);
      constexpr int CH = BN / 16 / (OZP_EPI_WARPS / 4);
#pragma unroll 1
      for (int c = part * CH; c < (part + 1) * CH; c++) {
        uint32_t r0[16], r1[16], r2[16], r3[16];
        tmem_ld16(tl + 0 * BN + c * 16, r0);
        tmem_ld16(tl + 1 * BN + c * 16, r1);
        tmem_ld16(tl + 2 * BN + c * 16, r2);
        if constexpr (NS == 4) tmem_ld16(tl + 3 * BN + c * 16, r3);
        tmem_ld_wait();
        if (c == (part + 1) * CH - 1) {
          // this warp's last accumulator read is complete: release the
          // accumulators before converting and storing this chunk, so the
          // next tile's MMAs overlap that work
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar_tempty) : "memory");
        }
        if (!row_ok) continue;
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int n = n0 + c * 16 + j;
          if (n < Nst) {
            long long v;
            if constexpr (NS == 4)
              v = ((long long)(int)r0[j] << (3 * BITS)) + ((long long)(int)r1[j] << (2 * BITS)) +
                  ((long long)(int)r2[j] << BITS) + (long long)(int)r3[j];
            else
              v = ((long long)(int)r0[j] << (2 * BITS)) + ((long long)(int)r1[j] << BITS) + (long long)(int)r2[j];
            out[(size_t)n * ldo + m] = (OutT)((double)v * fa * sb[n]);
          }
        }
      }
      if (!ok) break;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------
// digit extraction
// ---------------------------------------------------------------------------
__device__ __forceinline__ double absmax_key(double a) { return isfinite(a) ? fabs(a) : INFINITY; }

// rowmax[row] = max |x[row][:]| (as the bit pattern of a non-negative double,
// whose integer order is its numeric order); +inf if any entry is not finite.
// Element sources of the digit passes: a stored row, or the row of i G_d c
// formed on the fly from c (Re = -G_d Im c, Im = G_d Re c; G = 0 and the
// padding give 0), the vector whose projection is dZ/dR_d.
struct SrcRows {
  const double *x;
  int ldx;
  __device__ __forceinline__ double operator()(int row, int c) const { return x[(size_t)row * ldx + c]; }
};
struct SrcIGc {
  const double *v;  // rows of 2 ngp: re[0, ngp), im[ngp, 2 ngp)
  const double *gk; // G_d per coefficient
  int ngp, ncoef;
  __device__ __forceinline__ double operator()(int row, int c) const {
    const double *r = v + (size_t)row * 2 * ngp;
    const bool im = c >= ngp;
    const int g = im ? c - ngp : c;
    if (g >= ncoef - 1) return 0.0;
    return im ? gk[g] * r[g] : -gk[g] * r[ngp + g];
  }
};

template <typename SRC>
__global__ void k_row_absmax(SRC src, int cols, unsigned long long *rowmax) {
  const int row = blockIdx.x;
  double m = 0.0;
  for (int c = blockIdx.y * blockDim.x + threadIdx.x; c < cols; c += gridDim.y * blockDim.x)
    m = fmax(m, absmax_key(src(row, c)));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
    atomicMax(rowmax + row, (unsigned long long)__double_as_longlong(m));
  }
}

// Exponent E with max < 2^E (E = 0 for an all-zero row, clamped below so
// that 2^(6-E) stays finite).
__device__ __forceinline__ int row_exponent(unsigned long long maxbits) {
  if (maxbits == 0) return 0;
  const int field = (int)(maxbits >> 52) & 0x7ff;
  return max(-1000, max(field, 1) - 1022);
}

// Digits of one value, all steps exact in FP64.  OZ_7x4: four round-to-
// nearest digits of x 2^(6-E) (|.| < 64), the remainder times 2^7 each
// step.  OZ_8x3: floor(x 2^(7-E)) in [-128, 127], then two floors of the
// remainder (in [0, 1)) times 2^8, in [0, 255].
template <int FMT> __device__ __forceinline__ void digits_of(double r, int *d) {
#pragma unroll
  for (int s = 0; s < OzF<FMT>::NS; s++) {
    const double q = FMT == OZ_7x4 ? rint(r) : floor(r);
    d[s] = (int)q;
    r = (r - q) * (FMT == OZ_7x4 ? 128.0 : 256.0);
  }
}
template <int FMT> constexpr int kTopShift = FMT == OZ_7x4 ? 6 : 7;  // x 2^(shift - E) is the top digit's value

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  return (uint32_t)(a & 0xff) | ((uint32_t)(b & 0xff) << 8) | ((uint32_t)(c & 0xff) << 16) |
         ((uint32_t)(d & 0xff) << 24);
}

// digits of rows x cols doubles; 4 consecutive columns per thread, zero
// digits for cols <= k < ld.
template <int FMT, typename SRC>
__global__ void k_slice_rows(SRC src, int rows, int cols, const unsigned long long *__restrict__ rowmax,
                             int8_t *__restrict__ dig, int ld, size_t sstride, double *__restrict__ scale) {
  constexpr int NS = OzF<FMT>::NS;
  const int g4 = ld >> 2;
  const size_t tot = (size_t)rows * g4;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(i / g4), c4 = (int)(i - (size_t)row * g4) * 4;
    const unsigned long long mb = rowmax[row];
    const bool bad = mb >= 0x7ff0000000000000ull;
    const int E = bad ? 0 : row_exponent(mb);
    const double p = ldexp(1.0, kTopShift<FMT> - E);
    int d[4][NS];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int c = c4 + e;
      const double v = (c < cols && !bad) ? src(row, c) : 0.0;
      digits_of<FMT>(v * p, d[e]);
    }
#pragma unroll
    for (int s = 0; s < NS; s++)
      *(uint32_t *)(dig + s * sstride + (size_t)row * ld + c4) = pack4(d[0][s], d[1][s], d[2][s], d[3][s]);
    if (c4 == 0) scale[row] = bad ? __longlong_as_double(0x7ff8000000000000ll) : ldexp(1.0, E);
  }
}

// Sum of split-K partials for one row per CTA, then the digit form of the
// row (second sweep over the just-written row, which is L2 resident).
template <int FMT>
__global__ void k_reduce_slice(const double *__restrict__ part, int split, size_t stride, int ldo, int Mst,
                               double *__restrict__ out, int8_t *__restrict__ dig, size_t dig_stride,
                               double *__restrict__ scale, unsigned long long *__restrict__ zero_rowmax) {
  constexpr int NS = OzF<FMT>::NS;
  const int n = blockIdx.x;
  if (zero_rowmax && threadIdx.x == 0) zero_rowmax[n] = 0ull;
  double mx = 0.0;
  for (int m = threadIdx.x; m < ldo; m += blockDim.x) {
    double s = 0.0;
    if (m < Mst)
      for (int z = 0; z < split; z++) s += part[z * stride + (size_t)n * ldo + m];
    out[(size_t)n * ldo + m] = s;
    mx = fmax(mx, absmax_key(s));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ double red[32];
  __shared__ unsigned long long mbits;
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmax(mx, red[w]);
    mbits = (unsigned long long)__double_as_longlong(mx);
  }
  __syncthreads();
  const bool bad = mbits >= 0x7ff0000000000000ull;
  const int E = bad ? 0 : row_exponent(mbits);
  const double p = ldexp(1.0, kTopShift<FMT> - E);
  for (int m4 = threadIdx.x * 4; m4 < ldo; m4 += blockDim.x * 4) {
    int d[4][NS];
#pragma unroll
    for (int e = 0; e < 4; e++) digits_of<FMT>(bad ? 0.0 : out[(size_t)n * ldo + m4 + e] * p, d[e]);
#pragma unroll
    for (int s = 0; s < NS; s++)
      *(uint32_t *)(dig + s * dig_stride + (size_t)n * ldo + m4) = pack4(d[0][s], d[1][s], d[2][s], d[3][s]);
  }
  if (threadIdx.x == 0) scale[n] = bad ? __longlong_as_double(0x7ff8000000000000ll) : ldexp(1.0, E);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*PFN_encodeTiledOz)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                      const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                      CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                      CUtensorMapFloatOOBfill);

static PFN_encodeTiledOz get_encode_oz() {
  static PFN_encodeTiledOz fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_encodeTiledOz)p;
  }
  return fn;
}

bool gemm_oz_available() { return get_encode_oz() != nullptr; }

int make_tmap_oz(CUtensorMap *tm, const int8_t *dig, int rows, int ld, int fmt, int box_rows) {
  PFN_encodeTiledOz enc = get_encode_oz();
  if (!enc) return set_error(SDFT_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  if (box_rows != 64 && box_rows != 128) return set_error(SDFT_ERR_ARG, "oz tensor map box");
  if (((uintptr_t)dig & 15) || ld % OZ_BK || rows % 128) return set_error(SDFT_ERR_ARG, "oz tensor map alignment");
  const int ns = oz_slices(fmt);
  cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)rows, (cuuint64_t)ns};
  cuuint64_t strides[2] = {(cuuint64_t)ld, (cuuint64_t)ld * rows};
  cuuint32_t box[3] = {(cuuint32_t)OZ_BK, (cuuint32_t)box_rows, (cuuint32_t)ns};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void *)dig, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(SDFT_ERR_CUDA, "cuTensorMapEncodeTiled failed (oz)");
  return SDFT_OK;
}

int oz_min_split(int K, int fmt) {
  const int ktiles = (K + OZ_BK - 1) / OZ_BK;
  const int kmax = (fmt == OZ_8x3 ? OzF<OZ_8x3>::MAX_KRANGE : OzF<OZ_7x4>::MAX_KRANGE) / OZ_BK;
  return (ktiles + kmax - 1) / kmax;
}

int oz_choose_split(int tiles, int ktiles, int max_split) {
  // cost model in MMA-stage units: waves x K tiles per CTA, plus the
  // partial-tile write + read of each extra split (about 8 stages' worth of
  // one CTA's time, spread over the 148 SMs)
  const int nsm = 148;
  int best = 1;
  double best_cost = 1e300;
  const int lim = max_split < 1 ? 1 : max_split;
  for (int s = 1; s <= lim && s <= ktiles; s++) {
    const int kps = (ktiles + s - 1) / s;
    if (kps * OZ_BK > OzF<OZ_7x4>::MAX_KRANGE) continue;
    const int se = (ktiles + kps - 1) / kps;
    const int waves = (tiles * se + nsm - 1) / nsm;
    const double cost = (double)waves * kps + (se > 1 ? 8.0 * se * tiles / nsm : 0.0);
    if (cost < best_cost - 1e-9) { best_cost = cost; best = se; }
  }
  return best;
}

template <typename OutT, int FMT, int BN>
static int run_gemm_oz_t(const OzGemm &g, int split, OutT *out, size_t split_stride, int *err, cudaStream_t st,
                         int *split_used) {
  using S = OzSmem<FMT, BN>;
  const int ktiles = (g.K + OZ_BK - 1) / OZ_BK;
  if (g.M % OZ_BM || g.N % BN || ktiles < 1) return set_error(SDFT_ERR_ARG, "oz gemm: shape");
  if (split < 1) split = 1;
  if (split > ktiles) split = ktiles;
  int kps = (ktiles + split - 1) / split;
  if (kps * OZ_BK > OzF<FMT>::MAX_KRANGE) {
    if (split_stride == 0) return set_error(SDFT_ERR_ARG, "oz gemm: K range per CTA too long");
    kps = OzF<FMT>::MAX_KRANGE / OZ_BK;
  }
  split = (ktiles + kps - 1) / kps;
  if (split_used) *split_used = split;  // the partials written: what a reduction must sum
  if (split == 1 && kOzPersistent) {
    static const bool attr_p = (cudaFuncSetAttribute(k_gemm_oz8p<OutT, FMT, BN>,
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL), true);
    (void)attr_p;
    const int ntn = g.N / BN, ntiles = ntn * (g.M / OZ_BM);
    const int grid = ntiles < 148 ? ntiles : 148;
    k_gemm_oz8p<OutT, FMT, BN><<<grid, OZP_THREADS, S::TOTAL, st>>>(g.tA, g.tB, ktiles, ntn, ntiles, g.sa, g.sb, out, g.ldo,
                                                               g.Mst, g.Nst, err);
    return SDFT_OK;
  }
  static const bool attr_once =
      (cudaFuncSetAttribute(k_gemm_oz8<OutT, FMT, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL), true);
  (void)attr_once;
  dim3 grid(g.N / BN, g.M / OZ_BM, split);
  k_gemm_oz8<OutT, FMT, BN><<<grid, OZ_THREADS, S::TOTAL, st>>>(g.tA, g.tB, ktiles, kps, g.sa, g.sb, out, split_stride,
                                                            g.ldo, g.Mst, g.Nst, err);
  return SDFT_OK;
}

template <typename OutT>
static int run_gemm_oz_any(const OzGemm &g, int split, OutT *out, size_t split_stride, int *err, cudaStream_t st,
                           int *su) {
  if (g.bn != 64 && g.bn != 128) return set_error(SDFT_ERR_ARG, "oz gemm: tile width");
  if (g.fmt == OZ_8x3)
    return g.bn == 64 ? run_gemm_oz_t<OutT, OZ_8x3, 64>(g, split, out, split_stride, err, st, su)
                      : run_gemm_oz_t<OutT, OZ_8x3, 128>(g, split, out, split_stride, err, st, su);
  return g.bn == 64 ? run_gemm_oz_t<OutT, OZ_7x4, 64>(g, split, out, split_stride, err, st, su)
                    : run_gemm_oz_t<OutT, OZ_7x4, 128>(g, split, out, split_stride, err, st, su);
}
int run_gemm_oz(const OzGemm &g, int split, double *out, size_t split_stride, int *err, cudaStream_t st,
                int *split_used) {
  return run_gemm_oz_any(g, split, out, split_stride, err, st, split_used);
}
int run_gemm_oz(const OzGemm &g, int split, float *out, size_t split_stride, int *err, cudaStream_t st,
                int *split_used) {
  return run_gemm_oz_any(g, split, out, split_stride, err, st, split_used);
}

template <typename SRC>
static void rowmax_of(SRC src, int rows, int cols, unsigned long long *rowmax, cudaStream_t st) {
  cudaMemsetAsync(rowmax, 0, (size_t)rows * sizeof(unsigned long long), st);
  int chunks = (cols + 255) / 256;  // grid = rows x chunks (rows on x: up to 2^31 - 1)
  if (chunks > 64) chunks = 64;
  if (chunks < 1) chunks = 1;
  k_row_absmax<SRC><<<dim3(rows, chunks), 256, 0, st>>>(src, cols, rowmax);
}

template <typename SRC>
static void slice_of(SRC src, int rows, int cols, const unsigned long long *rowmax, int8_t *dig, int ld,
                     size_t slice_stride, double *scale, cudaStream_t st, int fmt) {
  const size_t tot = (size_t)rows * (ld / 4);
  int blocks = (int)((tot + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (fmt == OZ_8x3)
    k_slice_rows<OZ_8x3, SRC><<<blocks, 256, 0, st>>>(src, rows, cols, rowmax, dig, ld, slice_stride, scale);
  else
    k_slice_rows<OZ_7x4, SRC><<<blocks, 256, 0, st>>>(src, rows, cols, rowmax, dig, ld, slice_stride, scale);
}

void launch_oz_rowmax(const double *x, int ldx, int rows, int cols, unsigned long long *rowmax, cudaStream_t st) {
  rowmax_of(SrcRows{x, ldx}, rows, cols, rowmax, st);
}

// Row maxima of i G_d c for d = x, y, z in one pass over c: |Re| = |G_d| |Im c|
// and |Im| = |G_d| |Re c|, so each coefficient contributes |G_d| max(|Re c|,
// |Im c|) (G = 0 and the padding contribute 0).  rowmax3: 3 rows-long words.
__global__ void k_row_absmax_igc3(const double *__restrict__ v, const double *__restrict__ gk, int ngp, int ncoef,
                                  int rows, unsigned long long *rowmax3) {
  const int row = blockIdx.x;
  const double *r = v + (size_t)row * 2 * ngp;
  double m[3] = {0.0, 0.0, 0.0};
  for (int g = blockIdx.y * blockDim.x + threadIdx.x; g < ncoef - 1; g += gridDim.y * blockDim.x) {
    const double a = fmax(absmax_key(r[g]), absmax_key(r[ngp + g]));
#pragma unroll
    for (int d = 0; d < 3; d++) m[d] = fmax(m[d], absmax_key(gk[(size_t)d * ngp + g] * a));
  }
  __shared__ double red[3][32];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    for (int o = 16; o > 0; o >>= 1) m[d] = fmax(m[d], __shfl_xor_sync(0xffffffffu, m[d], o));
    if ((threadIdx.x & 31) == 0) red[d][threadIdx.x >> 5] = m[d];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int d = threadIdx.x;
    double x = red[d][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) x = fmax(x, red[d][w]);
    atomicMax(rowmax3 + (size_t)d * rows + row, (unsigned long long)__double_as_longlong(x));
  }
}

void launch_oz_rowmax_igc3(const double *v, const double *gk, int ngp, int ncoef, int rows,
                           unsigned long long *rowmax3, cudaStream_t st) {
  cudaMemsetAsync(rowmax3, 0, (size_t)3 * rows * sizeof(unsigned long long), st);
  int chunks = (ncoef + 255) / 256;
  if (chunks > 64) chunks = 64;
  if (chunks < 1) chunks = 1;
  k_row_absmax_igc3<<<dim3(rows, chunks), 256, 0, st>>>(v, gk, ngp, ncoef, rows, rowmax3);
}

void launch_oz_slice_igc(const double *v, const double *gk, int ngp, int ncoef, int rows,
                         const unsigned long long *rowmax, int8_t *dig, int ld, size_t slice_stride, double *scale,
                         cudaStream_t st) {
  slice_of(SrcIGc{v, gk, ngp, ncoef}, rows, 2 * ngp, rowmax, dig, ld, slice_stride, scale, st, OZ_7x4);
}

void launch_oz_slice(const double *x, int ldx, int rows, int cols, const unsigned long long *rowmax, int8_t *dig,
                     int ld, size_t slice_stride, double *scale, cudaStream_t st, int fmt) {
  slice_of(SrcRows{x, ldx}, rows, cols, rowmax, dig, ld, slice_stride, scale, st, fmt);
}

void launch_oz_slice_rows(const double *x, int ldx, int rows, int cols, unsigned long long *rowmax, int8_t *dig,
                          int ld, size_t slice_stride, double *scale, cudaStream_t st, int fmt) {
  launch_oz_rowmax(x, ldx, rows, cols, rowmax, st);
  launch_oz_slice(x, ldx, rows, cols, rowmax, dig, ld, slice_stride, scale, st, fmt);
}

void launch_oz_reduce_slice(const double *part, int split, size_t stride, int ldo, int Mst, int Nst, double *out,
                            int8_t *dig, size_t dig_stride, double *scale, unsigned long long *zero_rowmax,
                            cudaStream_t st, int fmt) {
  if (fmt == OZ_8x3)
    k_reduce_slice<OZ_8x3><<<Nst, 256, 0, st>>>(part, split, stride, ldo, Mst, out, dig, dig_stride, scale,
                                                 zero_rowmax);
  else
    k_reduce_slice<OZ_7x4><<<Nst, 256, 0, st>>>(part, split, stride, ldo, Mst, out, dig, dig_stride, scale,
                                                 zero_rowmax);
}

// The bounded wait of the GEMM pipeline, made to run out on purpose: an
// mbarrier initialised for one arrival that never comes.  mbar_wait polls it
// `polls` times, sets the error word and returns; the kernel then ends.
__global__ void k_selftest_wait(int *err, long long polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  const uint32_t a = smem_u32(&bar);
  mbar_init(a, 1);
  mbar_wait(a, 0, err, polls);
}

void launch_selftest_wait(int *err, long long polls, cudaStream_t st) { k_selftest_wait<<<1, 32, 0, st>>>(err, polls); }

}  // namespace sdft
