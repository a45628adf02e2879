// sdft_gemm_tc.cu -- TF32x3 tensor-core GEMM (tcgen05 + TMA + TMEM) for the
// Kleinman-Bylander projection / back projection in mixed precision.
//
//   out[n*ldo + m] (+)= sum_k A[m][k] B[n][k]
//
// A and B are each stored as two FP32 arrays holding TF32 values
// (hi = tf32(x), lo = tf32(x - hi)); the product is formed as
// hi*hi + hi*lo + lo*hi with FP32 accumulation in tensor memory (the
// "3xTF32" split-precision scheme), i.e. about FP32 accuracy from TF32
// tensor cores.  Long K is split over CTAs and the partials are summed in
// FP64 by a second kernel.
//
// CTA = 6 warps: warp 0 issues TMA loads (128B-swizzled K-major tiles,
// one mbarrier per stage), warp 1 owns the TMEM allocation and issues the
// tcgen05.mma instructions from one thread, warps 2..5 drain the
// accumulator (tcgen05.ld 32x32b) and store.  Every mbarrier wait is
// bounded; a wait that gives up raises a device error flag that the host
// reads after the filter (SDFT_ERR_TIMEOUT) instead of hanging.
// No TMA multicast is used.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include "sdft_internal.h"
#include "sdft_gemm_tc.cuh"

namespace sdft {

constexpr int TC_BM = 128, TC_BK = 32;     // K tile = 32 fp32 = 128 B (one swizzle row)
constexpr long long kWaitLimit = 1ll << 22; // bounded spin on mbarriers

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count));
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, int *err) {
  for (long long i = 0; i < kWaitLimit; i++)
    if (mbar_try(a, parity)) return true;
  atomicExch(err, 1);
  return false;
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *tm, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(tm), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  // tcgen05 shared-memory descriptor: K-major, 128B swizzle, 8-row groups
  // 1024 B apart (SBO), LBO field 1, descriptor version 1.
  return (uint64_t)((saddr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

template <int BN, int STAGES>
struct TcSmem {
  static constexpr int A_BYTES = TC_BM * TC_BK * 4;   // 16 KB
  static constexpr int B_BYTES = BN * TC_BK * 4;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int BAR_OFF = STAGES * STAGE_BYTES;
  static constexpr int TOTAL = BAR_OFF + 8 * (2 * STAGES + 1) + 16 + 1024;  // + alignment slack
};

// out_f32 != nullptr: FP32 partials at out_f32 + split*split_stride;
// else FP64 result in out_f64.
template <int BN, int STAGES>
__global__ void __launch_bounds__(192, 1)
k_gemm_tf32x3(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
              const __grid_constant__ CUtensorMap tBh, const __grid_constant__ CUtensorMap tBl, int ktiles_total,
              int ktiles_per_split, float *__restrict__ out_f32, size_t split_stride, double *__restrict__ out_f64,
              int ldo, int Mst, int Nst, int *err) {
  using S = TcSmem<BN, STAGES>;
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bar_full = sbase + S::BAR_OFF;
  const uint32_t bar_empty = bar_full + 8 * STAGES;
  const uint32_t bar_tmem = bar_empty + 8 * STAGES;
  uint32_t *tmem_slot = (uint32_t *)(smem + S::BAR_OFF + 8 * (2 * STAGES + 1));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * TC_BM;
  const int kt0 = blockIdx.z * ktiles_per_split;
  const int nkt = max(0, min(ktiles_total, kt0 + ktiles_per_split) - kt0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(bar_full + 8 * s, 1);
      mbar_init(bar_empty + 8 * s, 1);
    }
    mbar_init(bar_tmem, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      for (int it = 0; it < nkt; it++) {
        const int s = it % STAGES;
        const uint32_t par = ((it / STAGES) & 1) ^ 1;
        if (!mbar_wait(bar_empty + 8 * s, par, err)) break;
        const uint32_t st = sbase + s * S::STAGE_BYTES;
        mbar_expect_tx(bar_full + 8 * s, S::STAGE_BYTES);
        const int kx = (kt0 + it) * TC_BK;
        tma_load_2d(st, &tAh, kx, m0, bar_full + 8 * s);
        tma_load_2d(st + S::A_BYTES, &tAl, kx, m0, bar_full + 8 * s);
        tma_load_2d(st + 2 * S::A_BYTES, &tBh, kx, n0, bar_full + 8 * s);
        tma_load_2d(st + 2 * S::A_BYTES + S::B_BYTES, &tBl, kx, n0, bar_full + 8 * s);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                                 ((uint32_t)(TC_BM >> 4) << 24);
      uint32_t acc = 0;
      for (int it = 0; it < nkt; it++) {
        const int s = it % STAGES;
        if (!mbar_wait(bar_full + 8 * s, (it / STAGES) & 1, err)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = sbase + s * S::STAGE_BYTES;
        const uint32_t ah = st, al = st + S::A_BYTES, bh = st + 2 * S::A_BYTES, bl = bh + S::B_BYTES;
#pragma unroll
        for (int k8 = 0; k8 < TC_BK / 8; k8++) {
          const uint32_t off = k8 * 32;  // 8 tf32 = 32 bytes inside the swizzled row
          mma_tf32(tmem, sw128_desc(ah + off), sw128_desc(bh + off), idesc, acc);
          acc = 1;
          mma_tf32(tmem, sw128_desc(ah + off), sw128_desc(bl + off), idesc, 1);
          mma_tf32(tmem, sw128_desc(al + off), sw128_desc(bh + off), idesc, 1);
        }
        mma_commit(bar_empty + 8 * s);  // stage free once these MMAs retire
      }
      mma_commit(bar_tmem);  // accumulator complete (also fires when nkt == 0)
    }
  } else {  // epilogue warps 2..5: TMEM lane quadrant = warp % 4
    const int q = warp & 3;
    const bool ok = mbar_wait(bar_tmem, 0, err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int m = m0 + 32 * q + lane;
#pragma unroll 1
    for (int c = 0; c < BN / 32; c++) {
      uint32_t r[32];
      const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(c * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
            "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
            "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
            "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(ta));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (!ok || m >= Mst) continue;
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const int n = n0 + c * 32 + j;
        if (n < Nst) {
          const float v = (nkt > 0) ? __uint_as_float(r[j]) : 0.0f;
          if (out_f32)
            out_f32[(size_t)blockIdx.z * split_stride + (size_t)n * ldo + m] = v;
          else
            out_f64[(size_t)n * ldo + m] = (double)v;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
  }
}

// ---------------------------------------------------------------------------
// conversions
// ---------------------------------------------------------------------------
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// hi = tf32(x), lo = tf32(x - hi) of a double array (row-major rows x cols,
// source pitch lds, destination pitch ldd).
__global__ void k_split_tf32(const double *__restrict__ src, int lds, float *__restrict__ hi,
                             float *__restrict__ lo, int ldd, int rows, int cols) {
  const size_t tot = (size_t)rows * cols;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i - (size_t)r * cols);
    const double x = src[(size_t)r * lds + c];
    const float h = to_tf32((float)x);
    const float l = to_tf32((float)(x - (double)h));
    hi[(size_t)r * ldd + c] = h;
    lo[(size_t)r * ldd + c] = l;
  }
}

// FP64 sum of split-K partials -> out (FP64) and its TF32 hi/lo split.
__global__ void k_reduce_split_tf32(const float *__restrict__ part, int split, size_t stride, int ldo, int Mst,
                                    int Nst, double *__restrict__ out, float *__restrict__ hi,
                                    float *__restrict__ lo) {
  const size_t tot = (size_t)Mst * Nst;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    const int n = (int)(i / Mst), m = (int)(i - (size_t)n * Mst);
    const size_t idx = (size_t)n * ldo + m;
    double s = 0.0;
    for (int z = 0; z < split; z++) s += (double)part[z * stride + idx];
    out[idx] = s;
    if (hi) {
      const float h = to_tf32((float)s);
      hi[idx] = h;
      lo[idx] = to_tf32((float)(s - (double)h));
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*PFN_encodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                    const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode() {
  static PFN_encodeTiled fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_encodeTiled)p;
  }
  return fn;
}

bool gemm_tf32x3_available() { return get_encode() != nullptr; }

// K-major fp32 matrix [rows][ld] (ld >= K, ld % 4 == 0): box {32, box_rows}, 128B swizzle.
int make_tmap(CUtensorMap *tm, const float *base, int rows, int K, int ld, int box_rows) {
  PFN_encodeTiled enc = get_encode();
  if (!enc) return set_error(SDFT_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  if (((uintptr_t)base & 15) || (ld * 4) % 16 || K % TC_BK) return set_error(SDFT_ERR_ARG, "tensor map alignment");
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)base, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(SDFT_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return SDFT_OK;
}

template <int BN>
static int launch_bn(const TcGemm &gm, int split, int kps, float *part, size_t stride, double *out64, int *err,
                     cudaStream_t st) {
  constexpr int STAGES = (BN == 256) ? 2 : 3;
  using S = TcSmem<BN, STAGES>;
  auto k = k_gemm_tf32x3<BN, STAGES>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::TOTAL);
    attr = true;
  }
  dim3 grid(gm.N / BN, gm.M / TC_BM, split);
  k<<<grid, 192, S::TOTAL, st>>>(gm.tAh, gm.tAl, gm.tBh, gm.tBl, gm.K / TC_BK, kps, part, stride, out64, gm.ldo,
                                 gm.Mst, gm.Nst, err);
  return SDFT_OK;
}

int run_gemm_tf32x3(const TcGemm &gm, int split, float *part, size_t part_elems, double *out64, float *out_hi,
                    float *out_lo, int *err, cudaStream_t st) {
  const int ktiles = gm.K / TC_BK;
  if (split < 1) split = 1;
  if (split > ktiles) split = ktiles;
  const int kps = (ktiles + split - 1) / split;
  split = (ktiles + kps - 1) / kps;
  const size_t stride = (size_t)gm.N * gm.ldo;
  const bool use_part = (split > 1) || out_hi;
  if (use_part && (size_t)split * stride > part_elems) return set_error(SDFT_ERR_ARG, "tc gemm: workspace too small");
  int r = (gm.bn == 256) ? launch_bn<256>(gm, split, kps, use_part ? part : nullptr, stride, out64, err, st)
                         : launch_bn<128>(gm, split, kps, use_part ? part : nullptr, stride, out64, err, st);
  if (r) return r;
  if (use_part) {
    const size_t tot = (size_t)gm.Mst * gm.Nst;
    int blocks = (int)((tot + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_reduce_split_tf32<<<blocks, 256, 0, st>>>(part, split, stride, gm.ldo, gm.Mst, gm.Nst, out64, out_hi, out_lo);
  }
  return SDFT_OK;
}

void launch_split_tf32(const double *src, int lds, float *hi, float *lo, int ldd, int rows, int cols,
                       cudaStream_t st) {
  const size_t tot = (size_t)rows * cols;
  int blocks = (int)((tot + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_split_tf32<<<blocks, 256, 0, st>>>(src, lds, hi, lo, ldd, rows, cols);
}

}  // namespace sdft
