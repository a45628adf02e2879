// sdft_api.cu -- device context and C ABI of the B200 stochastic-DFT filter
// hot path.  Host buffers follow PINY's layout (state-major, half sphere,
// G=0 last, separate re/im arrays); device buffers hold one orbital as
// [re block | im block], each block padded to ngp doubles.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <mutex>
#include <unordered_map>
#include <algorithm>
#include "sdft_internal.h"
#include "sdft_kernels.cuh"
#include "sdft_ctx.h"
#include "sdft_kernels2.cuh"
#include "sdft_noise.h"
#include "sdft_lanczos.h"

namespace sdft {

static thread_local std::string g_err;
int set_error(int code, const char *msg) {
  g_err = msg ? msg : "";
  return code;
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e__ = (call);                                                      \
    if (e__ != cudaSuccess) {                                                      \
      char b__[512];                                                               \
      snprintf(b__, sizeof b__, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e__), \
               __FILE__, __LINE__);                                                \
      return set_error(e__ == cudaErrorMemoryAllocation ? SDFT_ERR_NOMEM : SDFT_ERR_CUDA, b__); \
    }                                                                              \
  } while (0)

static bool edge_ok(int n) {
  if (n < 2 || n > kMaxEdge) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}
static inline size_t rup(size_t a, size_t b) { return (a + b - 1) / b * b; }

template <typename T> size_t plane_smem(const DevGeom &g);

}  // namespace sdft

using namespace sdft;


namespace sdft {
// Device memory comes from one stream-ordered pool per device: allocations
// and releases are ordered on the owning context's stream and never
// synchronise the whole device, so contexts created and destroyed while
// other contexts' work runs (a server) do not wait for that work.  Released
// blocks stay in the pool for reuse (release threshold unlimited).
static cudaMemPool_t pool_of(int device) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  if (device < 0 || device >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[device]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[device] = pool;
  }
  return pools[device];
}

// Bytes this library holds on each device (every allocation goes through
// dev_alloc / dev_free) and the optional cap of sdft_set_device_memory_limit.
struct DevAccount {
  std::mutex mu;
  std::unordered_map<void *, std::pair<int, size_t>> live;  // pointer -> (device, bytes)
  long long used[64] = {}, limit[64] = {};
};
static DevAccount &dev_account() {
  static DevAccount a;
  return a;
}

int dev_alloc(int device, void *stream, void **p, size_t bytes) {
  *p = nullptr;
  if (device < 0 || device >= 64) return set_error(SDFT_ERR_ARG, "device index >= 64");
  DevAccount &acc = dev_account();
  {
    std::lock_guard<std::mutex> lk(acc.mu);
    if (acc.limit[device] > 0 && acc.used[device] + (long long)bytes > acc.limit[device]) {
      char b[256];
      snprintf(b, sizeof b, "device allocation of %zu bytes refused: %lld of the %lld-byte limit in use", bytes,
               acc.used[device], acc.limit[device]);
      return set_error(SDFT_ERR_NOMEM, b);
    }
    acc.used[device] += (long long)bytes;  // reserved before the allocation, released on failure
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaMemPool_t pool = pool_of(device);
  cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaErrorMemoryAllocation;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // usable from any stream on return
  if (e != cudaSuccess) {
    if (*p) cudaFreeAsync(*p, st);
    *p = nullptr;
    {
      std::lock_guard<std::mutex> lk(acc.mu);
      acc.used[device] -= (long long)bytes;
    }
    char b[256];
    snprintf(b, sizeof b, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return set_error(SDFT_ERR_NOMEM, b);
  }
  std::lock_guard<std::mutex> lk(acc.mu);
  acc.live[*p] = {device, bytes};
  return SDFT_OK;
}

void dev_free(void *p, void *stream) {
  if (!p) return;
  {
    DevAccount &acc = dev_account();
    std::lock_guard<std::mutex> lk(acc.mu);
    auto it = acc.live.find(p);
    if (it != acc.live.end()) {
      acc.used[it->second.first] -= (long long)it->second.second;
      acc.live.erase(it);
    }
  }
  cudaFreeAsync(p, reinterpret_cast<cudaStream_t>(stream));
}

int dmalloc(sdft_ctx *c, void **p, size_t bytes) {
  int r = dev_alloc(c->device, c->st, p, bytes);
  if (r) return r;
  c->dev_bytes += (long long)bytes;
  return SDFT_OK;
}
#define DM(ptr, bytes)                                                   \
  do {                                                                   \
    int r__ = dmalloc(ctx, (void **)&(ptr), (bytes));                    \
    if (r__) return r__;                                                 \
  } while (0)

// Build the column decomposition from the PINY-ordered half sphere.
static int build_columns(sdft_ctx *ctx, std::vector<int> &cp_gstart, std::vector<int> &cp_gcount,
                         std::vector<int> &col_ab) {
  const int nk = ctx->ncoef - 1;
  const int *ka = ctx->ka.data(), *kb = ctx->kb.data(), *kc = ctx->kc.data();
  int zs = -1, zc = 0, kamax = 0;
  for (int i = 0; i < nk; i++) {
    if (std::abs(ka[i]) * 2 + 1 > ctx->n1 || std::abs(kb[i]) * 2 + 1 > ctx->n2 ||
        std::abs(kc[i]) * 2 + 1 > ctx->n3)
      return set_error(SDFT_ERR_UNSUPPORTED, "G sphere does not fit the FFT grid (|k| >= n/2)");
    kamax = std::max(kamax, std::abs(ka[i]));
    const bool half = ka[i] > 0 || (ka[i] == 0 && kb[i] > 0) || (ka[i] == 0 && kb[i] == 0 && kc[i] > 0);
    if (!half) return set_error(SDFT_ERR_ARG, "G list is not a half sphere (ka,kb,kc) > 0");
  }
  if (ctx->ka[nk] != 0 || ctx->kb[nk] != 0 || ctx->kc[nk] != 0)
    return set_error(SDFT_ERR_ARG, "G=0 must be stored last");
  int i = 0;
  while (i < nk) {
    int j = i;
    while (j < nk && ka[j] == ka[i] && kb[j] == kb[i]) j++;
    if (ka[i] == 0 && kb[i] == 0) {
      if (zs >= 0) return set_error(SDFT_ERR_ARG, "(0,0) column not contiguous");
      zs = i;
      zc = j - i;
    } else {
      cp_gstart.push_back(i);
      cp_gcount.push_back(j - i);
      auto w = [](int k, int n) { return k < 0 ? k + n : k; };
      col_ab.push_back((w(ka[i], ctx->n1) << 16) | w(kb[i], ctx->n2));
      col_ab.push_back((w(-ka[i], ctx->n1) << 16) | w(-kb[i], ctx->n2));
    }
    i = j;
  }
  // duplicate columns would mean the list is not grouped by (ka,kb)
  {
    std::vector<int> chk(col_ab);
    std::sort(chk.begin(), chk.end());
    if (std::adjacent_find(chk.begin(), chk.end()) != chk.end())
      return set_error(SDFT_ERR_ARG, "G list not grouped by (ka,kb) columns");
  }
  cp_gstart.push_back(zs < 0 ? 0 : zs);
  cp_gcount.push_back(zc);
  col_ab.push_back(0);
  ctx->cols.ncp = (int)cp_gstart.size();
  ctx->cols.ncols = (int)col_ab.size();
  ctx->cols.ncols_pad = (int)rup(ctx->cols.ncols, 4);
  ctx->cols.kamax = kamax;
  return SDFT_OK;
}

// Replace the block *p (have bytes) by one of need bytes.  The new block is
// allocated first, so a refused allocation leaves *p, its contents and the
// caller's recorded capacity as they were; the old block is freed in stream
// order after the work queued on it.
static int grow(sdft_ctx *ctx, void **p, size_t have, size_t need) {
  void *q = nullptr;
  int r = dmalloc(ctx, &q, need);
  if (r) return r;
  if (*p) {
    dev_free(*p, ctx->st);
    ctx->dev_bytes -= (long long)have;
  }
  *p = q;
  return SDFT_OK;
}

static int ensure_x(sdft_ctx *ctx, int npairs) {
  const size_t csz = ctx->fft64 ? sizeof(double2) : sizeof(float2);
  const size_t need = (size_t)npairs * ctx->n3 * ctx->cols.ncols_pad * csz;
  if (need <= ctx->x_bytes) return SDFT_OK;
  int r = grow(ctx, &ctx->d_x, ctx->x_bytes, need);
  if (r) return r;
  ctx->x_bytes = need;
  return SDFT_OK;
}

// Pairs per chunk when the column scratch holds FP64 data (the one-off
// transforms -- noise, density -- run in FP64 in every context); the
// scratch is grown to at least two FP32 pairs so a chunk is never empty.
static int fp64_chunk(sdft_ctx *ctx, int npairs, int *chunk) {
  int r = ensure_x(ctx, std::max(npairs, 2));
  if (r) return r;
  const size_t per = (size_t)ctx->n3 * ctx->cols.ncols_pad * sizeof(double2);
  *chunk = (int)std::min<size_t>((size_t)npairs, ctx->x_bytes / per);
  return *chunk >= 1 ? SDFT_OK : set_error(SDFT_ERR_STATE, "column scratch too small");
}

static int ensure_coef(sdft_ctx *ctx, size_t n) {
  if (n <= ctx->coef_cap) return SDFT_OK;
  int r = grow(ctx, (void **)&ctx->d_coef, ctx->coef_cap * 8, n * sizeof(double));
  if (r) return r;
  ctx->coef_cap = n;
  return SDFT_OK;
}

static int ensure_acc(sdft_ctx *ctx, int nmu) {
  if (nmu <= ctx->acc_nmu) return SDFT_OK;
  int r = grow(ctx, (void **)&ctx->d_acc, (size_t)ctx->acc_nmu * ctx->vec_elems * 8,
               (size_t)nmu * ctx->vec_elems * sizeof(double));
  if (r) return r;
  CK(cudaMemsetAsync(ctx->d_acc, 0, (size_t)nmu * ctx->vec_elems * sizeof(double), ctx->st));
  ctx->acc_nmu = nmu;
  return SDFT_OK;
}

static int ensure_mom(sdft_ctx *ctx, size_t n) {
  if (n <= ctx->mom_cap) return SDFT_OK;
  int r = grow(ctx, (void **)&ctx->d_mom, ctx->mom_cap * 8, n * sizeof(double));
  if (r) return r;
  ctx->mom_cap = n;
  return SDFT_OK;
}

// Host <-> device orbital block copies (PINY layout <-> [s][re|im][ngp]).
static int upload_block(sdft_ctx *ctx, double *dst, int nstate, const double *re, const double *im) {
  const size_t w = (size_t)ctx->ncoef * sizeof(double);
  const size_t dp = (size_t)2 * ctx->ngp * sizeof(double);
  CK(cudaMemcpy2DAsync(dst, dp, re, w, w, nstate, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpy2DAsync(dst + ctx->ngp, dp, im, w, w, nstate, cudaMemcpyHostToDevice, ctx->st));
  return SDFT_OK;
}
static int download_block(sdft_ctx *ctx, const double *src, int nstate, double *re, double *im) {
  const size_t w = (size_t)ctx->ncoef * sizeof(double);
  const size_t sp = (size_t)2 * ctx->ngp * sizeof(double);
  CK(cudaMemcpy2DAsync(re, w, src, sp, w, nstate, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpy2DAsync(im, w, src + ctx->ngp, sp, w, nstate, cudaMemcpyDeviceToHost, ctx->st));
  return SDFT_OK;
}

static bool is_fp64(const sdft_ctx *c) { return c->fft64; }

// Default CTA size of the FP32 plane stage: 128 threads for planes of 48 x 48
// to 72 x 72 points, where registers, not the plane's shared memory, bound
// the CTAs per SM (stage B 24 % faster at 48 x 48, config 2 +8.8 %; the
// autotuner took 128 for 30 of the 32 batch systems), 256 otherwise (12 %
// faster at 96 x 96; config 1's 24 x 24 planes 1.3 % faster at 256).
static int default_plane_threads(const sdft_ctx *c) {
  return (!c->fft64 && c->fast && c->n1 <= 72 && c->n2 <= 72 && c->n1 * c->n2 >= 48 * 48) ? 128 : 256;
}

// Nonlocal projection Z = Pj C and back projection FNL = Bk Z for `nstate`
// orbitals held in `vec`, mixed precision: INT8 Ozaki GEMMs on the digit
// form of the orbitals; Z = Pj C is split over K with FP64 partial sums, the
// reduction also produces the digit form of Z for FNL = Bk Z.
// gk (nullable): project i G_d vec instead of vec, formed inside the digit
// pass (gk = G_d per coefficient) under the row maxima gk_max
static int run_kb_oz(sdft_ctx *ctx, const double *vec, int nstate, bool want_enl, bool back = true,
                     const double *gk = nullptr, const unsigned long long *gk_max = nullptr) {
  const int K1 = 2 * ctx->ngp, S = ctx->s_oz, Ppad = ctx->Ppad;
  // tile width of both GEMMs: the set one, else 64 where it pads the orbitals less
  const int bn = ctx->gemm_bn ? ctx->gemm_bn : ((nstate + 63) / 64 * 64 < (nstate + 127) / 128 * 128 ? 64 : 128);
  const int N = (nstate + bn - 1) / bn * bn;
  {
    TScope ts(ctx, 7);
    if (gk) {
      launch_oz_slice_igc(vec, gk, ctx->ngp, ctx->ncoef, nstate, gk_max, ctx->d_c_dig, ctx->kp_oz,
                          (size_t)S * ctx->kp_oz, ctx->d_c_sc, ctx->st);
      ctx->launches++;
    } else {
      // row maxima: from the stage C that wrote `vec`, else one pass over it
      if (!(ctx->track_omax && ctx->omax_vec == vec && ctx->omax_n == nstate)) {  // (set only when oz)
        launch_oz_rowmax(vec, K1, nstate, K1, ctx->d_rowmax, ctx->st);  // clears the rows first
        ctx->launches++;
      }
      launch_oz_slice(vec, K1, nstate, K1, ctx->d_rowmax, ctx->d_c_dig, ctx->kp_oz, (size_t)S * ctx->kp_oz,
                      ctx->d_c_sc, ctx->st);
      ctx->launches++;
    }
  }
  OzGemm g1 = ctx->om1, g2 = ctx->om2;
  g1.N = N; g1.Nst = nstate;
  g2.N = N; g2.Nst = nstate;
  g1.bn = g2.bn = bn;
  if (bn == 64) {
    g1.tB = ctx->om1_tb64;
    g2.tB = ctx->om2_tb64;
  }
  const size_t stride = (size_t)N * Ppad;
  const int max_split = (int)std::min<size_t>(32, ctx->oz_part_elems / stride);
  const int min_split = oz_min_split(ctx->kp_oz, OZ_7x4);
  if (min_split > max_split) return set_error(SDFT_ERR_NOMEM, "oz gemm: partial buffer too small for K");
  const int split = ctx->gemm_split > 0 ? std::max(min_split, std::min(ctx->gemm_split, std::max(1, max_split)))
                                        : oz_choose_split((Ppad / 128) * (N / bn), ctx->kp_oz / 64, max_split);
  int r;
  {
    TScope ts(ctx, 3);
    int used = split;  // the partials the launch writes (K tiles dealt out evenly)
    r = run_gemm_oz(g1, split, ctx->d_oz_part, stride, ctx->d_err, ctx->st, &used);
    if (r) return r;
    // also zeroes d_rowmax[0, nstate) for the next stage C (the slice above
    // has consumed it)
    launch_oz_reduce_slice(ctx->d_oz_part, used, stride, Ppad, ctx->P, nstate, ctx->d_z, ctx->d_z_dig,
                           (size_t)S * Ppad, ctx->d_z_sc, ctx->d_rowmax, ctx->st, ctx->om2.fmt);
    ctx->launches += 2;
    ctx->rowmax_zero_n = nstate;
    ctx->omax_vec = nullptr;
  }
  if (want_enl) {
    launch_enl(ctx->d_z, Ppad, ctx->d_w, ctx->P, nstate, ctx->d_enl, ctx->st);
    ctx->launches += 2;
  }
  if (!back) return SDFT_OK;
  {
    TScope ts(ctx, 4);
    // FNL in FP32 (its rounding is below the FP32 transforms' error in the
    // same force); stage C reads it through EpiArgs::FNLf
    r = run_gemm_oz(g2, 1, reinterpret_cast<float *>(ctx->d_fnl), 0, ctx->d_err, ctx->st);
    ctx->launches++;
  }
  return r;
}

static int run_kb(sdft_ctx *ctx, const double *vec, int nstate, bool want_enl, bool back = true) {
  if (ctx->P == 0) return SDFT_OK;
  if (ctx->oz) return run_kb_oz(ctx, vec, nstate, want_enl, back);
  const int spad = (int)rup(nstate, 64);
  const int K1 = 2 * ctx->ngp;
  // split K of the projection so that >= ~2 waves of CTAs exist
  const int tiles = (ctx->Ppad / 128) * (spad / 64);
  int split = 1;
  while (tiles * split < 2 * 148 && split < 64 && (K1 / 16) / (split * 2) >= 8 &&
         (size_t)(split * 2) * spad * ctx->Ppad <= ctx->zwork_elems)
    split *= 2;
  if (ctx->gemm_split > 0) {  // tuned override, within the workspace and K
    split = std::min(ctx->gemm_split, std::max(1, K1 / 16));
    while (split > 1 && (size_t)split * spad * ctx->Ppad > ctx->zwork_elems) split--;
  }
  {
    TScope ts(ctx, 3);
    launch_gemm_nt_f64(ctx->d_pj, K1, vec, K1, ctx->d_z, ctx->Ppad, ctx->Ppad, spad, K1, ctx->P, nstate,
                       split, ctx->d_zwork, ctx->st);
  }
  ctx->launches += split > 1 ? 2 : 1;
  if (want_enl) {
    launch_enl(ctx->d_z, ctx->Ppad, ctx->d_w, ctx->P, nstate, ctx->d_enl, ctx->st);
    ctx->launches += 2;
  }
  if (!back) return SDFT_OK;
  {
    TScope ts(ctx, 4);
    launch_gemm_nt_f64(ctx->d_bk, ctx->Ppad, ctx->d_z, ctx->Ppad, ctx->d_fnl, K1, ctx->Mpad2, spad,
                       ctx->Ppad, K1, nstate, 1, nullptr, ctx->st);
  }
  ctx->launches++;
  return SDFT_OK;
}

// One application of the fused H pipeline on `cur` with epilogue `e`.
static int apply_h(sdft_ctx *ctx, const double *cur, int nstate, EpiArgs e, bool want_enl) {
  int r = run_kb(ctx, cur, nstate, want_enl);
  if (r) return r;
  const int npairs = (nstate + 1) / 2;
  if ((r = ensure_x(ctx, npairs))) return r;
  e.nstate = nstate;
  e.pair0 = 0;
  e.C = cur;
  if (ctx->P && ctx->oz) e.FNLf = reinterpret_cast<const float *>(ctx->d_fnl);
  else e.FNL = ctx->P ? ctx->d_fnl : nullptr;
  e.invN = 1.0 / (double)ctx->N;
  if (ctx->oz && ctx->track_omax && e.OUT) {  // (row maxima exist only for the digit GEMMs)
    if (ctx->rowmax_zero_n < nstate) CK(cudaMemsetAsync(ctx->d_rowmax, 0, (size_t)nstate * 8, ctx->st));
    e.omax = ctx->d_rowmax;
  }
  // inside a loop the previous stage C already packed and c-transformed `cur`
  // into the column scratch; this step's stage C does the same for OUT when
  // another application follows
  const bool fuse = ctx->fast && ctx->track_omax && !is_fp64(ctx);
  const bool have_x = fuse && ctx->x_vec == cur && ctx->x_n == nstate;
  e.Xnext = (fuse && e.pack_next && e.OUT) ? ctx->d_x : nullptr;
  int nl = 3;
  if (ctx->fast) {
    if (is_fp64(ctx)) {
      if (!have_x) { TScope ts(ctx, 0); fast_stage_a<double>(ctx->g, cur, nstate, 0, npairs, ctx->d_x, ctx->st); }
      { TScope ts(ctx, 1); fast_stage_b<double>(ctx->g, ctx->d_x, (const double *)ctx->d_vp, npairs, ctx->st); }
      { TScope ts(ctx, 2); fast_stage_c<double>(ctx->g, ctx->d_x, e, npairs, ctx->st); }
    } else {
      if (!have_x) { TScope ts(ctx, 0); fast_stage_a<float>(ctx->g, cur, nstate, 0, npairs, ctx->d_x, ctx->st); }
      { TScope ts(ctx, 1); fast_stage_b<float>(ctx->g, ctx->d_x, (const float *)ctx->d_vp, npairs, ctx->st); }
      { TScope ts(ctx, 2); fast_stage_c<float>(ctx->g, ctx->d_x, e, npairs, ctx->st); }
    }
    if (have_x) nl = 2;
  } else if (is_fp64(ctx)) {
    { TScope ts(ctx, 0); launch_stage_a<double>(ctx->g, cur, nstate, 0, npairs, ctx->d_x, ctx->st); }
    { TScope ts(ctx, 1); launch_stage_b<double>(ctx->g, ctx->d_x, (const double *)ctx->d_vp, npairs, ctx->st); }
    { TScope ts(ctx, 2); launch_stage_c<double>(ctx->g, ctx->d_x, e, npairs, ctx->st); }
  } else {
    { TScope ts(ctx, 0); launch_stage_a<float>(ctx->g, cur, nstate, 0, npairs, ctx->d_x, ctx->st); }
    { TScope ts(ctx, 1); launch_stage_b<float>(ctx->g, ctx->d_x, (const float *)ctx->d_vp, npairs, ctx->st); }
    { TScope ts(ctx, 2); launch_stage_c<float>(ctx->g, ctx->d_x, e, npairs, ctx->st); }
  }
  ctx->launches += nl;
  CK(cudaGetLastError());
  if (e.omax) {
    ctx->omax_vec = e.OUT;
    ctx->omax_n = nstate;
    ctx->rowmax_zero_n = 0;
  }
  ctx->x_vec = e.Xnext ? e.OUT : nullptr;
  ctx->x_n = nstate;
  return SDFT_OK;
}

// For the duration of one filter / moments loop: row-maximum tracking (mixed
// precision) and the stage A fused into the previous stage C (fast path).
struct OmaxScope {
  sdft_ctx *c;
  explicit OmaxScope(sdft_ctx *ctx) : c(ctx) { c->track_omax = true; c->omax_vec = nullptr; c->x_vec = nullptr; }
  ~OmaxScope() { c->track_omax = false; c->omax_vec = nullptr; c->x_vec = nullptr; }
};

static int check_ready(sdft_ctx *ctx, int nstate) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (nstate < 1 || nstate > ctx->max_states) return set_error(SDFT_ERR_ARG, "nstate out of range (1..max_states)");
  if (!ctx->have_v) return set_error(SDFT_ERR_STATE, "V_KS not set (sdft_ctx_set_vks)");
  return SDFT_OK;
}

static EpiArgs base_epi(sdft_ctx *ctx) {
  EpiArgs e{};
  e.acc_stride = ctx->vec_elems;
  e.nmu = 0;
  e.ndots = 0;
  return e;
}

// The filter sum acc = sum_k a_k v_k is updated every other step: step k
// (odd, >= 3) adds a_{k-1} v_{k-1} + a_k v_k -- v_{k-1} is the step's input
// vector, which the epilogue reads anyway -- and even steps skip the
// accumulator, except the last step (then only a_k v_k).  Same terms, half
// the accumulator traffic.
static void pair_accumulation(sdft_ctx *ctx, EpiArgs &e, int k, int L, int nmu) {
  if (k < 2) return;
  if (k % 2 == 0) {
    if (k != L - 1) e.ACC = nullptr;
  } else {
    e.acoefp = ctx->d_coef + (size_t)(k - 1) * nmu;
  }
}

// Chebyshev filter on resident chi (d_chi) -> d_acc.  moments (device, may
// be null): per step dots written to d_mom[k*3 .. k*3+2].
static int filter_cheby_core(sdft_ctx *ctx, int nstate, int L, int nmu, double scale, double emean,
                             bool store_moments) {
  int r;
  OmaxScope om(ctx);
  if ((r = ensure_acc(ctx, nmu))) return r;
  const double prefact = -scale * emean, s1 = -scale * 0.25, s2 = -scale * 0.5;
  double *cur = ctx->d_chi, *prev = nullptr;
  double *bufs[2] = {ctx->d_b1, ctx->d_b2};
  const int nparts = ((nstate + 1) / 2) * ctx->g.nbatch;
  for (int k = 1; k < L; k++) {
    EpiArgs e = base_epi(ctx);
    double *out = (k == 1) ? bufs[0] : (k == 2 ? bufs[1] : prev);
    e.OUT = out;
    e.ACC = ctx->d_acc;
    e.nmu = nmu;
    e.acoef = ctx->d_coef + (size_t)k * nmu;
    e.acoef0 = (k == 1) ? ctx->d_coef : nullptr;
    pair_accumulation(ctx, e, k, L, nmu);
    e.pack_next = k + 1 < L;
    e.CHI = ctx->d_chi;
    if (k == 1) {
      e.mode = EPI_CHEB1;
      e.s1 = s1; e.s2 = s2; e.pre = prefact;
    } else {
      e.mode = EPI_CHEBK;
      e.s1 = 2.0 * s1; e.s2 = 2.0 * s2; e.pre = 2.0 * prefact;
      e.PREV = prev;
    }
    if (store_moments) {
      e.dots = ctx->d_dots;
      e.ndots = (k == 1) ? 2 : 1;
    }
    if ((r = apply_h(ctx, cur, nstate, e, false))) return r;
    if (store_moments) {
      launch_dots_reduce(ctx->d_dots, nparts, 3, ctx->d_dots + ctx->dots_cap * 3, ctx->d_mom + (size_t)k * 3,
                         ctx->st);
      ctx->launches += 2;
    }
    prev = cur;
    cur = out;
  }
  return SDFT_OK;
}

static int filter_newton_core(sdft_ctx *ctx, int nstate, int L, int nmu, const double *samp, double scale,
                              double emean) {
  int r;
  OmaxScope om(ctx);
  if ((r = ensure_acc(ctx, nmu))) return r;
  const double s1 = -scale * 0.25, s2 = -scale * 0.5;
  double *cur = ctx->d_chi;
  for (int k = 1; k < L; k++) {
    EpiArgs e = base_epi(ctx);
    e.mode = EPI_NEWTON;
    e.OUT = ctx->d_b1;  // k==1 writes B1, then in place
    e.ACC = ctx->d_acc;
    e.nmu = nmu;
    e.acoef = ctx->d_coef + (size_t)k * nmu;
    e.acoef0 = (k == 1) ? ctx->d_coef : nullptr;
    pair_accumulation(ctx, e, k, L, nmu);
    e.pack_next = k + 1 < L;
    e.s1 = s1; e.s2 = s2;
    e.pre = -scale * emean - samp[k - 1];
    if ((r = apply_h(ctx, cur, nstate, e, false))) return r;
    cur = ctx->d_b1;
  }
  return SDFT_OK;
}

// Moments by the doubling identities (calcChebyMoments).
static int moments_core(sdft_ctx *ctx, int nstate, int L, double scale, double emean, double *mom_host) {
  int r;
  OmaxScope om(ctx);
  const int M = (L % 2 == 0) ? (L / 2 + 1) : ((L + 1) / 2);
  if ((r = ensure_mom(ctx, (size_t)(M + 1) * 3))) return r;
  const double prefact = -scale * emean, s1 = -scale * 0.25, s2 = -scale * 0.5;
  const int nparts = ((nstate + 1) / 2) * ctx->g.nbatch;
  double *cur = ctx->d_chi, *prev = nullptr;
  double *bufs[2] = {ctx->d_b1, ctx->d_b2};
  for (int k = 1; k < std::max(M, 2); k++) {
    EpiArgs e = base_epi(ctx);
    double *out = (k == 1) ? bufs[0] : (k == 2 ? bufs[1] : prev);
    e.OUT = out;
    e.CHI = ctx->d_chi;
    e.dots = ctx->d_dots;
    e.pack_next = k + 1 < std::max(M, 2);
    if (k == 1) {
      e.mode = EPI_CHEB1;
      e.ndots = 2;
      e.s1 = s1; e.s2 = s2; e.pre = prefact;
    } else {
      e.mode = EPI_MOMK;
      e.ndots = 3;
      e.s1 = 2.0 * s1; e.s2 = 2.0 * s2; e.pre = 2.0 * prefact;
      e.PREV = prev;
    }
    if ((r = apply_h(ctx, cur, nstate, e, false))) return r;
    launch_dots_reduce(ctx->d_dots, nparts, 3, ctx->d_dots + ctx->dots_cap * 3, ctx->d_mom + (size_t)k * 3,
                       ctx->st);
    ctx->launches += 2;
    prev = cur;
    cur = out;
  }
  std::vector<double> h((size_t)(M + 1) * 3);
  CK(cudaMemcpyAsync(h.data(), ctx->d_mom, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  // assemble in the order calcChebyMoments writes (later writes win)
  for (int i = 0; i <= L; i++) mom_host[i] = 0.0;
  mom_host[0] = h[1 * 3 + 1];  // <chi,chi> from step 1
  mom_host[1] = h[1 * 3 + 0];
  for (int k = 2; k < M; k++) {
    mom_host[k] = h[k * 3 + 0];
    mom_host[2 * k - 1] = 2.0 * h[k * 3 + 1] - mom_host[1];
    mom_host[2 * k] = 2.0 * h[k * 3 + 2] - mom_host[0];
    // calcChebyMoments zeroes [k], [2k], [2k-1] at the start of step k and
    // then writes all three; step k' > k overwrites [k'] with the direct dot.
  }
  // direct dots of steps k' overwrite doubled values written earlier
  for (int k = 2; k < M; k++) mom_host[k] = h[k * 3 + 0];
  return SDFT_OK;
}

}  // namespace sdft

// ============================================================================
// C ABI
// ============================================================================
extern "C" const char *sdft_last_error(void) { return g_err.c_str(); }
extern "C" int sdft_version(void) { return 10000; }

extern "C" int sdft_ctx_create(int n1, int n2, int n3, int ncoef, const int *ka, const int *kb,
                               const int *kc, const double *hmat, int precision, int max_states,
                               int device, sdft_ctx **out) {
  if (!out || !ka || !kb || !kc || !hmat) return set_error(SDFT_ERR_ARG, "ctx_create: null argument");
  *out = nullptr;
  if (!edge_ok(n1) || !edge_ok(n2) || !edge_ok(n3))
    return set_error(SDFT_ERR_UNSUPPORTED, "FFT edges must be 2^a 3^b in [2,128]");
  if (ncoef < 2 || max_states < 1) return set_error(SDFT_ERR_ARG, "ctx_create: ncoef/max_states");
  if (precision != SDFT_PREC_FP64 && precision != SDFT_PREC_MIXED && precision != SDFT_PREC_MIXED_FAST)
    return set_error(SDFT_ERR_ARG, "ctx_create: precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(SDFT_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return set_error(SDFT_ERR_ARG, "ctx_create: device index");
  sdft_ctx *ctx = new sdft_ctx();
  auto fail = [&](int code) { sdft_ctx_destroy(ctx); return code; };
  ctx->device = device;
  ctx->prec = precision;
  ctx->fft64 = (precision == SDFT_PREC_FP64);
  ctx->n1 = n1; ctx->n2 = n2; ctx->n3 = n3;
  ctx->N = n1 * n2 * n3;
  ctx->ncoef = ncoef;
  ctx->ngp = (int)rup(ncoef, 16);
  std::memcpy(ctx->hmat, hmat, sizeof(double) * 9);
  ctx->vol = cell_volume(hmat);
  ctx->ka.assign(ka, ka + ncoef);
  ctx->kb.assign(kb, kb + ncoef);
  ctx->kc.assign(kc, kc + ncoef);
  ctx->max_states = max_states;
  ctx->s_pad = (int)rup(max_states, 64);
  ctx->npairs_max = (max_states + 1) / 2;
  ctx->vec_elems = (size_t)ctx->s_pad * 2 * ctx->ngp;
  if (cudaSetDevice(device) != cudaSuccess) return fail(set_error(SDFT_ERR_CUDA, "cudaSetDevice failed"));
  if (cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error(SDFT_ERR_CUDA, "stream create failed"));
  if (init_const_twiddles()) return fail(set_error(SDFT_ERR_CUDA, "constant twiddle tables"));
  std::vector<int> cpg, cpc, colab;
  int r = build_columns(ctx, cpg, cpc, colab);
  if (r) return fail(r);
  // shared-memory budget of the plane stage
  {
    DevGeom t{};
    t.n1 = n1; t.n2 = n2; t.n3 = n3;
    size_t need = is_fp64(ctx) ? plane_smem<double>(t) : plane_smem<float>(t);
    if (need > 227 * 1024) return fail(set_error(SDFT_ERR_UNSUPPORTED, "plane does not fit shared memory"));
    if (n1 * n2 > 512 * 24) return fail(set_error(SDFT_ERR_UNSUPPORTED, "plane too large"));
  }
  {
    const char *ev = getenv("SDFT_GENERIC_FFT");  // force the runtime-size kernels (testing)
    ctx->fast = fast_supported(n1, n2, n3) && !(ev && ev[0] == '1');
  }
  std::vector<int> gkc(ncoef);
  for (int i = 0; i < ncoef; i++) gkc[i] = kc[i];
  std::vector<double> ak2(ncoef);
  sdft_ak2_kinetic(hmat, ncoef, ka, kb, kc, 0.0, ak2.data());
  std::vector<double2> tw(n1 + n2 + n3);
  std::vector<float2> twf(n1 + n2 + n3);
  int off = 0;
  for (int n : {n1, n2, n3}) {
    for (int t = 0; t < n; t++) {
      double a = 2.0 * M_PI * (double)t / (double)n;
      tw[off + t] = make_double2(std::cos(a), -std::sin(a));
      twf[off + t] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
    off += n;
  }
#define DMF(ptr, bytes) do { int r__ = dmalloc(ctx, (void **)&(ptr), (bytes)); if (r__) return fail(r__); } while (0)
#define CKF(call) do { cudaError_t e__ = (call); if (e__ != cudaSuccess) return fail(set_error(SDFT_ERR_CUDA, cudaGetErrorString(e__))); } while (0)
  DMF(ctx->d_cp_gstart, cpg.size() * sizeof(int));
  DMF(ctx->d_cp_gcount, cpc.size() * sizeof(int));
  DMF(ctx->d_col_ab, colab.size() * sizeof(int));
  DMF(ctx->d_gkc, ncoef * sizeof(int));
  DMF(ctx->d_ak2, ncoef * sizeof(double));
  DMF(ctx->d_tw, tw.size() * sizeof(double2));
  DMF(ctx->d_twf, twf.size() * sizeof(float2));
  CKF(cudaMemcpyAsync(ctx->d_cp_gstart, cpg.data(), cpg.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKF(cudaMemcpyAsync(ctx->d_cp_gcount, cpc.data(), cpc.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKF(cudaMemcpyAsync(ctx->d_col_ab, colab.data(), colab.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKF(cudaMemcpyAsync(ctx->d_gkc, gkc.data(), ncoef * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKF(cudaMemcpyAsync(ctx->d_ak2, ak2.data(), ncoef * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  CKF(cudaMemcpyAsync(ctx->d_tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
  CKF(cudaMemcpyAsync(ctx->d_twf, twf.data(), twf.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->st));
  DevGeom &g = ctx->g;
  g.n1 = n1; g.n2 = n2; g.n3 = n3; g.N = ctx->N;
  g.plane_nt = default_plane_threads(ctx);
  g.ncoef = ncoef; g.ngp = ctx->ngp;
  g.ncols = ctx->cols.ncols; g.ncols_pad = ctx->cols.ncols_pad; g.ncp = ctx->cols.ncp; g.kamax = ctx->cols.kamax;
  g.nbatch = (g.ncp + kCPB - 1) / kCPB;
  g.cp_gstart = ctx->d_cp_gstart; g.cp_gcount = ctx->d_cp_gcount; g.col_ab = ctx->d_col_ab;
  g.gkc = ctx->d_gkc; g.ak2 = ctx->d_ak2;
  g.tw1 = ctx->d_tw; g.tw2 = ctx->d_tw + n1; g.tw3 = ctx->d_tw + n1 + n2;
  g.tw1f = ctx->d_twf; g.tw2f = ctx->d_twf + n1; g.tw3f = ctx->d_twf + n1 + n2;
  // signed kb range of the sphere columns on each plane row a (a = ka mod n1),
  // and whether every row's columns fill their range
  {
    std::vector<int2> rng(n1, make_int2(1, 0));
    std::vector<int> cnt(n1, 0);
    for (int ab : colab) {
      const int a = ab >> 16, b = ab & 0xffff;
      const int kb = b <= n2 / 2 ? b : b - n2;
      if (cnt[a]++ == 0) rng[a] = make_int2(kb, kb);
      else rng[a] = make_int2(std::min(rng[a].x, kb), std::max(rng[a].y, kb));
    }
    g.kb_contig = 1;
    g.kbmax = 0;
    for (int a = 0; a < n1; a++) {
      if (cnt[a] && cnt[a] != rng[a].y - rng[a].x + 1) g.kb_contig = 0;
      if (cnt[a]) g.kbmax = std::max(g.kbmax, std::max(std::abs(rng[a].x), std::abs(rng[a].y)));
    }
    g.prune34 = (8 * g.kamax < 3 * n1 && 8 * g.kbmax < 3 * n2) ? (4 * g.kamax >= n1 ? 2 : 1) : 0;
    DMF(ctx->d_kb_rng, n1 * sizeof(int2));
    CKF(cudaMemcpyAsync(ctx->d_kb_rng, rng.data(), n1 * sizeof(int2), cudaMemcpyHostToDevice, ctx->st));
    CKF(cudaStreamSynchronize(ctx->st));  // (rng is a local)
    g.kb_rng = ctx->d_kb_rng;
  }

  // orbital blocks (zero padded)
  const size_t vb = ctx->vec_elems * sizeof(double);
  DMF(ctx->d_chi, vb);
  DMF(ctx->d_b1, vb);
  DMF(ctx->d_b2, vb);
  CKF(cudaMemsetAsync(ctx->d_chi, 0, vb, ctx->st));
  CKF(cudaMemsetAsync(ctx->d_b1, 0, vb, ctx->st));
  CKF(cudaMemsetAsync(ctx->d_b2, 0, vb, ctx->st));
  // per-CTA moment partials, then kDotBlocks block sums of the fixed-order reduction
  ctx->dots_cap = (size_t)ctx->npairs_max * g.nbatch;
  DMF(ctx->d_dots, (ctx->dots_cap + kDotBlocks) * 3 * sizeof(double));
  DMF(ctx->d_enl, (1 + kEnlBlocks) * sizeof(double));  // E_NL, then its block partials
  DMF(ctx->d_err, sizeof(int));
  CKF(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->st));
  const size_t vsz = is_fp64(ctx) ? sizeof(double) : sizeof(float);
  DMF(ctx->d_vp, (size_t)ctx->N * vsz);
  DMF(ctx->d_vks_tmp, (size_t)ctx->N * sizeof(double));
#undef DMF
#undef CKF
  *out = ctx;
  return SDFT_OK;
}

static void batch_detach(sdft_batch *b, sdft_ctx *c);

extern "C" int sdft_ctx_destroy(sdft_ctx *ctx) {
  if (!ctx) return SDFT_OK;
  cudaSetDevice(ctx->device);
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  void *ptrs[] = {ctx->d_cp_gstart, ctx->d_cp_gcount, ctx->d_col_ab, ctx->d_gkc, ctx->d_ak2, ctx->d_tw,
                  ctx->d_twf, ctx->d_vp, ctx->d_vks_tmp, ctx->d_pj, ctx->d_bk, ctx->d_w, ctx->d_z,
                  ctx->d_zwork, ctx->d_chi, ctx->d_b1, ctx->d_b2, ctx->d_fnl, ctx->d_acc, ctx->d_coef,
                  ctx->d_x, ctx->d_dots, ctx->d_mom, ctx->d_rho_part, ctx->d_rho, ctx->d_neg, ctx->d_noise_scratch,
                  ctx->d_enl, ctx->d_red, ctx->d_kb_rng,
                  ctx->d_err, ctx->d_pj_dig, ctx->d_bk_dig, ctx->d_c_dig,
                  ctx->d_z_dig, ctx->d_pj_sc, ctx->d_bk_sc, ctx->d_c_sc, ctx->d_z_sc, ctx->d_rowmax,
                  ctx->d_oz_part, ctx->d_kb_rs, ctx->d_kb_rc, ctx->d_gk, ctx->d_zsave, ctx->d_rowmax3};
  // a batch graph still holding the context: wait for its replays, drop the context from it
  for (sdft_batch *b : ctx->batches) batch_detach(b, ctx);
  ctx->batches.clear();
  for (void *p : ptrs) dev_free(p, ctx->st);
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  for (auto &t : ctx->tev_pending) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
  for (auto e : ctx->tev_free) cudaEventDestroy(e);
  if (ctx->st) cudaStreamDestroy(ctx->st);
  delete ctx;
  return SDFT_OK;
}

extern "C" int sdft_ctx_set_kinetic_cap(sdft_ctx *ctx, double gcut) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  ctx->gcut = gcut;
  std::vector<double> ak2(ctx->ncoef);
  sdft_ak2_kinetic(ctx->hmat, ctx->ncoef, ctx->ka.data(), ctx->kb.data(), ctx->kc.data(), gcut, ak2.data());
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(ctx->d_ak2, ak2.data(), ctx->ncoef * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  return SDFT_OK;
}

extern "C" int sdft_ctx_set_vks(sdft_ctx *ctx, const double *v) {
  if (!ctx || !v) return set_error(SDFT_ERR_ARG, "set_vks: null");
  cudaSetDevice(ctx->device);
  // host or device memory (a V_KS that sdft_vks_from_rho left on the device)
  CK(cudaMemcpyAsync(ctx->d_vks_tmp, v, (size_t)ctx->N * sizeof(double), cudaMemcpyDefault, ctx->st));
  if (ctx->fast) {
    if (is_fp64(ctx)) fast_vks_perm<double>(ctx->g, ctx->d_vks_tmp, (double *)ctx->d_vp, ctx->st);
    else fast_vks_perm<float>(ctx->g, ctx->d_vks_tmp, (float *)ctx->d_vp, ctx->st);
  } else if (is_fp64(ctx)) {
    launch_vks_transpose<double>(ctx->d_vks_tmp, (double *)ctx->d_vp, ctx->n1, ctx->n2, ctx->n3, ctx->st);
  } else {
    launch_vks_transpose<float>(ctx->d_vks_tmp, (float *)ctx->d_vp, ctx->n1, ctx->n2, ctx->n3, ctx->st);
  }
  ctx->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  ctx->have_v = true;
  return SDFT_OK;
}

extern "C" long long sdft_ctx_device_bytes(const sdft_ctx *ctx) { return ctx ? ctx->dev_bytes : 0; }
extern "C" void *sdft_ctx_stream(sdft_ctx *ctx) { return ctx ? (void *)ctx->st : nullptr; }
extern "C" long long sdft_launch_count(const sdft_ctx *ctx) { return ctx ? ctx->launches : 0; }
extern "C" int sdft_ctx_set_timing(sdft_ctx *ctx, int enable) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  ctx->timing = enable != 0;
  return SDFT_OK;
}

extern "C" int sdft_ctx_read_timing(sdft_ctx *ctx, double *ms, long long *count) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->st));
  for (auto &t : ctx->tev_pending) {
    float f = 0.f;
    if (cudaEventElapsedTime(&f, t.a, t.b) == cudaSuccess) {
      ctx->t_ms[t.kind] += f;
      ctx->t_n[t.kind] += 1;
    }
    ctx->tev_free.push_back(t.a);
    ctx->tev_free.push_back(t.b);
  }
  ctx->tev_pending.clear();
  for (int k = 0; k < SDFT_NKIND; k++) {
    if (ms) ms[k] = ctx->t_ms[k];
    if (count) count[k] = ctx->t_n[k];
    ctx->t_ms[k] = 0.0;
    ctx->t_n[k] = 0;
  }
  return SDFT_OK;
}

extern "C" int sdft_sync(sdft_ctx *ctx) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->st));
  CK(cudaGetLastError());
  int e = 0;
  CK(cudaMemcpyAsync(&e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (e) {
    // reported once: the word is cleared, so the context serves later calls
    // (the results of the work that timed out are not valid)
    CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return set_error(SDFT_ERR_TIMEOUT, "a bounded device wait gave up (tensor-core GEMM pipeline)");
  }
  return SDFT_OK;
}

// ---- events and the calling thread's device (host code without another CUDA binding)
extern "C" int sdft_set_device(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(SDFT_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return set_error(SDFT_ERR_ARG, "set_device: device index");
  CK(cudaSetDevice(device));
  return SDFT_OK;
}

extern "C" int sdft_event_create(int device, void **ev) {
  if (!ev) return set_error(SDFT_ERR_ARG, "event_create: null");
  *ev = nullptr;
  int r = sdft_set_device(device);
  if (r) return r;
  cudaEvent_t e = nullptr;
  CK(cudaEventCreateWithFlags(&e, cudaEventDefault));
  *ev = (void *)e;
  return SDFT_OK;
}

extern "C" int sdft_event_record(void *ev, void *stream) {
  if (!ev) return set_error(SDFT_ERR_ARG, "event_record: null event");
  CK(cudaEventRecord((cudaEvent_t)ev, (cudaStream_t)stream));
  return SDFT_OK;
}

extern "C" int sdft_event_query(void *ev, int *done) {
  if (!ev || !done) return set_error(SDFT_ERR_ARG, "event_query: null");
  const cudaError_t e = cudaEventQuery((cudaEvent_t)ev);
  if (e == cudaErrorNotReady) {
    cudaGetLastError();  // not-ready is not an error of the context
    *done = 0;
    return SDFT_OK;
  }
  CK(e);
  *done = 1;
  return SDFT_OK;
}

extern "C" int sdft_event_synchronize(void *ev) {
  if (!ev) return set_error(SDFT_ERR_ARG, "event_synchronize: null");
  CK(cudaEventSynchronize((cudaEvent_t)ev));
  return SDFT_OK;
}

extern "C" int sdft_event_elapsed_ms(void *ev0, void *ev1, float *ms) {
  if (!ev0 || !ev1 || !ms) return set_error(SDFT_ERR_ARG, "event_elapsed: null");
  CK(cudaEventElapsedTime(ms, (cudaEvent_t)ev0, (cudaEvent_t)ev1));
  return SDFT_OK;
}

extern "C" int sdft_event_destroy(void *ev) {
  if (ev) CK(cudaEventDestroy((cudaEvent_t)ev));
  return SDFT_OK;
}

extern "C" int sdft_set_device_memory_limit(int device, long long bytes) {
  if (device < 0 || device >= 64 || bytes < 0) return set_error(SDFT_ERR_ARG, "memory limit: device 0..63, bytes >= 0");
  DevAccount &acc = dev_account();
  std::lock_guard<std::mutex> lk(acc.mu);
  acc.limit[device] = bytes;
  return SDFT_OK;
}

extern "C" long long sdft_device_memory_in_use(int device) {
  if (device < 0 || device >= 64) return -1;
  DevAccount &acc = dev_account();
  std::lock_guard<std::mutex> lk(acc.mu);
  return acc.used[device];
}

extern "C" int sdft_ctx_selftest_wait(sdft_ctx *ctx, long long polls) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (polls < 1 || polls > kSelftestMaxPolls) return set_error(SDFT_ERR_ARG, "selftest_wait: polls in 1..2^22");
  cudaSetDevice(ctx->device);
  launch_selftest_wait(ctx->d_err, polls, ctx->st);
  ctx->launches++;
  CK(cudaGetLastError());
  return SDFT_OK;
}

// ---- KB projectors -------------------------------------------------------
int sdft_build_kb_device(sdft_ctx *ctx, const sdft_kb_desc *kb);  // sdft_kb.cu

extern "C" int sdft_ctx_set_kb(sdft_ctx *ctx, const sdft_kb_desc *kb) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  cudaSetDevice(ctx->device);
  return sdft_build_kb_device(ctx, kb);
}

// ---- hot path ---------------------------------------------------------------
extern "C" int sdft_upload_orbitals(sdft_ctx *ctx, int nstate, const double *cre, const double *cim) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (!cre || !cim) return set_error(SDFT_ERR_ARG, "upload: null");
  cudaSetDevice(ctx->device);
  if ((r = upload_block(ctx, ctx->d_chi, nstate, cre, cim))) return r;
  ctx->resident = nstate;
  return SDFT_OK;
}

extern "C" int sdft_hpsi(sdft_ctx *ctx, int nstate, const double *cre, const double *cim, double *fcre,
                         double *fcim, double *enl) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (!cre || !cim || !fcre || !fcim) return set_error(SDFT_ERR_ARG, "hpsi: null");
  cudaSetDevice(ctx->device);
  if ((r = upload_block(ctx, ctx->d_chi, nstate, cre, cim))) return r;
  ctx->resident = nstate;
  EpiArgs e = base_epi(ctx);
  e.mode = EPI_HPSI;
  e.OUT = ctx->d_b1;
  if ((r = apply_h(ctx, ctx->d_chi, nstate, e, enl != nullptr))) return r;
  if ((r = download_block(ctx, ctx->d_b1, nstate, fcre, fcim))) return r;
  if (enl) {
    if (ctx->P) CK(cudaMemcpyAsync(enl, ctx->d_enl, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    else *enl = 0.0;
  }
  CK(cudaStreamSynchronize(ctx->st));
  return SDFT_OK;
}

extern "C" int sdft_normh_cheby(sdft_ctx *ctx, int nstate, int ipoly, int cpy_flag, double scale,
                                double emean, double *cre, double *cim, double *wf1re, double *wf1im,
                                double *fcre, double *fcim) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (ipoly < 1 || !cre || !cim || !fcre || !fcim || (ipoly > 1 && (!wf1re || !wf1im)))
    return set_error(SDFT_ERR_ARG, "normh_cheby: bad argument");
  cudaSetDevice(ctx->device);
  if ((r = upload_block(ctx, ctx->d_chi, nstate, cre, cim))) return r;
  EpiArgs e = base_epi(ctx);
  const double prefact = -scale * emean, s1 = -scale * 0.25, s2 = -scale * 0.5;
  e.OUT = ctx->d_b2;
  if (ipoly == 1) {
    e.mode = EPI_CHEB1; e.s1 = s1; e.s2 = s2; e.pre = prefact;
  } else {
    if ((r = upload_block(ctx, ctx->d_b1, nstate, wf1re, wf1im))) return r;
    e.mode = EPI_CHEBK; e.s1 = 2 * s1; e.s2 = 2 * s2; e.pre = 2 * prefact; e.PREV = ctx->d_b1;
  }
  if ((r = apply_h(ctx, ctx->d_chi, nstate, e, false))) return r;
  if ((r = download_block(ctx, ctx->d_b2, nstate, fcre, fcim))) return r;
  CK(cudaStreamSynchronize(ctx->st));
  if (cpy_flag) {
    const size_t n = (size_t)nstate * ctx->ncoef * sizeof(double);
    if (ipoly > 1) { std::memcpy(wf1re, cre, n); std::memcpy(wf1im, cim, n); }
    std::memcpy(cre, fcre, n);
    std::memcpy(cim, fcim, n);
  }
  return SDFT_OK;
}

extern "C" int sdft_normh_newton(sdft_ctx *ctx, int nstate, double scale, double emean, double zn,
                                 double *cre, double *cim, double *fcre, double *fcim) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (!cre || !cim || !fcre || !fcim) return set_error(SDFT_ERR_ARG, "normh_newton: null");
  cudaSetDevice(ctx->device);
  if ((r = upload_block(ctx, ctx->d_chi, nstate, cre, cim))) return r;
  EpiArgs e = base_epi(ctx);
  e.mode = EPI_NEWTON;
  e.OUT = ctx->d_b1;
  e.s1 = -scale * 0.25; e.s2 = -scale * 0.5; e.pre = -scale * emean - zn;
  if ((r = apply_h(ctx, ctx->d_chi, nstate, e, false))) return r;
  if ((r = download_block(ctx, ctx->d_b1, nstate, fcre, fcim))) return r;
  CK(cudaStreamSynchronize(ctx->st));
  const size_t n = (size_t)nstate * ctx->ncoef * sizeof(double);
  std::memcpy(cre, fcre, n);  // normHNewtonHerm copies the force back
  std::memcpy(cim, fcim, n);
  return SDFT_OK;
}

static int upload_coef(sdft_ctx *ctx, const double *ec, size_t n) {
  int r = ensure_coef(ctx, n);
  if (r) return r;
  CK(cudaMemcpyAsync(ctx->d_coef, ec, n * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  return SDFT_OK;
}

extern "C" int sdft_filter_cheby_dev(sdft_ctx *ctx, int nstate, int L, int nmu, const double *ec,
                                     double scale, double emean) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (L < 2 || nmu < 1 || !ec) return set_error(SDFT_ERR_ARG, "filter_cheby: L >= 2, numChemPot >= 1");
  if (nstate > ctx->resident) return set_error(SDFT_ERR_STATE, "filter: orbitals not resident");
  cudaSetDevice(ctx->device);
  if ((r = upload_coef(ctx, ec, (size_t)L * nmu))) return r;
  if ((r = filter_cheby_core(ctx, nstate, L, nmu, scale, emean, false))) return r;
  ctx->filtered = nstate;
  return SDFT_OK;
}

extern "C" int sdft_filter_newton_dev(sdft_ctx *ctx, int nstate, int L, int nmu, const double *ec,
                                      const double *samp, double scale, double emean) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (L < 2 || nmu < 1 || !ec || !samp) return set_error(SDFT_ERR_ARG, "filter_newton: bad argument");
  if (nstate > ctx->resident) return set_error(SDFT_ERR_STATE, "filter: orbitals not resident");
  cudaSetDevice(ctx->device);
  if ((r = upload_coef(ctx, ec, (size_t)L * nmu))) return r;
  if ((r = filter_newton_core(ctx, nstate, L, nmu, samp, scale, emean))) return r;
  ctx->filtered = nstate;
  return SDFT_OK;
}

extern "C" int sdft_download_filtered(sdft_ctx *ctx, int nstate, int imu, double *re, double *im) {
  if (!ctx || !re || !im) return set_error(SDFT_ERR_ARG, "download: null");
  if (nstate < 1 || nstate > ctx->filtered || imu < 0 || imu >= ctx->acc_nmu)
    return set_error(SDFT_ERR_STATE, "download: no filtered orbitals");
  cudaSetDevice(ctx->device);
  int r = download_block(ctx, ctx->d_acc + (size_t)imu * ctx->vec_elems, nstate, re, im);
  if (r) return r;
  CK(cudaStreamSynchronize(ctx->st));
  return SDFT_OK;
}

extern "C" int sdft_filter_cheby(sdft_ctx *ctx, int nstate, const double *cre, const double *cim, int L,
                                 int nmu, const double *ec, double scale, double emean, double **sre,
                                 double **sim, double *moments) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (!cre || !cim || !ec || !sre || !sim || L < 2 || nmu < 1) return set_error(SDFT_ERR_ARG, "filter_cheby: bad argument");
  cudaSetDevice(ctx->device);
  if ((r = upload_block(ctx, ctx->d_chi, nstate, cre, cim))) return r;
  ctx->resident = nstate;
  if ((r = upload_coef(ctx, ec, (size_t)L * nmu))) return r;
  if (moments && (r = ensure_mom(ctx, (size_t)L * 3))) return r;
  if ((r = filter_cheby_core(ctx, nstate, L, nmu, scale, emean, moments != nullptr))) return r;
  ctx->filtered = nstate;
  for (int imu = 0; imu < nmu; imu++)
    if ((r = download_block(ctx, ctx->d_acc + (size_t)imu * ctx->vec_elems, nstate, sre[imu], sim[imu]))) return r;
  if (moments) {
    std::vector<double> h((size_t)L * 3);
    CK(cudaMemcpyAsync(h.data(), ctx->d_mom, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    moments[0] = h[1 * 3 + 1];
    for (int k = 1; k < L; k++) moments[k] = h[k * 3 + 0];
    moments[L] = 0.0;
  }
  CK(cudaStreamSynchronize(ctx->st));
  return SDFT_OK;
}

extern "C" int sdft_filter_newton(sdft_ctx *ctx, int nstate, const double *cre, const double *cim, int L,
                                  int nmu, const double *ec, const double *samp, double scale, double emean,
                                  double **sre, double **sim) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (!cre || !cim || !ec || !samp || !sre || !sim || L < 2 || nmu < 1)
    return set_error(SDFT_ERR_ARG, "filter_newton: bad argument");
  cudaSetDevice(ctx->device);
  if ((r = upload_block(ctx, ctx->d_chi, nstate, cre, cim))) return r;
  ctx->resident = nstate;
  if ((r = upload_coef(ctx, ec, (size_t)L * nmu))) return r;
  if ((r = filter_newton_core(ctx, nstate, L, nmu, samp, scale, emean))) return r;
  ctx->filtered = nstate;
  for (int imu = 0; imu < nmu; imu++)
    if ((r = download_block(ctx, ctx->d_acc + (size_t)imu * ctx->vec_elems, nstate, sre[imu], sim[imu]))) return r;
  CK(cudaStreamSynchronize(ctx->st));
  return SDFT_OK;
}

extern "C" int sdft_cheby_moments_dev(sdft_ctx *ctx, int nstate, int L, double scale, double emean,
                                      double *moments) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (L < 2 || !moments) return set_error(SDFT_ERR_ARG, "moments: bad argument");
  if (nstate > ctx->resident) return set_error(SDFT_ERR_STATE, "moments: orbitals not resident");
  cudaSetDevice(ctx->device);
  return moments_core(ctx, nstate, L, scale, emean, moments);
}

extern "C" int sdft_cheby_moments(sdft_ctx *ctx, int nstate, const double *cre, const double *cim, int L,
                                  double scale, double emean, double *moments) {
  int r = check_ready(ctx, nstate);
  if (r) return r;
  if (!cre || !cim || !moments || L < 2) return set_error(SDFT_ERR_ARG, "moments: bad argument");
  cudaSetDevice(ctx->device);
  if ((r = upload_block(ctx, ctx->d_chi, nstate, cre, cim))) return r;
  ctx->resident = nstate;
  return moments_core(ctx, nstate, L, scale, emean, moments);
}

// Density of the orbitals held in `vec`.
static int density_core(sdft_ctx *ctx, const double *vec, int nstate, double scale) {
  int r, chunk;
  const int npairs = (nstate + 1) / 2;
  if ((r = fp64_chunk(ctx, npairs, &chunk))) return r;
  const int nsplit = npairs;  // one |psi|^2 plane set per pair, summed in pair order
  if (nsplit > ctx->rho_split) {
    if ((r = grow(ctx, (void **)&ctx->d_rho_part, (size_t)ctx->rho_split * ctx->N * 8,
                  (size_t)nsplit * ctx->N * sizeof(double))))
      return r;
    ctx->rho_split = nsplit;
  }
  if (!ctx->d_rho) DM(ctx->d_rho, (size_t)ctx->N * sizeof(double));
  // one transform per pair (against 2 per pair per filter step): FP64 in
  // every precision, in chunks of pairs that fit the column scratch
  for (int p0 = 0; p0 < npairs; p0 += chunk) {
    const int np = std::min(chunk, npairs - p0);
    double *part = ctx->d_rho_part + (size_t)p0 * ctx->N;
    if (ctx->fast) {
      { TScope ts(ctx, 0); fast_stage_a<double>(ctx->g, vec, nstate, p0, np, ctx->d_x, ctx->st); }
      { TScope ts(ctx, 5); fast_stage_b_density<double>(ctx->g, ctx->d_x, np, part, ctx->st); }
    } else {
      { TScope ts(ctx, 0); launch_stage_a<double>(ctx->g, vec, nstate, p0, np, ctx->d_x, ctx->st); }
      { TScope ts(ctx, 5); launch_stage_b_density<double>(ctx->g, ctx->d_x, np, np, part, ctx->st); }
    }
    ctx->launches += 2;
  }
  { TScope ts(ctx, 7); launch_density_reduce(ctx->d_rho_part, nsplit, ctx->N, scale, ctx->d_rho, ctx->st); }
  ctx->launches += 1;
  CK(cudaGetLastError());
  return SDFT_OK;
}

extern "C" int sdft_density(sdft_ctx *ctx, int nstate, const double *cre, const double *cim, double *rho) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (nstate < 1 || nstate > ctx->max_states || !cre || !cim || !rho) return set_error(SDFT_ERR_ARG, "density: bad argument");
  cudaSetDevice(ctx->device);
  int r = upload_block(ctx, ctx->d_b2, nstate, cre, cim);
  if (r) return r;
  if ((r = density_core(ctx, ctx->d_b2, nstate, 1.0))) return r;
  CK(cudaMemcpyAsync(rho, ctx->d_rho, (size_t)ctx->N * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SDFT_OK;
}

extern "C" int sdft_density_dev(sdft_ctx *ctx, int nstate, int imu, double scale, double *rho) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (nstate < 1 || nstate > ctx->filtered || imu < 0 || imu >= ctx->acc_nmu)
    return set_error(SDFT_ERR_STATE, "density_dev: no filtered orbitals");
  cudaSetDevice(ctx->device);
  int r = density_core(ctx, ctx->d_acc + (size_t)imu * ctx->vec_elems, nstate, scale);
  if (r) return r;
  if (rho) {
    // host or device destination (unified addressing)
    CK(cudaMemcpyAsync(rho, ctx->d_rho, (size_t)ctx->N * sizeof(double), cudaMemcpyDefault, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  return SDFT_OK;
}

// Noise: signs of gaussran2 on the device (sdft_noise.cu: the DURAND
// sequence jumped ahead per thread, identical to the host generator), then
// the FFT to G.
static int noise_core(sdft_ctx *ctx, int nstate, double seed, int np_states, int myid) {
  if (np_states < 1 || myid < 0 || myid >= np_states) return set_error(SDFT_ERR_ARG, "noise: rank");
  std::vector<double> seeds(np_states);
  noise_rank_seeds(seed, np_states, seeds.data());
  double q = seeds[myid];
  const size_t n = (size_t)nstate * ctx->N;
  if (n > ctx->neg_cap) {
    int r0 = grow(ctx, (void **)&ctx->d_neg, ctx->neg_cap, n);
    if (r0) return r0;
    ctx->neg_cap = n;
  }
  if (!ctx->d_noise_scratch) DM(ctx->d_noise_scratch, noise_scratch_bytes());
  {
    int nk = 0, r0 = device_gauss_signs((long long)n, &q, ctx->d_neg, ctx->d_noise_scratch, ctx->st, &nk);
    ctx->launches += nk;
    if (r0) return r0;
  }
  const int npairs = (nstate + 1) / 2;
  int r, chunk;
  if ((r = fp64_chunk(ctx, npairs, &chunk))) return r;
  CK(cudaMemsetAsync(ctx->d_chi, 0, ctx->vec_elems * sizeof(double), ctx->st));
  // the noise orbitals are input data: FP64 transforms in every precision
  for (int p0 = 0; p0 < npairs; p0 += chunk) {
    const int np = std::min(chunk, npairs - p0);
    EpiArgs e = base_epi(ctx);
    e.mode = EPI_NOISE;
    e.nstate = nstate;
    e.pair0 = p0;
    e.OUT = ctx->d_chi;
    e.invN = 1.0 / (double)ctx->N;
    if (ctx->fast) {
      { TScope ts(ctx, 6); fast_stage_b_noise<double>(ctx->g, ctx->d_neg, nstate, p0, np, ctx->d_x, ctx->st); }
      { TScope ts(ctx, 2); fast_stage_c<double>(ctx->g, ctx->d_x, e, np, ctx->st); }
    } else {
      { TScope ts(ctx, 6); launch_stage_b_noise<double>(ctx->g, ctx->d_neg, nstate, p0, np, ctx->d_x, ctx->st); }
      { TScope ts(ctx, 2); launch_stage_c<double>(ctx->g, ctx->d_x, e, np, ctx->st); }
    }
    ctx->launches += 2;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  ctx->resident = nstate;
  return SDFT_OK;
}

extern "C" int sdft_noise_real_dev(sdft_ctx *ctx, int nstate, double seed, int np_states, int myid) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (nstate < 1 || nstate > ctx->max_states) return set_error(SDFT_ERR_ARG, "noise: nstate");
  cudaSetDevice(ctx->device);
  return noise_core(ctx, nstate, seed, np_states, myid);
}

extern "C" int sdft_noise_real(sdft_ctx *ctx, int nstate, double seed, int np_states, int myid, double *cre,
                               double *cim) {
  if (!ctx || !cre || !cim) return set_error(SDFT_ERR_ARG, "noise: null");
  if (nstate < 1 || nstate > ctx->max_states) return set_error(SDFT_ERR_ARG, "noise: nstate");
  cudaSetDevice(ctx->device);
  int r = noise_core(ctx, nstate, seed, np_states, myid);
  if (r) return r;
  if ((r = download_block(ctx, ctx->d_chi, nstate, cre, cim))) return r;
  CK(cudaStreamSynchronize(ctx->st));
  return SDFT_OK;
}

// ============================================================================
// Tuning knob and batched filters (one CUDA graph over several contexts)
// ============================================================================
// ---- spectral bounds and energies --------------------------------------------
static int ensure_red(sdft_ctx *ctx) {
  if (ctx->d_red) return SDFT_OK;
  DM(ctx->d_red, (kRedBlocks + 8) * sizeof(double));
  return SDFT_OK;
}

// Lanczos with device-resident vectors: c in row 0 of d_chi, H c in d_b1,
// the previous vector in d_b2; alpha_k, beta_k read back per step.
extern "C" int sdft_lanczos_bounds(sdft_ctx *ctx, int nstep, const double *v0re, const double *v0im, double margin,
                                   double *alpha, double *beta, int *nsteps, double *emin, double *emax) {
  int r = check_ready(ctx, 1);
  if (r) return r;
  if (nstep < 1 || !v0re || !v0im || !emin || !emax) return set_error(SDFT_ERR_ARG, "lanczos_bounds: bad argument");
  cudaSetDevice(ctx->device);
  if ((r = ensure_red(ctx))) return r;
  const int nc = ctx->ncoef, ngp = ctx->ngp;
  double *c = ctx->d_chi, *f = ctx->d_b1, *p = ctx->d_b2;
  double *part = ctx->d_red, *sc = ctx->d_red + kRedBlocks;
  ctx->resident = 0;
  if ((r = upload_block(ctx, c, 1, v0re, v0im))) return r;
  launch_half_dot(c, c, nc, ngp, part, sc, ctx->st);
  launch_lz_div(c, sc, nc, ngp, ctx->st);
  ctx->launches += 3;
  std::vector<double> al, be;
  double b = 0.0;
  for (int k = 0; k < nstep; k++) {
    EpiArgs e = base_epi(ctx);
    e.mode = EPI_HPSI;
    e.OUT = f;
    if ((r = apply_h(ctx, c, 1, e, false))) return r;
    launch_lz_hc(f, nc, ngp, ctx->st);
    launch_half_dot(c, f, nc, ngp, part, sc, ctx->st);                 // alpha
    launch_lz_w(f, c, k > 0 ? p : nullptr, sc, b, nc, ngp, ctx->st);  // w = H c - alpha c - beta p
    launch_half_dot(f, f, nc, ngp, part, sc + 1, ctx->st);             // |w|^2
    ctx->launches += 6;
    double h2[2];
    CK(cudaMemcpyAsync(h2, sc, sizeof h2, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    al.push_back(h2[0]);
    b = std::sqrt(std::max(h2[1], 0.0));
    be.push_back(b);
    if (b < 1e-12) break;
    launch_lz_next(f, c, p, b, nc, ngp, ctx->st);
    ctx->launches++;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  const int k = (int)al.size();
  for (int i = 0; i < k; i++) {
    if (alpha) alpha[i] = al[i];
    if (beta) beta[i] = be[i];
  }
  if (nsteps) *nsteps = k;
  double lo = 0.0, hi = 0.0;
  tridiag_extremes(al.data(), be.data(), k, &lo, &hi);
  *emin = lo - margin;
  *emax = hi + margin;
  return SDFT_OK;
}

extern "C" int sdft_energy_chempot_dev(sdft_ctx *ctx, int nstate, int imu, double occ, int nsto_total,
                                       double *energy_ke, double *energy_pnl) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (nstate < 1 || nstate > ctx->filtered || imu < 0 || imu >= ctx->acc_nmu)
    return set_error(SDFT_ERR_STATE, "energy_chempot_dev: no filtered orbitals");
  if (nsto_total < 1 || !energy_ke || !energy_pnl) return set_error(SDFT_ERR_ARG, "energy_chempot_dev: bad argument");
  cudaSetDevice(ctx->device);
  int r = ensure_red(ctx);
  if (r) return r;
  const double *v = ctx->d_acc + (size_t)imu * ctx->vec_elems;
  double *sc = ctx->d_red + kRedBlocks;
  launch_ekin(v, nstate, ctx->ncoef, ctx->ngp, ctx->d_ak2, ctx->d_red, sc + 2, ctx->st);
  ctx->launches += 2;
  double ek = 0.0, en = 0.0;
  if (ctx->P) {
    if ((r = run_kb(ctx, v, nstate, true, false))) return r;
    CK(cudaMemcpyAsync(&en, ctx->d_enl, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  }
  CK(cudaMemcpyAsync(&ek, sc + 2, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->st));
  *energy_ke = occ * 0.5 * ek / nsto_total;
  *energy_pnl = occ * en / nsto_total;
  return SDFT_OK;
}

// KB nonlocal atomic forces of the filtered orbitals of chemical potential
// imu (calcEnergyForce, stodft/calc-nuclei-force.c:33-480, its nonlocal part:
// calcNlPseudoPostScf then occNumber / numStateStoUp).  dZ/dR_d is the
// projection of i G_d c, so the force takes the same projection GEMM as H c:
// once on c (Z, kept) and once per direction; a per-atom reduction in fixed
// order forms F = -2 sum w Z dZ.
extern "C" int sdft_nl_force_dev(sdft_ctx *ctx, int nstate, int imu, double occ, int nsto_total, double *fatm,
                                 double *energy_pnl) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (nstate < 1 || nstate > ctx->filtered || imu < 0 || imu >= ctx->acc_nmu)
    return set_error(SDFT_ERR_STATE, "nl_force_dev: no filtered orbitals");
  if (nsto_total < 1 || !fatm) return set_error(SDFT_ERR_ARG, "nl_force_dev: bad argument");
  if (ctx->P == 0) {
    if (energy_pnl) *energy_pnl = 0.0;
    return SDFT_OK;
  }
  cudaSetDevice(ctx->device);
  int r;
  const size_t zel = (size_t)ctx->s_pad * ctx->Ppad;
  if (!ctx->d_zsave) {
    if ((r = dmalloc(ctx, (void **)&ctx->d_zsave, zel * sizeof(double)))) return r;
    ctx->kb_bytes += (long long)(zel * sizeof(double));  // released with the KB buffers
  }
  if (ctx->oz && !ctx->d_rowmax3) {
    const size_t b = (size_t)3 * ctx->s_pad * sizeof(unsigned long long);
    if ((r = dmalloc(ctx, (void **)&ctx->d_rowmax3, b))) return r;
    ctx->kb_bytes += (long long)b;
  }
  double *d_f = nullptr;
  if ((r = dev_alloc(ctx->device, ctx->st, (void **)&d_f, (size_t)3 * ctx->kb_natm * sizeof(double)))) return r;
  const double *v = ctx->d_acc + (size_t)imu * ctx->vec_elems;
  const double scale = occ / (double)nsto_total;
  double en = 0.0;
  std::vector<double> h((size_t)3 * ctx->kb_natm);
  cudaError_t e = cudaSuccess;
#define CKG(call)                       \
  do {                                  \
    if ((e = (call)) != cudaSuccess) goto out; \
  } while (0)
  if ((r = run_kb(ctx, v, nstate, true, false))) goto out;
  CKG(cudaMemcpyAsync(ctx->d_zsave, ctx->d_z, (size_t)nstate * ctx->Ppad * sizeof(double), cudaMemcpyDeviceToDevice,
                      ctx->st));
  if (ctx->oz) {  // row maxima of the three i G_d c in one pass over c
    launch_oz_rowmax_igc3(v, ctx->d_gk, ctx->ngp, ctx->ncoef, nstate, ctx->d_rowmax3, ctx->st);
    ctx->launches++;
  }
  for (int d = 0; d < 3; d++) {
    const double *gk = ctx->d_gk + (size_t)d * ctx->ngp;
    if (ctx->oz) {  // the digit pass forms i G_d c from c itself
      if ((r = run_kb_oz(ctx, v, nstate, false, false, gk, ctx->d_rowmax3 + (size_t)d * nstate))) goto out;
    } else {
      // i G_d c into the back-projection buffer, which this call does not otherwise use
      launch_dcoef(v, nstate, ctx->ncoef, ctx->ngp, gk, ctx->d_fnl, ctx->st);
      ctx->launches++;
      if ((r = run_kb(ctx, ctx->d_fnl, nstate, false, false))) goto out;
    }
    launch_nl_force_atoms(ctx->d_zsave, ctx->d_z, ctx->Ppad, ctx->d_w, ctx->d_kb_rs, ctx->d_kb_rc, ctx->kb_natm,
                          nstate, scale, d, d_f, ctx->st);
    ctx->launches++;
  }
  // (the direction projections leave d_enl alone: it still holds E_NL of c)
  CKG(cudaMemcpyAsync(h.data(), d_f, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CKG(cudaMemcpyAsync(&en, ctx->d_enl, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CKG(cudaGetLastError());
  CKG(cudaStreamSynchronize(ctx->st));
  std::memcpy(fatm, h.data(), h.size() * sizeof(double));
  if (energy_pnl) *energy_pnl = scale * en;
out:
  dev_free(d_f, ctx->st);
  if (!r && e != cudaSuccess) r = set_error(SDFT_ERR_CUDA, cudaGetErrorString(e));
  return r;
#undef CKG
}

extern "C" int sdft_ctx_set_plane_threads(sdft_ctx *ctx, int nt) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (nt != 0 && nt != 128 && nt != 256) return set_error(SDFT_ERR_ARG, "plane_threads: 0 (default), 128 or 256");
  if (nt == 128 && (is_fp64(ctx) || !ctx->fast))
    return set_error(SDFT_ERR_UNSUPPORTED, "plane_threads: 128 exists for the FP32 fast plane stage only");
  ctx->g.plane_nt = nt == 0 ? default_plane_threads(ctx) : nt;
  return SDFT_OK;
}

extern "C" int sdft_ctx_set_gemm_bn(sdft_ctx *ctx, int bn) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (bn != 0 && bn != 64 && bn != 128) return set_error(SDFT_ERR_ARG, "gemm_bn: 0 (per call), 64 or 128");
  ctx->gemm_bn = bn;
  return SDFT_OK;
}

extern "C" int sdft_ctx_set_gemm_split(sdft_ctx *ctx, int split) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  if (split < 0 || split > 64) return set_error(SDFT_ERR_ARG, "gemm_split: 0 (cost model) or 1..64");
  ctx->gemm_split = split;
  return SDFT_OK;
}

// Replace an idle stream by one of the given CUDA priority (lower = more
// urgent), clamped to the device's range.
static int replace_stream(cudaStream_t *st, int priority) {
  int least = 0, greatest = 0;
  CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  priority = std::min(least, std::max(greatest, priority));
  cudaStream_t ns = nullptr;
  CK(cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, priority));
  if (*st) {
    cudaStreamSynchronize(*st);
    cudaStreamDestroy(*st);
  }
  *st = ns;
  return SDFT_OK;
}

extern "C" int sdft_ctx_set_priority(sdft_ctx *ctx, int priority) {
  if (!ctx) return set_error(SDFT_ERR_ARG, "null context");
  cudaSetDevice(ctx->device);
  return replace_stream(&ctx->st, priority);
}

struct sdft_batch {
  int device = 0;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<sdft_ctx *> ctxs;
  std::vector<int> nstate;
  std::vector<cudaEvent_t> evs;  // [0] fork, [1..n] joins
  long long launches_per_replay = 0;
};

namespace sdft {
// Every buffer the filter + density path touches, sized up front (no
// allocation may happen while the stream is captured).
static int prepare_filter(sdft_ctx *ctx, int nstate, int L) {
  int r;
  if ((r = ensure_coef(ctx, (size_t)L))) return r;
  if ((r = ensure_acc(ctx, 1))) return r;
  const int npairs = (nstate + 1) / 2;
  if ((r = ensure_x(ctx, std::max(npairs, 2)))) return r;  // as fp64_chunk needs it
  if (npairs > ctx->rho_split) {
    if ((r = grow(ctx, (void **)&ctx->d_rho_part, (size_t)ctx->rho_split * ctx->N * 8,
                  (size_t)npairs * ctx->N * sizeof(double))))
      return r;
    ctx->rho_split = npairs;
  }
  if (!ctx->d_rho && (r = dmalloc(ctx, (void **)&ctx->d_rho, (size_t)ctx->N * sizeof(double)))) return r;
  return SDFT_OK;
}
}  // namespace sdft

static void batch_detach(sdft_batch *b, sdft_ctx *c) {
  if (b->st) cudaStreamSynchronize(b->st);
  b->ctxs.erase(std::remove(b->ctxs.begin(), b->ctxs.end(), c), b->ctxs.end());
}

extern "C" int sdft_batch_destroy(sdft_batch *b) {
  if (!b) return SDFT_OK;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  for (sdft_ctx *c : b->ctxs) c->batches.erase(std::remove(c->batches.begin(), c->batches.end(), b), c->batches.end());
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cudaEvent_t e : b->evs) cudaEventDestroy(e);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return SDFT_OK;
}

extern "C" int sdft_batch_create(int n, sdft_ctx *const *ctxs, const int *nstate, const int *L,
                                 const double *const *coeffs, const double *scale, const double *emean,
                                 const double *occ_over_nsto, sdft_batch **out) {
  if (!out || n < 1 || !ctxs || !nstate || !L || !coeffs || !scale || !emean || !occ_over_nsto)
    return set_error(SDFT_ERR_ARG, "batch_create: bad argument");
  *out = nullptr;
  const int dev = ctxs[0] ? ctxs[0]->device : 0;
  for (int i = 0; i < n; i++) {
    sdft_ctx *c = ctxs[i];
    if (!c || c->device != dev) return set_error(SDFT_ERR_ARG, "batch_create: contexts must share one device");
    int r = check_ready(c, nstate[i]);
    if (r) return r;
    if (L[i] < 2 || !coeffs[i]) return set_error(SDFT_ERR_ARG, "batch_create: L >= 2 and coefficients required");
    if (nstate[i] > c->resident) return set_error(SDFT_ERR_STATE, "batch_create: orbitals not resident");
    for (int j = 0; j < i; j++)
      if (ctxs[j] == c) return set_error(SDFT_ERR_ARG, "batch_create: a context appears twice");
  }
  cudaSetDevice(dev);
  sdft_batch *b = new sdft_batch;
  b->device = dev;
  auto fail = [&](int code) { sdft_batch_destroy(b); return code; };
  auto ck = [&](cudaError_t e) { return e == cudaSuccess ? SDFT_OK : set_error(SDFT_ERR_CUDA, cudaGetErrorString(e)); };
  int r;
  if ((r = ck(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)))) return fail(r);
  b->evs.resize(n + 1, nullptr);
  for (auto &e : b->evs)
    if ((r = ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)))) return fail(r);
  // buffers and coefficients, outside the capture
  for (int i = 0; i < n; i++) {
    sdft_ctx *c = ctxs[i];
    if ((r = prepare_filter(c, nstate[i], L[i]))) return fail(r);
    if ((r = ck(cudaMemcpyAsync(c->d_coef, coeffs[i], (size_t)L[i] * sizeof(double), cudaMemcpyHostToDevice,
                                c->st))))
      return fail(r);
    if ((r = ck(cudaStreamSynchronize(c->st)))) return fail(r);
    b->ctxs.push_back(c);
    b->nstate.push_back(nstate[i]);
  }
  // capture: fork every context's stream from the batch stream, record its
  // filter + density, join back
  std::vector<bool> timing(n);
  long long l0 = 0;
  for (int i = 0; i < n; i++) { timing[i] = ctxs[i]->timing; ctxs[i]->timing = false; l0 += ctxs[i]->launches; }
  if ((r = ck(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal)))) return fail(r);
  int rc = ck(cudaEventRecord(b->evs[0], b->st));
  for (int i = 0; i < n && rc == SDFT_OK; i++) {
    sdft_ctx *c = ctxs[i];
    if ((rc = ck(cudaStreamWaitEvent(c->st, b->evs[0], 0)))) break;
    if ((rc = filter_cheby_core(c, nstate[i], L[i], 1, scale[i], emean[i], false))) break;
    if ((rc = density_core(c, c->d_acc, nstate[i], occ_over_nsto[i]))) break;
    if ((rc = ck(cudaEventRecord(b->evs[i + 1], c->st)))) break;
    if ((rc = ck(cudaStreamWaitEvent(b->st, b->evs[i + 1], 0)))) break;
  }
  cudaGraph_t g = nullptr;
  cudaError_t ee = cudaStreamEndCapture(b->st, &g);
  for (int i = 0; i < n; i++) ctxs[i]->timing = timing[i];
  b->graph = g;
  if (rc) return fail(rc);
  if ((r = ck(ee))) return fail(r);
  if ((r = ck(cudaGraphInstantiate(&b->exec, b->graph, 0)))) return fail(r);
  long long l1 = 0;
  for (int i = 0; i < n; i++) { l1 += ctxs[i]->launches; ctxs[i]->filtered = nstate[i]; }
  b->launches_per_replay = l1 - l0;
  for (sdft_ctx *c : b->ctxs) c->batches.push_back(b);
  *out = b;
  return SDFT_OK;
}

extern "C" int sdft_batch_launch(sdft_batch *b) {
  if (!b || !b->exec) return set_error(SDFT_ERR_ARG, "batch_launch: no batch");
  cudaSetDevice(b->device);
  CK(cudaGraphLaunch(b->exec, b->st));
  return SDFT_OK;
}

extern "C" int sdft_batch_sync(sdft_batch *b) {
  if (!b) return set_error(SDFT_ERR_ARG, "batch_sync: no batch");
  cudaSetDevice(b->device);
  CK(cudaStreamSynchronize(b->st));
  for (sdft_ctx *c : b->ctxs) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (e) return set_error(SDFT_ERR_TIMEOUT, "a bounded device wait gave up (tensor-core GEMM pipeline)");
  }
  return SDFT_OK;
}

extern "C" int sdft_batch_set_priority(sdft_batch *b, int priority) {
  if (!b) return set_error(SDFT_ERR_ARG, "batch_set_priority: no batch");
  cudaSetDevice(b->device);
  return replace_stream(&b->st, priority);
}

extern "C" void *sdft_batch_stream(sdft_batch *b) { return b ? (void *)b->st : nullptr; }
extern "C" long long sdft_batch_kernel_count(const sdft_batch *b) { return b ? b->launches_per_replay : 0; }

extern "C" int sdft_download_density(sdft_ctx *ctx, double *rho) {
  if (!ctx || !rho) return set_error(SDFT_ERR_ARG, "download_density: null");
  if (!ctx->d_rho) return set_error(SDFT_ERR_STATE, "download_density: no density computed yet");
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(rho, ctx->d_rho, (size_t)ctx->N * sizeof(double), cudaMemcpyDefault, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return SDFT_OK;
}
