// sdft_ctx.h -- device context of the filter-path library (internal).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "sdft_internal.h"
#include "sdft_kernels.cuh"
#include "sdft_gemm_oz.cuh"

struct sdft_batch;

struct sdft_ctx {
  int device = 0;
  int prec = SDFT_PREC_FP64;
  cudaStream_t st = nullptr;
  // geometry
  int n1 = 0, n2 = 0, n3 = 0, N = 0, ncoef = 0, ngp = 0;
  double hmat[9];
  double vol = 0.0;
  std::vector<int> ka, kb, kc;
  sdft::SphereCols cols;
  sdft::DevGeom g{};
  int max_states = 0, s_pad = 0, npairs_max = 0;
  size_t vec_elems = 0;  // doubles per orbital block (s_pad*2*ngp)
  // device geometry arrays
  int *d_cp_gstart = nullptr, *d_cp_gcount = nullptr, *d_col_ab = nullptr, *d_gkc = nullptr;
  double *d_ak2 = nullptr;
  double2 *d_tw = nullptr;  // n1+n2+n3
  float2 *d_twf = nullptr;
  // potential
  void *d_vp = nullptr;     // [n3][n1][n2] (double or float)
  double *d_vks_tmp = nullptr;
  bool have_v = false;
  // KB
  int P = 0, Ppad = 0, Mpad2 = 0;
  double *d_pj = nullptr, *d_bk = nullptr, *d_w = nullptr, *d_z = nullptr, *d_zwork = nullptr;
  // KB atomic forces: projector rows of each atom, G (cartesian, per coefficient), saved Z
  int kb_natm = 0;
  int *d_kb_rs = nullptr, *d_kb_rc = nullptr;
  double *d_gk = nullptr;  // [3][ngp], G = 0 and padding 0
  double *d_zsave = nullptr;
  unsigned long long *d_rowmax3 = nullptr;  // row maxima of i G_d c, d = x, y, z (3 s_pad words)
  size_t zwork_elems = 0;
  // orbital blocks
  double *d_chi = nullptr, *d_b1 = nullptr, *d_b2 = nullptr, *d_fnl = nullptr;
  double *d_acc = nullptr;
  int acc_nmu = 0;
  double *d_coef = nullptr;
  size_t coef_cap = 0;
  // scratch
  void *d_x = nullptr;
  size_t x_bytes = 0;
  double *d_dots = nullptr;
  size_t dots_cap = 0;  // CTA partial slots of d_dots (kDotBlocks*3 block sums follow them)
  double *d_mom = nullptr;
  size_t mom_cap = 0;
  double *d_rho_part = nullptr, *d_rho = nullptr;
  int rho_split = 0;
  unsigned char *d_neg = nullptr;
  size_t neg_cap = 0;
  void *d_noise_scratch = nullptr;  // stop flag + phi margin list of the sign generator
  std::vector<sdft_batch *> batches;  // graphs that replay this context's filter
  double *d_enl = nullptr;
  double *d_red = nullptr;  // reduction partials + scalars (Lanczos, energies)
  int2 *d_kb_rng = nullptr;  // per plane row: signed kb range of its sphere columns
  // state
  int resident = 0;          // orbitals in d_chi
  int filtered = 0;          // orbitals with results in d_acc
  long long launches = 0;
  long long dev_bytes = 0;
  long long kb_bytes = 0;  // the part of dev_bytes held by the KB buffers (released by a rebuild)
  double gcut = 0.0;
  bool fast = false;  // compile-time-edge FFT kernels available
  bool fft64 = true;  // FFT scratch / V_KS in FP64 (plain form)
  // mixed precision KB GEMMs (Ozaki scheme on INT8 tensor cores)
  bool oz = false;
  int s_oz = 0;                                   // orbital rows of the digit arrays (multiple of 128)
  int kp_oz = 0;                                  // K1 rounded up to 64 (digit row pitch)
  int8_t *d_pj_dig = nullptr, *d_bk_dig = nullptr, *d_c_dig = nullptr, *d_z_dig = nullptr;
  double *d_pj_sc = nullptr, *d_bk_sc = nullptr, *d_c_sc = nullptr, *d_z_sc = nullptr;
  unsigned long long *d_rowmax = nullptr;
  double *d_oz_part = nullptr;
  size_t oz_part_elems = 0;
  sdft::OzGemm om1{}, om2{};
  CUtensorMap om1_tb64{}, om2_tb64{};  // the B operands' maps with 64-row boxes (64-wide tiles)
  // Inside a filter / moments loop, stage C records the per-orbital max of
  // the vector it writes (d_rowmax), so the next projection can form that
  // vector's digits without another pass over it.
  int gemm_split = 0;                // projection split-K override (0: cost model)
  int gemm_bn = 0;                   // KB GEMM tile width: 0 = per call (64 where it pads less), 64 or 128
  bool track_omax = false;
  const double *omax_vec = nullptr;  // vector whose row maxima d_rowmax holds
  int omax_n = 0;
  int rowmax_zero_n = 0;             // d_rowmax[0, n) known to be zero
  const double *x_vec = nullptr;     // vector whose packed columns d_x holds (fast path, in loops)
  int x_n = 0;
  int *d_err = nullptr;
  // per-kind event timing (sdft_ctx_set_timing)
  bool timing = false;
  struct TEv { int kind; cudaEvent_t a, b; };
  std::vector<TEv> tev_pending;
  std::vector<cudaEvent_t> tev_free;
  double t_ms[8] = {0};
  long long t_n[8] = {0};
};

namespace sdft {
int dmalloc(sdft_ctx *c, void **p, size_t bytes);

// RAII event pair around the launches of one kernel kind.
struct TScope {
  sdft_ctx *c;
  int kind;
  cudaEvent_t a = nullptr;
  static cudaEvent_t get(sdft_ctx *c) {
    if (!c->tev_free.empty()) { cudaEvent_t e = c->tev_free.back(); c->tev_free.pop_back(); return e; }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  TScope(sdft_ctx *ctx, int k) : c(ctx), kind(k) {
    if (c->timing) { a = get(c); cudaEventRecord(a, c->st); }
  }
  ~TScope() {
    if (c->timing) {
      cudaEvent_t b = get(c);
      cudaEventRecord(b, c->st);
      c->tev_pending.push_back({kind, a, b});
    }
  }
};
}
