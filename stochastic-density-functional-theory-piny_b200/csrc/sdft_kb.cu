// sdft_kb.cu -- Kleinman-Bylander projector matrices for the GEMM form of
// the nonlocal term.
//
// The reference accumulates, per G vector and per channel (atom, l, m),
//   Z_r/Z_i += linear combinations of Re/Im c(G) e^{iG.R} v_l(|G|) Y_lm
// (getNlmatFilter, stodft/reduced-energy/cp-energy-eext-stodft.c:1105-1169;
// G = 0 term get_nlmat0, energy/cp/cp_energy_eext_nonloc.c:1083), and the
// force  f(G) -= (4/Omega) vnorm v_l conj(e^{iG.R} Y_lm) Z  (get_nlfor,
// cp_energy_eext_nonloc.c:2136-2173; G = 0: get_nlfor0 :2229).  Both maps
// are linear in the orbital coefficients, so they are written here as two
// dense real matrices over k = (Re c(G), Im c(G)):
//   Z[u] = sum_k Pj[u][k] c[k],     f[k] += sum_u Bk[k][u] Z[u].
// For each (atom, l) only 2l+1 of the 2(2l+1) real Z components are
// independent: m = 0 has a vanishing Re (l odd) or Im (l even) part, and
// the conjugate partner Y_{l,-m} = conj(Y_lm) (ylm index pairs 3/4, 6/7,
// 8/9 of get_ylm) gives Z components equal up to sign.  Those are merged:
// the partner's back-projection column is folded into the kept row with
// that sign and its energy weight doubles.  P = sum_atoms sum_l (2l+1).
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#include <cstdlib>
#include "sdft_ctx.h"

namespace sdft {

struct KbRow {
  int atom, type, l, ind;  // ind: 1-based ylm index of the kept channel
  int part;                // 0: Re Z, 1: Im Z
  int partner;             // partner ylm index or 0
  double psign;            // Z_partner = psign * Z_kept
  double vnorm;            // KB energy of the channel
};

__global__ void k_build_proj(int ncoef, int ngp, int Ppad, const int *__restrict__ kvec,
                             const double *__restrict__ frac, const int *__restrict__ row_start,
                             const int *__restrict__ row_count, const KbRow *__restrict__ rows,
                             const double *__restrict__ vtab, int lmax1,
                             const double *__restrict__ ylm,  // [10][ncoef][2]
                             const double *__restrict__ gz, double four_over_vol, double inv_vol,
                             double *__restrict__ Pj, double *__restrict__ Bk) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y;
  if (g >= ncoef) return;
  const int K1 = 2 * ngp;
  const int u0 = row_start[a], nu = row_count[a];
  if (g == ncoef - 1) {  // G = 0: l = 0 only
    const double y00 = 0.28209479177387814347;  // 1/sqrt(4 pi)
    for (int r = 0; r < nu; r++) {
      const KbRow R = rows[u0 + r];
      if (R.l != 0) continue;
      const int u = u0 + r;
      Pj[(size_t)u * K1 + g] = gz[R.type] * y00;
      Bk[(size_t)g * Ppad + u] = -2.0 * (y00 * gz[R.type] * R.vnorm * inv_vol);
    }
    return;
  }
  const double t = (double)kvec[3 * g] * frac[3 * a] + (double)kvec[3 * g + 1] * frac[3 * a + 1] +
                   (double)kvec[3 * g + 2] * frac[3 * a + 2];
  double sphi, cphi;
  sincospi(2.0 * t, &sphi, &cphi);
  for (int r = 0; r < nu; r++) {
    const KbRow R = rows[u0 + r];
    const int u = u0 + r;
    const double v = vtab[((size_t)R.type * lmax1 + R.l) * ncoef + g];
    const double hr = v * cphi, hi = v * sphi;
    const double yr = ylm[((size_t)R.ind * ncoef + g) * 2], yi = ylm[((size_t)R.ind * ncoef + g) * 2 + 1];
    double pr, pi;  // coefficients on Re c, Im c
    const bool lodd = (R.l & 1);
    if (!lodd) {
      if (R.part == 0) { pr = 2.0 * yr * hr; pi = -2.0 * yr * hi; }
      else { pr = 2.0 * yi * hr; pi = -2.0 * yi * hi; }
    } else {
      if (R.part == 0) { pr = -2.0 * yi * hi; pi = -2.0 * yi * hr; }
      else { pr = 2.0 * yr * hi; pi = 2.0 * yr * hr; }
    }
    Pj[(size_t)u * K1 + g] = pr;
    Pj[(size_t)u * K1 + ngp + g] = pi;
    // back projection
    const double s = v * four_over_vol;
    const double Hr = cphi * s, Hi = sphi * s;
    auto bk = [&](double yr_, double yi_, double &bre, double &bim) {
      const double vfr = Hr * yr_ - Hi * yi_;
      const double vfi = -(Hi * yr_ + Hr * yi_);
      if (R.part == 0) { bre = -R.vnorm * vfr; bim = -R.vnorm * vfi; }
      else { bre = R.vnorm * vfi; bim = -R.vnorm * vfr; }
    };
    double bre, bim;
    bk(yr, yi, bre, bim);
    if (R.partner) {
      const double ypr = ylm[((size_t)R.partner * ncoef + g) * 2], ypi = ylm[((size_t)R.partner * ncoef + g) * 2 + 1];
      double b2r, b2i;
      bk(ypr, ypi, b2r, b2i);
      bre += R.psign * b2r;
      bim += R.psign * b2i;
    }
    Bk[(size_t)g * Ppad + u] = bre;
    Bk[(size_t)(ngp + g) * Ppad + u] = bim;
  }
}

// Y_lm (l <= 2) of get_ylm (energy/cp/cp_energy_eext_nonloc.c:2350), values only.
static void ylm_host(double xk, double yk, double zk, double g, double *yr, double *yi) {
  const double fpi = 4.0 * M_PI;
  const double rt_fpi = 1.0 / std::sqrt(fpi), rt_thrfpi = std::sqrt(3.0 / fpi), rt_threpi = std::sqrt(1.50 / fpi);
  const double hrt_fivfpi = 0.50 * std::sqrt(5.0 / fpi), rt_fiftepi = std::sqrt(7.50 / fpi);
  double ctheta = zk / g;
  double stheta = std::sqrt(xk * xk + yk * yk) / g;
  double xyd = std::sqrt(xk * xk + yk * yk);
  double cphi, sphi;
  if (xyd == 0) { cphi = 1.0; sphi = 0.0; }
  else { cphi = xk / xyd; sphi = yk / xyd; }
  double c2phi = cphi * cphi - sphi * sphi, s2phi = 2.0 * cphi * sphi;
  for (int i = 0; i < 10; i++) yr[i] = yi[i] = 0.0;
  yr[1] = rt_fpi;
  double y10r = rt_thrfpi * ctheta, y11r = rt_threpi * stheta * cphi, y11i = rt_threpi * stheta * sphi;
  yr[2] = y10r;
  yr[3] = y11r; yi[3] = y11i;
  yr[4] = y11r; yi[4] = -y11i;
  double y20r = hrt_fivfpi * (3.0 * ctheta * ctheta - 1.0);
  double y21r = rt_fiftepi * stheta * ctheta * cphi, y21i = rt_fiftepi * stheta * ctheta * sphi;
  double y22r = 0.50 * rt_fiftepi * stheta * stheta * c2phi, y22i = 0.50 * rt_fiftepi * stheta * stheta * s2phi;
  yr[5] = y20r;
  yr[6] = y21r; yi[6] = y21i;
  yr[7] = y21r; yi[7] = -y21i;
  yr[8] = y22r; yi[8] = y22i;
  yr[9] = y22r; yi[9] = -y22i;
}

// get_vpsnow (energy/cp/cp_energy_eext.c:2139-2185) for one table.
static double spline_eval(const double *tab, int nsplin, double gmin, double dg, double g) {
  int iii = (int)((g - gmin) / dg) + 1;
  if (iii > nsplin) iii = nsplin;
  if (iii < 1) iii = 1;
  double h0 = (double)(iii - 1) * dg + gmin;
  double h = g - h0;
  const double *v0 = tab, *v1 = tab + nsplin, *v2 = tab + 2 * nsplin, *v3 = tab + 3 * nsplin;
  int i = iii - 1;
  return ((v3[i] * h + v2[i]) * h + v1[i]) * h + v0[i];
}

}  // namespace sdft

using namespace sdft;

#define CKT(call)                                                           \
  do {                                                                      \
    int r__ = (call);                                                       \
    if (r__) { rc = r__; goto done; }                                       \
  } while (0)
#define CKB(call)                                                           \
  do {                                                                      \
    cudaError_t e__ = (call);                                               \
    if (e__ != cudaSuccess) { rc = set_error(SDFT_ERR_CUDA, cudaGetErrorString(e__)); goto done; } \
  } while (0)

// Release the context's projector set (all KB arrays, P = 0).
static void kb_release(sdft_ctx *ctx) {
  double **old[] = {&ctx->d_pj, &ctx->d_bk, &ctx->d_w, &ctx->d_z, &ctx->d_zwork, &ctx->d_fnl, &ctx->d_gk, &ctx->d_zsave};
  for (double **p : old)
    if (*p) { dev_free(*p, ctx->st); *p = nullptr; }
  void *oldo[] = {ctx->d_pj_dig, ctx->d_bk_dig, ctx->d_c_dig, ctx->d_z_dig, ctx->d_pj_sc, ctx->d_bk_sc,
                  ctx->d_c_sc,   ctx->d_z_sc,   ctx->d_rowmax, ctx->d_oz_part};
  for (void *p : oldo) dev_free(p, ctx->st);
  ctx->d_pj_dig = ctx->d_bk_dig = ctx->d_c_dig = ctx->d_z_dig = nullptr;
  ctx->d_pj_sc = ctx->d_bk_sc = ctx->d_c_sc = ctx->d_z_sc = nullptr;
  ctx->d_rowmax = nullptr;
  ctx->d_oz_part = nullptr;
  dev_free(ctx->d_kb_rs, ctx->st);
  dev_free(ctx->d_kb_rc, ctx->st);
  dev_free(ctx->d_rowmax3, ctx->st);
  ctx->d_kb_rs = ctx->d_kb_rc = nullptr;
  ctx->d_rowmax3 = nullptr;
  ctx->kb_natm = 0;
  ctx->P = 0;
  ctx->oz = false;
  ctx->dev_bytes -= ctx->kb_bytes;
  ctx->kb_bytes = 0;
}

static int kb_build(sdft_ctx *ctx, const sdft_kb_desc *kb) {
  if (!kb || kb->natm == 0) return SDFT_OK;
  // whatever this build leaves allocated counts as KB bytes, on every return path
  struct KbBytes {
    sdft_ctx *c;
    long long before;
    ~KbBytes() { c->kb_bytes = c->dev_bytes - before; }
  } kb_guard{ctx, ctx->dev_bytes};
  if (!kb->pos || !kb->type || !kb->lmax_type || !kb->vps || !kb->vpsnorm || !kb->gzvps0 || kb->ntype < 1 ||
      kb->nsplin_g < 1 || kb->dg_spl <= 0.0)
    return set_error(SDFT_ERR_ARG, "set_kb: incomplete projector description");
  if (kb->lmax < 0 || kb->lmax > 2) return set_error(SDFT_ERR_UNSUPPORTED, "set_kb: l channels 0..2 only");
  const int lmax1 = kb->lmax + 1;
  const int ncoef = ctx->ncoef, ngp = ctx->ngp;
  double hi[9];
  invert_cell(ctx->hmat, hi);
  // rows
  std::vector<KbRow> rows;
  std::vector<int> rstart(kb->natm), rcount(kb->natm);
  for (int a = 0; a < kb->natm; a++) {
    const int t = kb->type[a];
    if (t < 0 || t >= kb->ntype) return set_error(SDFT_ERR_ARG, "set_kb: atom type out of range");
    const int lm = kb->lmax_type[t];
    if (lm > kb->lmax) return set_error(SDFT_ERR_ARG, "set_kb: lmax_type > lmax");
    rstart[a] = (int)rows.size();
    for (int l = 0; l <= lm; l++) {
      const double vn = kb->vpsnorm[t * lmax1 + l];
      auto add = [&](int ind, int part, int partner, double sgn) {
        rows.push_back(KbRow{a, t, l, ind, part, partner, sgn, vn});
      };
      if (l == 0) add(1, 0, 0, 0.0);
      if (l == 1) { add(2, 1, 0, 0.0); add(3, 0, 4, -1.0); add(3, 1, 4, +1.0); }
      if (l == 2) { add(5, 0, 0, 0.0); add(6, 0, 7, +1.0); add(6, 1, 7, -1.0); add(8, 0, 9, +1.0); add(8, 1, 9, -1.0); }
    }
    rcount[a] = (int)rows.size() - rstart[a];
  }
  const int P = (int)rows.size();
  if (P == 0) return SDFT_OK;
  const int Ppad = (int)((P + 127) / 128 * 128);
  const int K1 = 2 * ngp;
  const int Mpad2 = (K1 + 127) / 128 * 128;
  // per-G tables
  std::vector<int> kv(3 * ncoef);
  std::vector<double> vtab((size_t)kb->ntype * lmax1 * ncoef, 0.0), ylm((size_t)10 * ncoef * 2, 0.0);
  std::vector<double> gk((size_t)3 * ngp, 0.0);
  const double tpi = 2.0 * M_PI;
  for (int g = 0; g < ncoef; g++) {
    kv[3 * g] = ctx->ka[g]; kv[3 * g + 1] = ctx->kb[g]; kv[3 * g + 2] = ctx->kc[g];
    if (g == ncoef - 1) continue;
    const double aka = ctx->ka[g], akb = ctx->kb[g], akc = ctx->kc[g];
    const double xk = (aka * hi[0] + akb * hi[1] + akc * hi[2]) * tpi;
    const double yk = (aka * hi[3] + akb * hi[4] + akc * hi[5]) * tpi;
    const double zk = (aka * hi[6] + akb * hi[7] + akc * hi[8]) * tpi;
    const double gg = std::sqrt(xk * xk + yk * yk + zk * zk);
    gk[g] = xk; gk[(size_t)ngp + g] = yk; gk[(size_t)2 * ngp + g] = zk;
    double yr[10], yi[10];
    ylm_host(xk, yk, zk, gg, yr, yi);
    for (int i = 0; i < 10; i++) {
      ylm[((size_t)i * ncoef + g) * 2] = yr[i];
      ylm[((size_t)i * ncoef + g) * 2 + 1] = yi[i];
    }
    for (int t = 0; t < kb->ntype; t++)
      for (int l = 0; l <= kb->lmax_type[t]; l++)
        vtab[((size_t)t * lmax1 + l) * ncoef + g] =
            spline_eval(kb->vps + ((size_t)t * lmax1 + l) * 4 * kb->nsplin_g, kb->nsplin_g, kb->gmin_spl,
                        kb->dg_spl, gg);
  }
  // fractional coordinates wrapped as controlEwdNonlocFilter (box centre 0)
  std::vector<double> frac(3 * kb->natm);
  for (int a = 0; a < kb->natm; a++) {
    const double x = kb->pos[3 * a], y = kb->pos[3 * a + 1], z = kb->pos[3 * a + 2];
    double s[3] = {x * hi[0] + y * hi[3] + z * hi[6], x * hi[1] + y * hi[4] + z * hi[7],
                   x * hi[2] + y * hi[5] + z * hi[8]};
    for (int d = 0; d < 3; d++) frac[3 * a + d] = s[d] - std::nearbyint(s[d]);
  }
  std::vector<double> w(Ppad, 0.0);
  for (int u = 0; u < P; u++) w[u] = rows[u].vnorm / ctx->vol * (rows[u].partner ? 2.0 : 1.0);

  int rc = SDFT_OK;
  int *d_kv = nullptr, *d_rs = nullptr, *d_rcnt = nullptr;
  double *d_frac = nullptr, *d_vtab = nullptr, *d_ylm = nullptr, *d_gz = nullptr;
  KbRow *d_rows = nullptr;
  {
    int r;
    if ((r = dmalloc(ctx, (void **)&ctx->d_pj, (size_t)Ppad * K1 * sizeof(double)))) return r;
    if ((r = dmalloc(ctx, (void **)&ctx->d_bk, (size_t)Mpad2 * Ppad * sizeof(double)))) return r;
    if ((r = dmalloc(ctx, (void **)&ctx->d_w, (size_t)Ppad * sizeof(double)))) return r;
    if ((r = dmalloc(ctx, (void **)&ctx->d_z, (size_t)ctx->s_pad * Ppad * sizeof(double)))) return r;
    ctx->zwork_elems = (size_t)16 * ctx->s_pad * Ppad;
    if ((r = dmalloc(ctx, (void **)&ctx->d_zwork, ctx->zwork_elems * sizeof(double)))) return r;
    if ((r = dmalloc(ctx, (void **)&ctx->d_fnl, ctx->vec_elems * sizeof(double)))) return r;
    if ((r = dmalloc(ctx, (void **)&ctx->d_gk, gk.size() * sizeof(double)))) return r;
    if ((r = dmalloc(ctx, (void **)&ctx->d_kb_rs, rstart.size() * sizeof(int)))) return r;
    if ((r = dmalloc(ctx, (void **)&ctx->d_kb_rc, rcount.size() * sizeof(int)))) return r;
  }
  CKB(cudaMemcpyAsync(ctx->d_gk, gk.data(), gk.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(ctx->d_kb_rs, rstart.data(), rstart.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(ctx->d_kb_rc, rcount.data(), rcount.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemsetAsync(ctx->d_pj, 0, (size_t)Ppad * K1 * sizeof(double), ctx->st));
  CKB(cudaMemsetAsync(ctx->d_bk, 0, (size_t)Mpad2 * Ppad * sizeof(double), ctx->st));
  CKB(cudaMemsetAsync(ctx->d_z, 0, (size_t)ctx->s_pad * Ppad * sizeof(double), ctx->st));
  CKB(cudaMemsetAsync(ctx->d_fnl, 0, ctx->vec_elems * sizeof(double), ctx->st));
  CKB(cudaMemcpyAsync(ctx->d_w, w.data(), Ppad * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  CKT(dev_alloc(ctx->device, ctx->st, (void **)&d_kv, kv.size() * sizeof(int)));
  CKT(dev_alloc(ctx->device, ctx->st, (void **)&d_rs, rstart.size() * sizeof(int)));
  CKT(dev_alloc(ctx->device, ctx->st, (void **)&d_rcnt, rcount.size() * sizeof(int)));
  CKT(dev_alloc(ctx->device, ctx->st, (void **)&d_frac, frac.size() * sizeof(double)));
  CKT(dev_alloc(ctx->device, ctx->st, (void **)&d_vtab, vtab.size() * sizeof(double)));
  CKT(dev_alloc(ctx->device, ctx->st, (void **)&d_ylm, ylm.size() * sizeof(double)));
  CKT(dev_alloc(ctx->device, ctx->st, (void **)&d_gz, kb->ntype * sizeof(double)));
  CKT(dev_alloc(ctx->device, ctx->st, (void **)&d_rows, rows.size() * sizeof(KbRow)));
  CKB(cudaMemcpyAsync(d_kv, kv.data(), kv.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(d_rs, rstart.data(), rstart.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(d_rcnt, rcount.data(), rcount.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(d_frac, frac.data(), frac.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(d_vtab, vtab.data(), vtab.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(d_ylm, ylm.data(), ylm.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(d_gz, kb->gzvps0, kb->ntype * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  CKB(cudaMemcpyAsync(d_rows, rows.data(), rows.size() * sizeof(KbRow), cudaMemcpyHostToDevice, ctx->st));
  {
    dim3 grid((ncoef + 127) / 128, kb->natm);
    k_build_proj<<<grid, 128, 0, ctx->st>>>(ncoef, ngp, Ppad, d_kv, d_frac, d_rs, d_rcnt, d_rows, d_vtab, lmax1,
                                            d_ylm, d_gz, 4.0 / ctx->vol, 1.0 / ctx->vol, ctx->d_pj, ctx->d_bk);
    ctx->launches++;
    CKB(cudaGetLastError());
    CKB(cudaStreamSynchronize(ctx->st));
  }
  ctx->P = P;
  ctx->kb_natm = kb->natm;
  ctx->Ppad = Ppad;
  ctx->Mpad2 = Mpad2;
  if ((ctx->prec == SDFT_PREC_MIXED || ctx->prec == SDFT_PREC_MIXED_FAST) && gemm_oz_available()) {
    // digit form of the projector matrices for the INT8 tensor-core GEMMs
    const int S = (ctx->max_states + 127) / 128 * 128;
    const int Kp = (K1 + 63) / 64 * 64;
    ctx->s_oz = S;
    ctx->kp_oz = Kp;
    int r;
    // the projection (FP64 partials, FP64 Z) uses the 28-bit digits; the back
    // projection (FP32 result) the 24-bit ones in SDFT_PREC_MIXED_FAST (K =
    // Ppad; that format accumulates K ranges up to 16384 exactly)
    const int f2 = (ctx->prec == SDFT_PREC_MIXED_FAST && Ppad <= 16384) ? OZ_8x3 : OZ_7x4;
    const size_t pjd = (size_t)kOzSlices * Ppad * Kp, bkd = (size_t)oz_slices(f2) * Mpad2 * Ppad;
    const size_t cd = (size_t)kOzSlices * S * Kp, zd = (size_t)oz_slices(f2) * S * Ppad;
    const int maxrows = std::max(std::max(Ppad, Mpad2), S);
    ctx->oz_part_elems = (size_t)32 * S * Ppad;
    if ((r = dmalloc(ctx, (void **)&ctx->d_pj_dig, pjd)) || (r = dmalloc(ctx, (void **)&ctx->d_bk_dig, bkd)) ||
        (r = dmalloc(ctx, (void **)&ctx->d_c_dig, cd)) || (r = dmalloc(ctx, (void **)&ctx->d_z_dig, zd)) ||
        (r = dmalloc(ctx, (void **)&ctx->d_pj_sc, Ppad * sizeof(double))) ||
        (r = dmalloc(ctx, (void **)&ctx->d_bk_sc, Mpad2 * sizeof(double))) ||
        (r = dmalloc(ctx, (void **)&ctx->d_c_sc, S * sizeof(double))) ||
        (r = dmalloc(ctx, (void **)&ctx->d_z_sc, S * sizeof(double))) ||
        (r = dmalloc(ctx, (void **)&ctx->d_rowmax, maxrows * sizeof(unsigned long long))) ||
        (r = dmalloc(ctx, (void **)&ctx->d_oz_part, ctx->oz_part_elems * sizeof(double)))) {
      rc = r;
      goto done;
    }
    CKB(cudaMemsetAsync(ctx->d_c_dig, 0, cd, ctx->st));
    CKB(cudaMemsetAsync(ctx->d_z_dig, 0, zd, ctx->st));
    CKB(cudaMemsetAsync(ctx->d_c_sc, 0, S * sizeof(double), ctx->st));
    CKB(cudaMemsetAsync(ctx->d_z_sc, 0, S * sizeof(double), ctx->st));
    launch_oz_slice_rows(ctx->d_pj, K1, Ppad, K1, ctx->d_rowmax, ctx->d_pj_dig, Kp, (size_t)Ppad * Kp, ctx->d_pj_sc,
                         ctx->st);
    launch_oz_slice_rows(ctx->d_bk, Ppad, Mpad2, Ppad, ctx->d_rowmax, ctx->d_bk_dig, Ppad, (size_t)Mpad2 * Ppad,
                         ctx->d_bk_sc, ctx->st, f2);
    ctx->launches += 4;
    CKB(cudaGetLastError());
    CKB(cudaStreamSynchronize(ctx->st));
    OzGemm &g1 = ctx->om1, &g2 = ctx->om2;
    if ((r = make_tmap_oz(&g1.tA, ctx->d_pj_dig, Ppad, Kp)) || (r = make_tmap_oz(&g1.tB, ctx->d_c_dig, S, Kp)) ||
        (r = make_tmap_oz(&g2.tA, ctx->d_bk_dig, Mpad2, Ppad, f2)) ||
        (r = make_tmap_oz(&g2.tB, ctx->d_z_dig, S, Ppad, f2)) ||
        (r = make_tmap_oz(&ctx->om1_tb64, ctx->d_c_dig, S, Kp, OZ_7x4, 64)) ||
        (r = make_tmap_oz(&ctx->om2_tb64, ctx->d_z_dig, S, Ppad, f2, 64))) {
      rc = r;
      goto done;
    }
    g1.M = Ppad; g1.K = Kp; g1.ldo = Ppad; g1.Mst = P; g1.sa = ctx->d_pj_sc; g1.sb = ctx->d_c_sc;
    g2.M = Mpad2; g2.K = Ppad; g2.ldo = K1; g2.Mst = K1; g2.sa = ctx->d_bk_sc; g2.sb = ctx->d_z_sc;
    g1.fmt = OZ_7x4;
    g2.fmt = f2;
    // the FP64 projector copies are not used by the mixed path
    dev_free(ctx->d_pj, ctx->st); ctx->d_pj = nullptr;
    dev_free(ctx->d_bk, ctx->st); ctx->d_bk = nullptr;
    ctx->dev_bytes -= (long long)((size_t)Ppad * K1 + (size_t)Mpad2 * Ppad) * 8;
    ctx->oz = true;
    ctx->rowmax_zero_n = 0;  // the projector slicing above left row maxima behind
  }
done:
  for (void *p : {(void *)d_kv, (void *)d_rs, (void *)d_rcnt, (void *)d_frac, (void *)d_vtab, (void *)d_ylm,
                  (void *)d_gz, (void *)d_rows})
    dev_free(p, ctx->st);
  cudaStreamSynchronize(ctx->st);
  return rc;
}

// A previous set is released first; a build that fails part way (an
// allocation refused, say) is released too, so the context is left without
// projectors -- never with a projector count whose arrays are missing.
int sdft_build_kb_device(sdft_ctx *ctx, const sdft_kb_desc *kb) {
  kb_release(ctx);
  const int rc = kb_build(ctx, kb);
  if (rc) kb_release(ctx);
  return rc;
}
