/*
 * sdft_piny_adapter.c -- the PINY-side drop-in: the reference's own routine
 * signatures (stodft/proto_stodft_local.h) implemented on the sdft C ABI
 * (include/sdft_b200.h), so that a PINY build links these instead of
 *
 *   filterChebyPolyHerm    stodft/filter.c:318
 *   filterNewtonPolyHerm   stodft/filter.c:33
 *   normHCheby             stodft/normh.c:182
 *   normHNewtonHerm        stodft/normh.c:35
 *   calcChebyMoments       stodft/calc-chempot-chebyshev.c:596
 *   calcCoefForceWrapSCF   stodft/reduced-energy/energy-wrapper-scf.c:1066
 *   rhoCalcRealStoHybrid   stodft/density.c:43
 *   genNoiseOrbitalReal    stodft/gen-noise.c:162  (unless SDFT_PINY_ADAPTER_NO_NOISE;
 *                          its body is also sdft_piny_noise)
 *
 * and leaves every caller unchanged.  The file is empty unless compiled with
 * -DSDFT_PINY_ADAPTER and a PINY tree on the include path:
 *
 *   cc -c -DSDFT_PINY_ADAPTER -I<piny>/include/pentium_nopar -I<piny>/stodft \
 *      -I<this repo>/include sdft_piny_adapter.c
 *
 * and linked with lib/libsdft_b200.so in place of the object files that
 * define the routines above.  It reads only PINY struct fields; no PINY code
 * is repeated here.
 *
 * One device context per FFT package (cp->cp_sclr_fft_pkg3d_sm, one per
 * system), created on the first call that passes the CP: grid and G list
 * from the package and cpewald->k*str_sm, cell from general_data->cell,
 * kinetic cap from cpewald->gCutoffKe (when eCutoffKe >= 0), V_KS from
 * cpscr_rho.v_ks_up, Kleinman-Bylander tables from cp->pseudo and the atom
 * maps.  Later calls upload V_KS again only when it changed and rebuild the
 * projectors only when an atom moved.  The context is made for this rank's
 * share of the orbitals (nstate_up / np_states, or more when a call brings
 * more; the spectral range runs with nstate_up_proc = 1) and grows when a
 * call that carries the CLASS brings more than it holds.
 *
 * Environment: SDFT_PINY_PRECISION = fp64 | mixed (default) | mixed_fast;
 * SDFT_PINY_DEVICE = CUDA device ordinal (default 0); SDFT_PINY_MAX_STATES =
 * the least number of orbitals a context is made for.
 *
 * Supported as in the product: spin-unpolarised (cp_lsda = 0), one radial KB
 * projector per channel (n_rad_max = 1), l <= 2, the CP box equal to the cell
 * (cp_dual_grid_opt = 0), no entropy filter (smearOpt = 0 or filterDiagFlag).
 * Anything else stops with PINY's error banner, as PINY does.
 *
 * Differences from the replaced routines, none read by their callers:
 * filterChebyPolyHerm / filterNewtonPolyHerm leave cre_up / cim_up holding
 * the input orbitals (the reference leaves the last polynomial vector
 * there); normHCheby / normHNewtonHerm do not add the KB energy of their
 * H c to stat_avg->cp_enl; genNoiseOrbitalReal does not leave the per-rank
 * seeds in stodftInfo->randSeedTot.
 */
#ifdef SDFT_PINY_ADAPTER

#include "standard_include.h"
#include "../typ_defs/typedefs_gen.h"
#include "../typ_defs/typedefs_class.h"
#include "../typ_defs/typedefs_bnd.h"
#include "../typ_defs/typedefs_cp.h"
#include "proto_stodft_local.h"
#include "sdft_b200.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void *cmalloc(size_t len); /* friend_lib/cmalloc.c:10 */

#define AD_MAX_SYSTEMS 16

typedef struct {
  const PARA_FFT_PKG3D *key; /* &cp->cp_sclr_fft_pkg3d_sm of the system   */
  sdft_ctx *ctx;
  int max_states, N, ncoef;
  double *vks;               /* host copy of the V_KS last uploaded       */
  int nkb;
  double *kbpos;             /* host copy of the KB atom positions used   */
} AdSys;

static AdSys g_sys[AD_MAX_SYSTEMS];

static void ad_die(const char *where, const char *msg) {
  printf("@@@@@@@@@@@@@@@@@@@@_ERROR_@@@@@@@@@@@@@@@@@@@@\n");
  printf("sdft adapter, %s: %s\n", where, msg ? msg : "");
  printf("@@@@@@@@@@@@@@@@@@@@_ERROR_@@@@@@@@@@@@@@@@@@@@\n");
  fflush(stdout);
  exit(1);
}

static void ad_ck(int rc, const char *where) {
  if (rc != SDFT_OK) ad_die(where, sdft_last_error());
}

static int ad_precision(void) {
  const char *p = getenv("SDFT_PINY_PRECISION");
  if (!p || !strcmp(p, "mixed")) return SDFT_PREC_MIXED;
  if (!strcmp(p, "fp64")) return SDFT_PREC_FP64;
  if (!strcmp(p, "mixed_fast")) return SDFT_PREC_MIXED_FAST;
  ad_die("SDFT_PINY_PRECISION", "expected fp64, mixed or mixed_fast");
  return 0;
}

static AdSys *ad_find(const PARA_FFT_PKG3D *key) {
  for (int i = 0; i < AD_MAX_SYSTEMS; i++)
    if (g_sys[i].key == key) return &g_sys[i];
  return NULL;
}

/* Positions of the nonlocal atoms as control_ewd_non_loc places them
 * (energy/cp/cp_energy_eext_nonloc.c:143-172): x - cp_box_center +
 * cp_box_center_rel; the context wraps them into the cell. */
static void ad_kb_positions(CP *cp, CELL *cell, CLATOMS_POS *ap, double *pos, int nkb) {
  const int *ip_nl = cp->pseudo.ip_nl;
  const double *c = cell->cp_box_center, *cr = cell->cp_box_center_rel;
  for (int k = 1; k <= nkb; k++) {
    const int ia = ip_nl[k];
    pos[3 * (k - 1)] = ap->x[ia] - c[1] + cr[1];
    pos[3 * (k - 1) + 1] = ap->y[ia] - c[2] + cr[2];
    pos[3 * (k - 1) + 2] = ap->z[ia] - c[3] + cr[3];
  }
}

/* The Kleinman-Bylander description of cp->pseudo in the context's form.
 * Nonlocal atom k (1..np_nonloc_cp_box_kb): spline block
 * imap_atm_typ_nl[iatm_atm_typ_nl_rev[k]] (control_nlmat's index_atm,
 * cp_energy_eext_nonloc.c:492-495), norm and G = 0 value of full type
 * iatm_atm_typ_nl[k] (get_vpsnorm :2311, control_ewd_non_loc :211), channel
 * l present when k is on the l list (ip_nl_rev[ipart + l natm_tot]).  Each
 * distinct (block, type, channel set) becomes one context type; a channel
 * absent below the type's top l gets a zero norm, which removes it. */
static void ad_set_kb(AdSys *s, CP *cp, CLASS *cl, CELL *cell, CLATOMS_POS *ap) {
  PSEUDO *ps = &cp->pseudo;
  ATOMMAPS *am = &cl->atommaps;
  const int nkb = ps->np_nonloc_cp_box_kb, natm_tot = cl->clatoms_info.natm_tot;
  free(s->kbpos);
  s->kbpos = NULL;
  s->nkb = 0;
  int lmax = -1;
  for (int l = 0; l <= ps->n_ang_max_kb; l++)
    if (ps->np_nl[l + 1] > 0) lmax = l;
  if (nkb <= 0 || lmax < 0) {
    ad_ck(sdft_ctx_set_kb(s->ctx, NULL), "sdft_ctx_set_kb");
    return;
  }
  if (ps->n_rad_max != 1) ad_die("Kleinman-Bylander", "one radial projector per channel only (n_rad_max = 1)");
  if (lmax > 2) ad_die("Kleinman-Bylander", "channels l <= 2 only");
  const int nsp = ps->nsplin_g, nang1 = ps->n_ang_max + 1;
  int *blk = calloc(nkb, sizeof(int)), *typ = calloc(nkb, sizeof(int)), *mask = calloc(nkb, sizeof(int));
  int *dtype = calloc(nkb, sizeof(int)), *ublk = calloc(nkb, sizeof(int)), *utyp = calloc(nkb, sizeof(int));
  int *umask = calloc(nkb, sizeof(int));
  for (int l = 0; l <= lmax; l++)
    for (int ipart = ps->np_nl_rad_str[l + 1][1]; ipart <= ps->np_nl[l + 1]; ipart++) {
      const int k = ps->ip_nl_rev[ipart + l * natm_tot];
      if (k >= 1 && k <= nkb) mask[k - 1] |= 1 << l;
    }
  int ntype = 0;
  for (int k = 1; k <= nkb; k++) {
    blk[k - 1] = am->imap_atm_typ_nl[am->iatm_atm_typ_nl_rev[k]];
    typ[k - 1] = am->iatm_atm_typ_nl[k];
    int t = 0;
    while (t < ntype && !(ublk[t] == blk[k - 1] && utyp[t] == typ[k - 1] && umask[t] == mask[k - 1])) t++;
    if (t == ntype) {
      ublk[t] = blk[k - 1];
      utyp[t] = typ[k - 1];
      umask[t] = mask[k - 1];
      ntype++;
    }
    dtype[k - 1] = t;
  }
  const int lmax1 = lmax + 1;
  int *lmax_type = calloc(ntype, sizeof(int));
  double *vps = calloc((size_t)ntype * lmax1 * 4 * nsp, sizeof(double));
  double *vpsnorm = calloc((size_t)ntype * lmax1, sizeof(double));
  double *gz = calloc(ntype, sizeof(double));
  const double *tab[4] = {ps->vps0, ps->vps1, ps->vps2, ps->vps3};
  for (int t = 0; t < ntype; t++) {
    lmax_type[t] = -1;
    for (int l = 0; l <= lmax; l++) {
      if (!(umask[t] & (1 << l))) continue;
      lmax_type[t] = l;
      const long off = (long)(ublk[t] - 1) * nsp * nang1 + (long)l * nsp; /* n_rad_max = 1 */
      for (int c = 0; c < 4; c++)
        for (int i = 0; i < nsp; i++) vps[(((size_t)t * lmax1 + l) * 4 + c) * nsp + i] = tab[c][off + 1 + i];
      vpsnorm[t * lmax1 + l] = ps->vpsnorm[(utyp[t] - 1) * nang1 + l + 1];
    }
    if (umask[t] & 1) gz[t] = ps->gzvps0[utyp[t]];
  }
  s->kbpos = malloc(sizeof(double) * 3 * nkb);
  s->nkb = nkb;
  ad_kb_positions(cp, cell, ap, s->kbpos, nkb);
  sdft_kb_desc d;
  d.natm = nkb;
  d.pos = s->kbpos;
  d.type = dtype;
  d.ntype = ntype;
  d.lmax = lmax;
  d.lmax_type = lmax_type;
  d.nsplin_g = nsp;
  d.gmin_spl = ps->gmin_spl;
  d.dg_spl = ps->dg_spl;
  d.vps = vps;
  d.vpsnorm = vpsnorm;
  d.gzvps0 = gz;
  ad_ck(sdft_ctx_set_kb(s->ctx, &d), "sdft_ctx_set_kb");
  free(blk); free(typ); free(mask); free(dtype); free(ublk); free(utyp); free(umask);
  free(lmax_type); free(vps); free(vpsnorm); free(gz);
}

static void ad_check_options(CP *cp, CELL *cell, const char *where) {
  if (cp->cpopts.cp_lsda != 0) ad_die(where, "spin-polarised runs (cp_lsda = 1) are not supported");
  if (cp->cpopts.cp_dual_grid_opt != 0) ad_die(where, "dual grids (cp_dual_grid_opt > 0) are not supported");
  for (int i = 1; i <= 9; i++)
    if (cell->hmat_cp[i] != cell->hmat[i]) ad_die(where, "the CP box must be the whole cell");
}

/* The context of this CP's system, created or brought up to date. */
static AdSys *ad_attach(CP *cp, CLASS *cl, GENERAL_DATA *gd, CLATOMS_POS *ap, int nstate, const char *where) {
  CELL *cell = &gd->cell;
  const PARA_FFT_PKG3D *key = &cp->cp_sclr_fft_pkg3d_sm;
  const int n1 = key->nkf1, n2 = key->nkf2, n3 = key->nkf3, N = n1 * n2 * n3;
  const int ncoef = cp->cpcoeffs_info.ncoef;
  ad_check_options(cp, cell, where);
  AdSys *s = ad_find(key);
  if (s && s->ctx && s->max_states < nstate) { /* grow */
    sdft_ctx_destroy(s->ctx);
    s->ctx = NULL;
  }
  if (!s) {
    s = ad_find(NULL);
    if (!s) ad_die(where, "too many systems");
    memset(s, 0, sizeof *s);
    s->key = key;
  }
  if (!s->ctx) {
    CPEWALD *ew = &cp->cpewald;
    int *ka = malloc(sizeof(int) * ncoef), *kb = malloc(sizeof(int) * ncoef), *kc = malloc(sizeof(int) * ncoef);
    for (int i = 0; i < ncoef; i++) {
      ka[i] = ew->kastr_sm[i + 1];
      kb[i] = ew->kbstr_sm[i + 1];
      kc[i] = ew->kcstr_sm[i + 1];
    }
    ka[ncoef - 1] = kb[ncoef - 1] = kc[ncoef - 1] = 0; /* G = 0 last */
    const char *dv = getenv("SDFT_PINY_DEVICE"), *ms = getenv("SDFT_PINY_MAX_STATES");
    const int np = cp->communicate.np_states > 0 ? cp->communicate.np_states : 1;
    int want = nstate > s->max_states ? nstate : s->max_states;
    const int share = (cp->cpcoeffs_info.nstate_up + np - 1) / np;
    if (share > want) want = share;
    if (ms && atoi(ms) > want) want = atoi(ms);
    ad_ck(sdft_ctx_create(n1, n2, n3, ncoef, ka, kb, kc, &cell->hmat_cp[1], ad_precision(), want, dv ? atoi(dv) : 0,
                          &s->ctx),
          "sdft_ctx_create");
    free(ka); free(kb); free(kc);
    s->max_states = want;
    s->N = N;
    s->ncoef = ncoef;
    if (ew->eCutoffKe >= 0.0) ad_ck(sdft_ctx_set_kinetic_cap(s->ctx, ew->gCutoffKe), "sdft_ctx_set_kinetic_cap");
    free(s->vks);
    s->vks = malloc(sizeof(double) * N);
    memcpy(s->vks, &cp->cpscr.cpscr_rho.v_ks_up[1], sizeof(double) * N);
    ad_ck(sdft_ctx_set_vks(s->ctx, s->vks), "sdft_ctx_set_vks");
    ad_set_kb(s, cp, cl, cell, ap);
    return s;
  }
  if (memcmp(s->vks, &cp->cpscr.cpscr_rho.v_ks_up[1], sizeof(double) * N)) {
    memcpy(s->vks, &cp->cpscr.cpscr_rho.v_ks_up[1], sizeof(double) * N);
    ad_ck(sdft_ctx_set_vks(s->ctx, s->vks), "sdft_ctx_set_vks");
  }
  if (s->nkb != cp->pseudo.np_nonloc_cp_box_kb) {
    ad_set_kb(s, cp, cl, cell, ap);
  } else if (s->nkb > 0) {
    double *p = malloc(sizeof(double) * 3 * s->nkb);
    ad_kb_positions(cp, cell, ap, p, s->nkb);
    if (memcmp(p, s->kbpos, sizeof(double) * 3 * s->nkb)) ad_set_kb(s, cp, cl, cell, ap);
    free(p);
  }
  return s;
}

static void ad_no_entropy(STODFTINFO *si, const char *where) {
  if (si->smearOpt > 0 && si->filterDiagFlag == 0) ad_die(where, "the entropy filter (smearOpt > 0) is not supported");
}

/* Releases every system's device context and host copies (for a caller's
 * shutdown path; the next adapted call creates the context again). */
void sdft_piny_adapter_finalize(void) {
  for (int i = 0; i < AD_MAX_SYSTEMS; i++) {
    AdSys *s = &g_sys[i];
    if (s->ctx) sdft_ctx_destroy(s->ctx);
    free(s->vks);
    free(s->kbpos);
    memset(s, 0, sizeof *s);
  }
}

/* ---- the replaced routines ---------------------------------------------- */

void calcCoefForceWrapSCF(CLASS *class, GENERAL_DATA *general_data, CP *cp, CPCOEFFS_POS *cpcoeffs_pos,
                          CLATOMS_POS *clatoms_pos) {
  const int ns = cp->cpcoeffs_info.nstate_up_proc;
  AdSys *s = ad_attach(cp, class, general_data, clatoms_pos, ns, "calcCoefForceWrapSCF");
  /* the V_ext restore of energy-wrapper-scf.c:1148-1151 */
  CPSCR_LOC *loc = &cp->cpscr.cpscr_loc;
  for (int i = 1; i <= cp->cp_para_fft_pkg3d_lg.ncoef_proc; i++) {
    loc->vextr[i] = loc->vextr_loc[i];
    loc->vexti[i] = loc->vexti_loc[i];
  }
  double enl = 0.0;
  ad_ck(sdft_hpsi(s->ctx, ns, &cpcoeffs_pos->cre_up[1], &cpcoeffs_pos->cim_up[1], &cpcoeffs_pos->fcre_up[1],
                  &cpcoeffs_pos->fcim_up[1], &enl),
        "calcCoefForceWrapSCF");
  general_data->stat_avg.cp_enl += enl;
}

void normHCheby(CP *cp, CLASS *class, GENERAL_DATA *general_data, CPCOEFFS_POS *cpcoeffs_pos,
                CLATOMS_POS *clatoms_pos, int iPoly, int cpyFlag) {
  STODFTINFO *si = cp->stodftInfo;
  STODFTCOEFPOS *sp = cp->stodftCoefPos;
  const int ns = cp->cpcoeffs_info.nstate_up_proc;
  AdSys *s = ad_attach(cp, class, general_data, clatoms_pos, ns, "normHCheby");
  ad_ck(sdft_normh_cheby(s->ctx, ns, iPoly, cpyFlag, si->chebyshevInfo->scale, si->energyMean,
                         &cpcoeffs_pos->cre_up[1], &cpcoeffs_pos->cim_up[1], &sp->wfUpRe1[1], &sp->wfUpIm1[1],
                         &cpcoeffs_pos->fcre_up[1], &cpcoeffs_pos->fcim_up[1]),
        "normHCheby");
}

void normHNewtonHerm(CP *cp, CLASS *class, GENERAL_DATA *general_data, CPCOEFFS_POS *cpcoeffs_pos,
                     CLATOMS_POS *clatoms_pos, double zn) {
  STODFTINFO *si = cp->stodftInfo;
  const int ns = cp->cpcoeffs_info.nstate_up_proc;
  AdSys *s = ad_attach(cp, class, general_data, clatoms_pos, ns, "normHNewtonHerm");
  ad_ck(sdft_normh_newton(s->ctx, ns, si->newtonInfo->scale, si->energyMean, zn, &cpcoeffs_pos->cre_up[1],
                          &cpcoeffs_pos->cim_up[1], &cpcoeffs_pos->fcre_up[1], &cpcoeffs_pos->fcim_up[1]),
        "normHNewtonHerm");
}

void filterChebyPolyHerm(CP *cp, CLASS *class, GENERAL_DATA *general_data, int ip_now) {
  STODFTINFO *si = cp->stodftInfo;
  STODFTCOEFPOS *sp = cp->stodftCoefPos;
  CPCOEFFS_POS *pos = &cp->cpcoeffs_pos[ip_now];
  const int ns = cp->cpcoeffs_info.nstate_up_proc, L = si->polynormLength, nmu = si->numChemPot;
  ad_no_entropy(si, "filterChebyPolyHerm");
  AdSys *s = ad_attach(cp, class, general_data, &class->clatoms_pos[ip_now], ns, "filterChebyPolyHerm");
  double **re = malloc(sizeof(double *) * nmu), **im = malloc(sizeof(double *) * nmu);
  for (int imu = 0; imu < nmu; imu++) {
    re[imu] = &sp->stoWfUpRe[imu][1];
    im[imu] = &sp->stoWfUpIm[imu][1];
  }
  double *mom = NULL;
  if (si->storeChebyMomentsFlag == 1) { /* a fresh array, as filter.c:460 */
    sp->chebyMomentsUp = (double *)cmalloc((L + 1) * sizeof(double));
    mom = sp->chebyMomentsUp;
  }
  /* normHCheby inside the reference's loop takes chebyshevInfo->scale */
  ad_ck(sdft_filter_cheby(s->ctx, ns, &pos->cre_up[1], &pos->cim_up[1], L, nmu, sp->expanCoeff,
                          si->chebyshevInfo->scale, si->energyMean, re, im, mom),
        "filterChebyPolyHerm");
  free(re);
  free(im);
}

void filterNewtonPolyHerm(CP *cp, CLASS *class, GENERAL_DATA *general_data, int ip_now) {
  STODFTINFO *si = cp->stodftInfo;
  STODFTCOEFPOS *sp = cp->stodftCoefPos;
  NEWTONINFO *ni = si->newtonInfo;
  CPCOEFFS_POS *pos = &cp->cpcoeffs_pos[ip_now];
  const int ns = cp->cpcoeffs_info.nstate_up_proc, L = si->polynormLength, nmu = si->numChemPot;
  ad_no_entropy(si, "filterNewtonPolyHerm");
  AdSys *s = ad_attach(cp, class, general_data, &class->clatoms_pos[ip_now], ns, "filterNewtonPolyHerm");
  if (si->storeChebyMomentsFlag) sp->chebyMomentsUp = (double *)cmalloc((L + 1) * sizeof(double)); /* filter.c:98 */
  double **re = malloc(sizeof(double *) * nmu), **im = malloc(sizeof(double *) * nmu);
  for (int imu = 0; imu < nmu; imu++) {
    re[imu] = &sp->stoWfUpRe[imu][1];
    im[imu] = &sp->stoWfUpIm[imu][1];
  }
  ad_ck(sdft_filter_newton(s->ctx, ns, &pos->cre_up[1], &pos->cim_up[1], L, nmu, sp->expanCoeff,
                           (const double *)ni->sampPoint, ni->scale, si->energyMean, re, im),
        "filterNewtonPolyHerm");
  free(re);
  free(im);
}

void calcChebyMoments(CP *cp, CLASS *class, GENERAL_DATA *general_data, int ip_now) {
  STODFTINFO *si = cp->stodftInfo;
  STODFTCOEFPOS *sp = cp->stodftCoefPos;
  CPCOEFFS_POS *pos = &cp->cpcoeffs_pos[ip_now];
  const int ns = cp->cpcoeffs_info.nstate_up_proc;
  if (cp->cpopts.cp_lsda != 0) ad_die("calcChebyMoments", "spin-polarised runs (cp_lsda = 1) are not supported");
  AdSys *s = ad_attach(cp, class, general_data, &class->clatoms_pos[ip_now], ns, "calcChebyMoments");
  genNoiseOrbitalReal(cp, pos); /* the noise as calc-chempot-chebyshev.c:685 draws it */
  ad_ck(sdft_cheby_moments(s->ctx, ns, &pos->cre_up[1], &pos->cim_up[1], si->polynormLength,
                           si->chebyshevInfo->scale, si->energyMean, sp->chebyMomentsUp),
        "calcChebyMoments");
}

void rhoCalcRealStoHybrid(CPSCR *cpscr, CPCOEFFS_INFO *cpcoeffs_info, CELL *cell, STODFTINFO *stodftInfo,
                          double *creal, double *cimag, double *rho_scr, int icoef_form, int icoef_orth, int nstate,
                          int ncoef, int cp_dual_grid_opt, COMMUNICATE *communicate,
                          PARA_FFT_PKG3D *cp_para_fft_pkg3d_lg, PARA_FFT_PKG3D *cp_sclr_fft_pkg3d_lg,
                          PARA_FFT_PKG3D *cp_para_fft_pkg3d_dens_cp_box,
                          PARA_FFT_PKG3D *cp_sclr_fft_pkg3d_dens_cp_box, PARA_FFT_PKG3D *cp_sclr_fft_pkg3d_sm) {
  (void)cpscr; (void)cpcoeffs_info; (void)cell; (void)stodftInfo; (void)cp_para_fft_pkg3d_lg;
  (void)cp_sclr_fft_pkg3d_lg; (void)cp_para_fft_pkg3d_dens_cp_box; (void)cp_sclr_fft_pkg3d_dens_cp_box;
  if (icoef_orth != 1) ad_die("rhoCalcRealStoHybrid", "the coefficients must be in orthogonal form");
  if (communicate->np_states > 1 && icoef_form == 1)
    ad_die("rhoCalcRealStoHybrid", "the coefficients must be in normal (not transposed) form");
  if (cp_dual_grid_opt != 0) ad_die("rhoCalcRealStoHybrid", "dual grids (cp_dual_grid_opt > 0) are not supported");
  AdSys *s = ad_find(cp_sclr_fft_pkg3d_sm);
  if (!s || !s->ctx)
    ad_die("rhoCalcRealStoHybrid", "no device context for this system yet: an H application or filter creates it");
  if (ncoef != s->ncoef) ad_die("rhoCalcRealStoHybrid", "ncoef differs from the system's");
  if (nstate > s->max_states) ad_die("rhoCalcRealStoHybrid", "more orbitals than the context holds");
  if (nstate < 1) {
    for (int i = 1; i <= s->N; i++) rho_scr[i] = 0.0;
    return;
  }
  ad_ck(sdft_density(s->ctx, nstate, &creal[1], &cimag[1], &rho_scr[1]), "rhoCalcRealStoHybrid");
}

/* genNoiseOrbitalReal (stodft/gen-noise.c:162-374), spin-unpolarised: the
 * noise orbitals of state rank myid_state of np_states from
 * stodftInfo->randSeed, generated on the device (the gaussran2 sign
 * sequence, +-sqrt(N) in real space, transformed to G).  The signature
 * carries no cell, so an earlier call with the CLASS must have made the
 * system's context. */
void sdft_piny_noise(CP *cp, CPCOEFFS_POS *cpcoeffs_pos) {
  const int ns = cp->cpcoeffs_info.nstate_up_proc;
  if (cp->cpopts.cp_lsda != 0) ad_die("genNoiseOrbitalReal", "spin-polarised runs (cp_lsda = 1) are not supported");
  AdSys *s = ad_find(&cp->cp_sclr_fft_pkg3d_sm);
  if (!s || !s->ctx)
    ad_die("genNoiseOrbitalReal", "no device context for this system yet: an H application or filter creates it");
  if (ns > s->max_states)
    ad_die("genNoiseOrbitalReal", "more orbitals than the context was made for (set SDFT_PINY_MAX_STATES)");
  ad_ck(sdft_noise_real(s->ctx, ns, cp->stodftInfo->randSeed, cp->communicate.np_states, cp->communicate.myid_state,
                        &cpcoeffs_pos->cre_up[1], &cpcoeffs_pos->cim_up[1]),
        "genNoiseOrbitalReal");
}

#ifndef SDFT_PINY_ADAPTER_NO_NOISE
void genNoiseOrbitalReal(CP *cp, CPCOEFFS_POS *cpcoeffs_pos) { sdft_piny_noise(cp, cpcoeffs_pos); }
#endif

#endif /* SDFT_PINY_ADAPTER */
