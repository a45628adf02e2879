/*
 * sdft_oracle.c -- CPU oracle for the stochastic-DFT filter hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain FP64 C restatement of the
 * reference (mingchenPurdueChem/stochastic-density-functional-theory-piny)
 * algorithm, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg as the checker.  The product library never links or calls
 * it.  Every routine cites the reference file:line it follows.  The
 * restatement is pinned against the reference's own C sources compiled in
 * this container (oracle/build_ref.sh -> oracle/_ref/, tests/test_oracle_pin.py);
 * FFTs use this file's own mixed-radix transform in place of FFTW.
 *
 * Conventions: orbital arrays are PINY's (state-major, half sphere, G = 0
 * last, separate re/im) but 0-based.  Grids: "filter layout" index
 * (ia*n2 + ib)*n3 + ic (c fastest); "package layout" ia + n1*(ib + n2*ic).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "sdft_oracle.h"

/* ------------------------------------------------------------------------ */
/* 1-D mixed radix (2,3) complex FFT, sign s: exp(s*2 pi i jk/n)            */
/* ------------------------------------------------------------------------ */
static void fft1d_rec(const double *xr, const double *xi, int n, int stride, double *yr, double *yi,
                      int sgn, double *scr) {
  if (n == 1) { yr[0] = xr[0]; yi[0] = xi[0]; return; }
  int r = (n % 3 == 0) ? 3 : ((n % 2 == 0) ? 2 : n);
  int m = n / r;
  double *sr = scr, *si = scr + n, *nscr = scr + 2 * n;
  for (int q = 0; q < r; q++) fft1d_rec(xr + q * stride, xi + q * stride, m, stride * r, sr + q * m, si + q * m, sgn, nscr);
  for (int k = 0; k < m; k++) {
    double vr[3], vi[3];
    for (int q = 0; q < r; q++) {
      double a = sgn * 2.0 * M_PI * (double)(q * k) / (double)n;
      double c = cos(a), s = sin(a);
      vr[q] = sr[q * m + k] * c - si[q * m + k] * s;
      vi[q] = sr[q * m + k] * s + si[q * m + k] * c;
    }
    for (int t = 0; t < r; t++) {
      double ar = 0.0, ai = 0.0;
      for (int q = 0; q < r; q++) {
        double a = sgn * 2.0 * M_PI * (double)(q * t) / (double)r;
        double c = cos(a), s = sin(a);
        ar += vr[q] * c - vi[q] * s;
        ai += vr[q] * s + vi[q] * c;
      }
      yr[k + t * m] = ar;
      yi[k + t * m] = ai;
    }
  }
}

/* in place 1-D FFT of n complex values with element stride es */
static void fft1d(double *re, double *im, int n, long es, int sgn) {
  double *xr = malloc(sizeof(double) * n * 2), *xi = xr + n;
  double *yr = malloc(sizeof(double) * n * 2), *yi = yr + n;
  double *scr = malloc(sizeof(double) * n * 8 * 8);
  for (int j = 0; j < n; j++) { xr[j] = re[j * es]; xi[j] = im[j * es]; }
  fft1d_rec(xr, xi, n, 1, yr, yi, sgn, scr);
  for (int j = 0; j < n; j++) { re[j * es] = yr[j]; im[j * es] = yi[j]; }
  free(xr); free(yr); free(scr);
}

/* 3-D FFT on the filter layout (c fastest), unnormalised. */
static void fft3d(double *re, double *im, int n1, int n2, int n3, int sgn) {
  for (int a = 0; a < n1; a++)
    for (int b = 0; b < n2; b++) fft1d(re + ((long)a * n2 + b) * n3, im + ((long)a * n2 + b) * n3, n3, 1, sgn);
  for (int a = 0; a < n1; a++)
    for (int c = 0; c < n3; c++) fft1d(re + (long)a * n2 * n3 + c, im + (long)a * n2 * n3 + c, n2, n3, sgn);
  for (int b = 0; b < n2; b++)
    for (int c = 0; c < n3; c++) fft1d(re + (long)b * n3 + c, im + (long)b * n3 + c, n1, (long)n2 * n3, sgn);
}

static void inv3(const double *h, double *hi) {
#define H(i, j) h[(i) + 3 * (j)]
  double det = H(0, 0) * (H(1, 1) * H(2, 2) - H(1, 2) * H(2, 1)) - H(0, 1) * (H(1, 0) * H(2, 2) - H(1, 2) * H(2, 0)) +
               H(0, 2) * (H(1, 0) * H(2, 1) - H(1, 1) * H(2, 0));
  double m[3][3];
  m[0][0] = (H(1, 1) * H(2, 2) - H(1, 2) * H(2, 1)) / det;
  m[0][1] = (H(0, 2) * H(2, 1) - H(0, 1) * H(2, 2)) / det;
  m[0][2] = (H(0, 1) * H(1, 2) - H(0, 2) * H(1, 1)) / det;
  m[1][0] = (H(1, 2) * H(2, 0) - H(1, 0) * H(2, 2)) / det;
  m[1][1] = (H(0, 0) * H(2, 2) - H(0, 2) * H(2, 0)) / det;
  m[1][2] = (H(0, 2) * H(1, 0) - H(0, 0) * H(1, 2)) / det;
  m[2][0] = (H(1, 0) * H(2, 1) - H(1, 1) * H(2, 0)) / det;
  m[2][1] = (H(0, 1) * H(2, 0) - H(0, 0) * H(2, 1)) / det;
  m[2][2] = (H(0, 0) * H(1, 1) - H(0, 1) * H(1, 0)) / det;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) hi[i + 3 * j] = m[i][j];
#undef H
}
static double det3(const double *h) {
  return fabs(h[0] * (h[4] * h[8] - h[7] * h[5]) - h[3] * (h[1] * h[8] - h[7] * h[2]) + h[6] * (h[1] * h[5] - h[4] * h[2]));
}

/* ------------------------------------------------------------------------ */
/* G vectors: setkvec3d_sm (interface/cp_ewald/set_cp_ewald.c:685-833)      */
/* ------------------------------------------------------------------------ */
static double try_e(const double *hi, double a, double b, double c) {
  double tpi = 2.0 * M_PI;
  double xk = (a * hi[0] + b * hi[1] + c * hi[2]) * tpi;
  double yk = (a * hi[3] + b * hi[4] + c * hi[5]) * tpi;
  double zk = (a * hi[6] + b * hi[7] + c * hi[8]) * tpi;
  return (xk * xk + yk * yk + zk * zk) * .5;
}

int oracle_gvec(const double *hmat, double ecut, const int *kmax, int cap, int *ka, int *kb, int *kc, int *ib1,
                int *ib2) {
  double hi[9];
  inv3(hmat, hi);
  int i, icount = 0;
  for (i = 1; i <= kmax[0]; ++i)
    if (try_e(hi, i, 0, 0) > ecut) break;
  int kamax = i - 1;
  for (int a = 0; a <= kamax; ++a) {
    int kbmin = (a == 0) ? 0 : -kmax[1];
    for (i = kbmin; i <= 0; ++i)
      if (try_e(hi, a, i, 0) <= ecut) break;
    kbmin = i;
    for (i = 1; i <= kmax[1]; ++i)
      if (try_e(hi, a, i, 0) > ecut) break;
    int kbmax = i - 1;
    for (int b = kbmin; b <= kbmax; ++b) {
      int kcmin = (a == 0 && b == 0) ? 1 : -kmax[2];
      for (i = kcmin; i <= 0; ++i)
        if (try_e(hi, a, b, i) <= ecut) break;
      kcmin = i;
      for (i = 1; i <= kmax[2]; ++i)
        if (try_e(hi, a, b, i) > ecut) break;
      int kcmax = i - 1;
      for (int c = kcmin; c <= kcmax; ++c) {
        if (ka && icount < cap) {
          ka[icount] = a; kb[icount] = b; kc[icount] = c;
          if (ib1) ib1[icount] = (c == kcmin);
          if (ib2) ib2[icount] = (c < kcmax);
        }
        icount++;
      }
    }
  }
  if (ka && icount < cap) { ka[icount] = kb[icount] = kc[icount] = 0; }
  return icount; /* nktot; ncoef = nktot + 1 */
}

/* ------------------------------------------------------------------------ */
/* Context                                                                  */
/* ------------------------------------------------------------------------ */
struct oracle_sys {
  int n1, n2, n3, N, ncoef;
  int *ka, *kb, *kc, *ib1, *ib2;
  int *map, *mapc;      /* filter maps (complex index) of G and -G       */
  double hmat[9], hmati[9], vol;
  double *ak2;          /* ak2Kinetic                                    */
  double *vks;          /* filter layout                                 */
  /* KB */
  int natm, ntype, lmax, nsplin;
  double *pos;          /* natm*3                                        */
  int *type, *lmax_type;
  double gmin, dg;
  double *vps, *vpsnorm, *gzvps0;
};

oracle_sys *oracle_create(int n1, int n2, int n3, int ncoef, const int *ka, const int *kb, const int *kc,
                          const int *ib1, const int *ib2, const double *hmat) {
  oracle_sys *s = calloc(1, sizeof(*s));
  s->n1 = n1; s->n2 = n2; s->n3 = n3; s->N = n1 * n2 * n3; s->ncoef = ncoef;
  s->ka = malloc(sizeof(int) * ncoef); s->kb = malloc(sizeof(int) * ncoef); s->kc = malloc(sizeof(int) * ncoef);
  s->ib1 = malloc(sizeof(int) * ncoef); s->ib2 = malloc(sizeof(int) * ncoef);
  memcpy(s->ka, ka, sizeof(int) * ncoef); memcpy(s->kb, kb, sizeof(int) * ncoef); memcpy(s->kc, kc, sizeof(int) * ncoef);
  memcpy(s->ib1, ib1, sizeof(int) * (ncoef - 1)); memcpy(s->ib2, ib2, sizeof(int) * (ncoef - 1));
  memcpy(s->hmat, hmat, sizeof(double) * 9);
  inv3(hmat, s->hmati);
  s->vol = det3(hmat);
  /* setfft_indx (mathlib/fft_create_package.c:981-1020) + (idx-1)/2 */
  s->map = malloc(sizeof(int) * ncoef); s->mapc = malloc(sizeof(int) * ncoef);
  for (int i = 0; i < ncoef - 1; i++) {
    int a = ka[i], b = kb[i], c = kc[i];
    int kap = (a < 0 ? a + n1 + 1 : a + 1), kbp = (b < 0 ? b + n2 + 1 : b + 1), kcp = (c < 0 ? c + n3 + 1 : c + 1);
    int idx = kcp * 2 - 1 + (kbp - 1) * 2 * n3 + (kap - 1) * 2 * n3 * n2;
    s->map[i] = (idx - 1) / 2;
    kap = (-a < 0 ? -a + n1 + 1 : -a + 1); kbp = (-b < 0 ? -b + n2 + 1 : -b + 1); kcp = (-c < 0 ? -c + n3 + 1 : -c + 1);
    idx = kcp * 2 - 1 + (kbp - 1) * 2 * n3 + (kap - 1) * 2 * n3 * n2;
    s->mapc[i] = (idx - 1) / 2;
  }
  s->map[ncoef - 1] = 0; s->mapc[ncoef - 1] = 0;
  /* get_ak2_sm (energy/cp/cp_energy_eext.c:2260-2303), no kinetic cap   */
  s->ak2 = malloc(sizeof(double) * ncoef);
  for (int i = 0; i < ncoef - 1; i++) {
    double tpi = 2.0 * M_PI, a = ka[i], b = kb[i], c = kc[i];
    double *h = s->hmati;
    double xk = (a * h[0] + b * h[1] + c * h[2]) * tpi, yk = (a * h[3] + b * h[4] + c * h[5]) * tpi,
           zk = (a * h[6] + b * h[7] + c * h[8]) * tpi;
    s->ak2[i] = xk * xk + yk * yk + zk * zk;
  }
  s->ak2[ncoef - 1] = 0.0;
  s->vks = calloc(s->N, sizeof(double));
  return s;
}

void oracle_destroy(oracle_sys *s) {
  if (!s) return;
  free(s->ka); free(s->kb); free(s->kc); free(s->ib1); free(s->ib2); free(s->map); free(s->mapc);
  free(s->ak2); free(s->vks); free(s->pos); free(s->type); free(s->lmax_type); free(s->vps); free(s->vpsnorm);
  free(s->gzvps0); free(s);
}

void oracle_set_vks(oracle_sys *s, const double *v) { memcpy(s->vks, v, sizeof(double) * s->N); }
void oracle_set_kinetic_cap(oracle_sys *s, double gcut) {
  double g2 = gcut > 0 ? gcut * gcut : 1e30;
  for (int i = 0; i < s->ncoef - 1; i++)
    if (s->ak2[i] > g2) s->ak2[i] = g2;
}

void oracle_set_kb(oracle_sys *s, int natm, const double *pos, const int *type, int ntype, int lmax,
                   const int *lmax_type, int nsplin, double gmin, double dg, const double *vps,
                   const double *vpsnorm, const double *gzvps0) {
  s->natm = natm; s->ntype = ntype; s->lmax = lmax; s->nsplin = nsplin; s->gmin = gmin; s->dg = dg;
  s->pos = malloc(sizeof(double) * 3 * natm); memcpy(s->pos, pos, sizeof(double) * 3 * natm);
  s->type = malloc(sizeof(int) * natm); memcpy(s->type, type, sizeof(int) * natm);
  s->lmax_type = malloc(sizeof(int) * ntype); memcpy(s->lmax_type, lmax_type, sizeof(int) * ntype);
  size_t nv = (size_t)ntype * (lmax + 1) * 4 * nsplin;
  s->vps = malloc(sizeof(double) * nv); memcpy(s->vps, vps, sizeof(double) * nv);
  s->vpsnorm = malloc(sizeof(double) * ntype * (lmax + 1)); memcpy(s->vpsnorm, vpsnorm, sizeof(double) * ntype * (lmax + 1));
  s->gzvps0 = malloc(sizeof(double) * ntype); memcpy(s->gzvps0, gzvps0, sizeof(double) * ntype);
}

/* get_vpsnow (energy/cp/cp_energy_eext.c:2139-2185) */
static double vpsnow(const oracle_sys *s, int t, int l, double g) {
  int iii = (int)((g - s->gmin) / s->dg) + 1;
  if (iii > s->nsplin) iii = s->nsplin;
  if (iii < 1) iii = 1;
  double h0 = (double)(iii - 1) * s->dg + s->gmin;
  double h = g - h0;
  const double *tab = s->vps + ((size_t)t * (s->lmax + 1) + l) * 4 * s->nsplin;
  int i = iii - 1;
  return ((tab[3 * s->nsplin + i] * h + tab[2 * s->nsplin + i]) * h + tab[s->nsplin + i]) * h + tab[i];
}

/* get_ylm values, l <= 2 (energy/cp/cp_energy_eext_nonloc.c:2350) */
static void ylm(double xk, double yk, double zk, double g, double *yr, double *yi) {
  double fpi = 4.0 * M_PI;
  double rt_fpi = 1.0 / sqrt(fpi), rt_thrfpi = sqrt(3.0 / fpi), rt_threpi = sqrt(1.50 / fpi);
  double hrt_fivfpi = 0.50 * sqrt(5.0 / fpi), rt_fiftepi = sqrt(7.50 / fpi);
  double ct = zk / g, st = sqrt(xk * xk + yk * yk) / g, xyd = sqrt(xk * xk + yk * yk), cp, sp;
  if (xyd == 0) { cp = 1.0; sp = 0.0; } else { cp = xk / xyd; sp = yk / xyd; }
  double c2 = cp * cp - sp * sp, s2 = 2.0 * cp * sp;
  for (int i = 0; i < 10; i++) yr[i] = yi[i] = 0.0;
  yr[1] = rt_fpi;
  yr[2] = rt_thrfpi * ct;
  yr[3] = rt_threpi * st * cp; yi[3] = rt_threpi * st * sp;
  yr[4] = yr[3]; yi[4] = -yi[3];
  yr[5] = hrt_fivfpi * (3.0 * ct * ct - 1.0);
  yr[6] = rt_fiftepi * st * ct * cp; yi[6] = rt_fiftepi * st * ct * sp;
  yr[7] = yr[6]; yi[7] = -yi[6];
  yr[8] = 0.50 * rt_fiftepi * st * st * c2; yi[8] = 0.50 * rt_fiftepi * st * st * s2;
  yr[9] = yr[8]; yi[9] = -yi[8];
}

/* ------------------------------------------------------------------------ */
/* KB nonlocal force, in the reference's per-G form                         */
/*   projection   controlEwdNonlocFilter stodft/reduced-energy/cp-energy-eext-stodft.c:701-951
 *                getNlmatFilter :1105-1169, get_nlmat0 energy/cp/cp_energy_eext_nonloc.c:1083
 *   energy       getNlPotPvFatmSCF :522-634 / sumNlPot :640-696
 *   back proj.   getnl_fcoef energy/cp/cp_energy_eext_nonloc.c:1669-1935, control_nlfcoef,
 *                get_nlfor :2136-2173, get_nlfor0 :2229-2265                             */
/* ------------------------------------------------------------------------ */
/* Z[atom][state][lm] re/im of the KB projection and, when dzr is given, its
 * derivatives by the atom positions dZ/dR_d (d = x, y, z; [d][atom][state][lm]),
 * as get_nlmat accumulates them next to Z (energy/cp/cp_energy_eext_nonloc.c:
 * 648-748): d(c e^{iG.R})/dR_d = i G_d c e^{iG.R}, so for even l
 * dZr_d += -cbyhel_i 2Yr G_d, dZi_d += -cbyhel_i 2Yi G_d and for odd l
 * dZr_d += -cbyhel_r 2Yi G_d, dZi_d += cbyhel_r 2Yr G_d.  The G = 0 term has
 * no position dependence.  Caller zeroes zr, zi (and dzr, dzi). */
static void kb_project(const oracle_sys *s, int nstate, const double *cre, const double *cim, double *zr, double *zi,
                       double *dzr, double *dzi) {
  const int ncoef = s->ncoef, nk = ncoef - 1, natm = s->natm;
  const int nlm = (s->lmax + 1) * (s->lmax + 1);
  const size_t zn = (size_t)natm * nstate * nlm;
  const double tpi = 2.0 * M_PI, *hi = s->hmati;
  double *sx = malloc(sizeof(double) * natm * 3), *cossc = malloc(sizeof(double) * natm),
         *sinsc = malloc(sizeof(double) * natm), *helr = malloc(sizeof(double) * natm),
         *heli = malloc(sizeof(double) * natm);
#define ZI(a, st, lm) (((size_t)(a) * nstate + (st)) * nlm + (lm))
  for (int a = 0; a < natm; a++) {
    double dx = s->pos[3 * a], dy = s->pos[3 * a + 1], dz = s->pos[3 * a + 2];
    double as[3] = {dx * hi[0] + dy * hi[3] + dz * hi[6], dx * hi[1] + dy * hi[4] + dz * hi[7],
                    dx * hi[2] + dy * hi[5] + dz * hi[8]};
    for (int d = 0; d < 3; d++) sx[3 * a + d] = as[d] - nearbyint(as[d]);
    cossc[a] = cos(sx[3 * a + 2] * tpi);
    sinsc[a] = sin(sx[3 * a + 2] * tpi);
  }
  double yr[10], yi[10];
  for (int ic = 0; ic < nk; ic++) {
    double aka = s->ka[ic], akb = s->kb[ic], akc = s->kc[ic];
    double xk = (aka * hi[0] + akb * hi[1] + akc * hi[2]) * tpi, yk = (aka * hi[3] + akb * hi[4] + akc * hi[5]) * tpi,
           zk = (aka * hi[6] + akb * hi[7] + akc * hi[8]) * tpi;
    double g = sqrt(xk * xk + yk * yk + zk * zk), gk[3] = {xk, yk, zk};
    if (s->ib1[ic])
      for (int a = 0; a < natm; a++) {
        double arg = (aka * sx[3 * a] + akb * sx[3 * a + 1] + akc * sx[3 * a + 2]) * tpi;
        helr[a] = cos(arg); heli[a] = sin(arg);
      }
    ylm(xk, yk, zk, g, yr, yi);
    for (int a = 0; a < natm; a++) {
      int t = s->type[a];
      for (int l = 0; l <= s->lmax_type[t]; l++) {
        double v = vpsnow(s, t, l, g);
        double hr = helr[a] * v, hm = heli[a] * v;
        for (int m = 1; m <= 2 * l + 1; m++) {
          int lm = m + l * l;
          double tyr = 2.0 * yr[lm], tyi = 2.0 * yi[lm];
          for (int st = 0; st < nstate; st++) {
            double c_r = cre[(size_t)st * ncoef + ic], c_i = cim[(size_t)st * ncoef + ic];
            double bhr = c_r * hr - c_i * hm, bhi = c_r * hm + c_i * hr;
            size_t z = ZI(a, st, lm - 1);
            if (l % 2 == 1) { zr[z] += -bhi * tyi; zi[z] += bhi * tyr; }
            else { zr[z] += bhr * tyr; zi[z] += bhr * tyi; }
            if (dzr)
              for (int d = 0; d < 3; d++) {
                if (l % 2 == 1) { dzr[d * zn + z] += -bhr * tyi * gk[d]; dzi[d * zn + z] += bhr * tyr * gk[d]; }
                else { dzr[d * zn + z] += -bhi * tyr * gk[d]; dzi[d * zn + z] += -bhi * tyi * gk[d]; }
              }
          }
        }
      }
    }
    if (s->ib2[ic])
      for (int a = 0; a < natm; a++) {
        double t = helr[a];
        helr[a] = helr[a] * cossc[a] - heli[a] * sinsc[a];
        heli[a] = heli[a] * cossc[a] + t * sinsc[a];
      }
  }
  /* G = 0, l = 0 */
  {
    double y00 = 1.0 / sqrt(4.0 * M_PI);
    for (int a = 0; a < natm; a++) {
      int t = s->type[a];
      if (s->lmax_type[t] < 0) continue;
      double vt = s->gzvps0[t] * y00;
      for (int st = 0; st < nstate; st++) zr[ZI(a, st, 0)] += cre[(size_t)st * ncoef + nk] * vt;
    }
  }
#undef ZI
  free(sx); free(cossc); free(sinsc); free(helr); free(heli);
}

static void kb_force(const oracle_sys *s, int nstate, const double *cre, const double *cim, double *fcre,
                     double *fcim, double *enl_out) {
  if (s->natm == 0) { if (enl_out) *enl_out = 0.0; return; }
  const int ncoef = s->ncoef, nk = ncoef - 1, natm = s->natm;
  const int nlm = (s->lmax + 1) * (s->lmax + 1);
  const double tpi = 2.0 * M_PI, *hi = s->hmati;
  /* Z[atom][state][lm] re/im */
  double *zr = calloc((size_t)natm * nstate * nlm, sizeof(double));
  double *zi = calloc((size_t)natm * nstate * nlm, sizeof(double));
  double *sx = malloc(sizeof(double) * natm * 3), *cossc = malloc(sizeof(double) * natm),
         *sinsc = malloc(sizeof(double) * natm), *helr = malloc(sizeof(double) * natm),
         *heli = malloc(sizeof(double) * natm);
#define ZI(a, st, lm) (((size_t)(a) * nstate + (st)) * nlm + (lm))
  for (int a = 0; a < natm; a++) {
    double dx = s->pos[3 * a], dy = s->pos[3 * a + 1], dz = s->pos[3 * a + 2];
    double as[3] = {dx * hi[0] + dy * hi[3] + dz * hi[6], dx * hi[1] + dy * hi[4] + dz * hi[7],
                    dx * hi[2] + dy * hi[5] + dz * hi[8]};
    for (int d = 0; d < 3; d++) sx[3 * a + d] = as[d] - nearbyint(as[d]);
  }
  double yr[10], yi[10];
  kb_project(s, nstate, cre, cim, zr, zi, NULL, NULL);
  /* energy */
  double enl = 0.0;
  for (int a = 0; a < natm; a++) {
    int t = s->type[a];
    for (int l = 0; l <= s->lmax_type[t]; l++) {
      double vn = s->vpsnorm[t * (s->lmax + 1) + l] / s->vol;
      for (int m = 1; m <= 2 * l + 1; m++)
        for (int st = 0; st < nstate; st++) {
          size_t z = ZI(a, st, m + l * l - 1);
          enl += (zr[z] * zr[z] + zi[z] * zi[z]) * vn;
        }
    }
  }
  if (enl_out) *enl_out = enl;
  /* back projection (getnl_fcoef uses -cp_box_center_rel; zero here) */
  for (int a = 0; a < natm; a++) { cossc[a] = cos(sx[3 * a + 2] * tpi); sinsc[a] = sin(sx[3 * a + 2] * tpi); }
  double rvol4 = 4.0 / s->vol;
  for (int ic = 0; ic < nk; ic++) {
    double aka = s->ka[ic], akb = s->kb[ic], akc = s->kc[ic];
    double xk = (aka * hi[0] + akb * hi[1] + akc * hi[2]) * tpi, yk = (aka * hi[3] + akb * hi[4] + akc * hi[5]) * tpi,
           zk = (aka * hi[6] + akb * hi[7] + akc * hi[8]) * tpi;
    double g = sqrt(xk * xk + yk * yk + zk * zk);
    if (s->ib1[ic])
      for (int a = 0; a < natm; a++) {
        double arg = (aka * sx[3 * a] + akb * sx[3 * a + 1] + akc * sx[3 * a + 2]) * tpi;
        helr[a] = cos(arg); heli[a] = sin(arg);
      }
    ylm(xk, yk, zk, g, yr, yi);
    for (int a = 0; a < natm; a++) {
      int t = s->type[a];
      for (int l = 0; l <= s->lmax_type[t]; l++) {
        double v = vpsnow(s, t, l, g);
        double tmp = v * rvol4;
        double hr = helr[a] * tmp, hm = heli[a] * tmp;
        double vn = s->vpsnorm[t * (s->lmax + 1) + l];
        for (int m = 1; m <= 2 * l + 1; m++) {
          int lm = m + l * l;
          double vfr = hr * yr[lm] - hm * yi[lm];
          double vfi = -(hm * yr[lm] + hr * yi[lm]);
          for (int st = 0; st < nstate; st++) {
            size_t z = ZI(a, st, lm - 1);
            fcre[(size_t)st * ncoef + ic] += -(vfr * zr[z] - vfi * zi[z]) * vn;
            fcim[(size_t)st * ncoef + ic] += -(vfi * zr[z] + vfr * zi[z]) * vn;
          }
        }
      }
    }
    if (s->ib2[ic])
      for (int a = 0; a < natm; a++) {
        double t = helr[a];
        helr[a] = helr[a] * cossc[a] - heli[a] * sinsc[a];
        heli[a] = heli[a] * cossc[a] + t * sinsc[a];
      }
  }
  {
    double y00 = 1.0 / sqrt(4.0 * M_PI);
    for (int a = 0; a < natm; a++) {
      int t = s->type[a];
      if (s->lmax_type[t] < 0) continue;
      double vn = s->vpsnorm[t * (s->lmax + 1)];
      double vf = y00 * s->gzvps0[t] * vn / s->vol;
      for (int st = 0; st < nstate; st++) fcre[(size_t)st * ncoef + nk] -= 2.0 * vf * zr[ZI(a, st, 0)];
    }
  }
#undef ZI
  free(zr); free(zi); free(sx); free(cossc); free(sinsc); free(helr); free(heli);
}

/* KB nonlocal atomic forces and energy of nstate orbitals, the sum that
 * calcNlPseudoPostScf (stodft/reduced-energy/energy-wrapper-post-scf.c:224-615)
 * forms through control_ewd_non_loc / get_nlmat and getnl_pot_pv_fatm ->
 * sumnl_pot_pv_fatm_hess (energy/cp/cp_energy_eext_nonloc.c:1122-1530), one
 * radial channel:  F_a,d = -2 sum_{state, l, m} (dZr_d Zr + dZi_d Zi) vnorm_l / vol,
 * E_NL = sum |Z|^2 vnorm_l / vol.  Raw sums over the given states, before the
 * occNumber / numStateStoUp of calcEnergyForce (stodft/calc-nuclei-force.c:
 * 462-480).  f: natm * 3 (x, y, z per atom). */
void oracle_nl_force(const oracle_sys *s, int nstate, const double *cre, const double *cim, double *f, double *enl) {
  const int natm = s->natm;
  for (int i = 0; i < 3 * natm; i++) f[i] = 0.0;
  if (enl) *enl = 0.0;
  if (natm == 0 || nstate < 1) return;
  const int nlm = (s->lmax + 1) * (s->lmax + 1);
  const size_t zn = (size_t)natm * nstate * nlm;
  double *zr = calloc(zn, sizeof(double)), *zi = calloc(zn, sizeof(double));
  double *dzr = calloc(3 * zn, sizeof(double)), *dzi = calloc(3 * zn, sizeof(double));
  kb_project(s, nstate, cre, cim, zr, zi, dzr, dzi);
  double e = 0.0;
  for (int a = 0; a < natm; a++) {
    int t = s->type[a];
    for (int l = 0; l <= s->lmax_type[t]; l++) {
      double vn = s->vpsnorm[t * (s->lmax + 1) + l] / s->vol;
      for (int m = 1; m <= 2 * l + 1; m++)
        for (int st = 0; st < nstate; st++) {
          size_t z = ((size_t)a * nstate + st) * nlm + (m + l * l - 1);
          e += (zr[z] * zr[z] + zi[z] * zi[z]) * vn;
          for (int d = 0; d < 3; d++) f[3 * a + d] += -2.0 * (dzr[d * zn + z] * zr[z] + dzi[d * zn + z] * zi[z]) * vn;
        }
    }
  }
  if (enl) *enl = e;
  free(zr); free(zi); free(dzr); free(dzi);
}

/* ------------------------------------------------------------------------ */
/* H psi: calcCoefForceWrapSCF (stodft/reduced-energy/energy-wrapper-scf.c:1066-1196)
 * -> coefForceCalcHybridSCF (cp-energy-ee-rho-stodft.c:38-355) with the
 * filter FFT wrappers (mathlib/fft_package.c:3195-3660) and cp_vpsi.       */
/* ------------------------------------------------------------------------ */
void oracle_hpsi(const oracle_sys *s, int nstate, const double *cre, const double *cim, double *fcre, double *fcim,
                 double *enl) {
  const int ncoef = s->ncoef, N = s->N;
  memset(fcre, 0, sizeof(double) * nstate * ncoef);
  memset(fcim, 0, sizeof(double) * nstate * ncoef);
  kb_force(s, nstate, cre, cim, fcre, fcim, enl);
  double *zr = malloc(sizeof(double) * N), *zi = malloc(sizeof(double) * N);
  const double inv = 1.0 / N;
  for (int is = 0; is < nstate; is += 2) {
    int pair = (is + 1 < nstate);
    const double *c1r = cre + (size_t)is * ncoef, *c1i = cim + (size_t)is * ncoef;
    memset(zr, 0, sizeof(double) * N);
    memset(zi, 0, sizeof(double) * N);
    if (pair) { /* dble_pack_coef_fftw3d_filter :3195-3259 */
      const double *c2r = cre + (size_t)(is + 1) * ncoef, *c2i = cim + (size_t)(is + 1) * ncoef;
      for (int i = 0; i < ncoef - 1; i++) {
        zr[s->map[i]] = c1r[i] - c2i[i]; zi[s->map[i]] = c1i[i] + c2r[i];
        zr[s->mapc[i]] = c1r[i] + c2i[i]; zi[s->mapc[i]] = -c1i[i] + c2r[i];
      }
      zr[0] = c1r[ncoef - 1]; zi[0] = c2r[ncoef - 1];
    } else { /* sngl_pack_coef_fftw3d_filter :3263-3327 */
      for (int i = 0; i < ncoef - 1; i++) {
        zr[s->map[i]] = c1r[i]; zi[s->map[i]] = c1i[i];
        zr[s->mapc[i]] = c1r[i]; zi[s->mapc[i]] = -c1i[i];
      }
      zr[0] = c1r[ncoef - 1]; zi[0] = c1i[ncoef - 1];
    }
    fft3d(zr, zi, s->n1, s->n2, s->n3, +1); /* FFTW_BACKWARD */
    for (int m = 0; m < N; m++) { zr[m] *= s->vks[m]; zi[m] *= s->vks[m]; } /* cp_vpsi */
    fft3d(zr, zi, s->n1, s->n2, s->n3, -1); /* FFTW_FORWARD */
    double *f1r = fcre + (size_t)is * ncoef, *f1i = fcim + (size_t)is * ncoef;
    if (pair) { /* dble_upack_coef_sum_fftw3d_filter :3513-3600 */
      double *f2r = fcre + (size_t)(is + 1) * ncoef, *f2i = fcim + (size_t)(is + 1) * ncoef;
      for (int i = 0; i < ncoef - 1; i++) {
        double tr = zr[s->map[i]] * inv, ti = zi[s->map[i]] * inv;
        double trc = zr[s->mapc[i]] * inv, tic = zi[s->mapc[i]] * inv;
        f2i[i] -= (2.0 * (-tr + trc));
        f1r[i] -= (2.0 * (tr + trc));
        f1i[i] -= (2.0 * (ti - tic));
        f2r[i] -= (2.0 * (ti + tic));
      }
      f1r[ncoef - 1] -= (2.0 * zr[0] * inv);
      f2r[ncoef - 1] -= (2.0 * zi[0] * inv);
    } else { /* sngl_upack_coef_sum_fftw3d_threads :1958-1990 */
      for (int i = 0; i < ncoef - 1; i++) {
        f1r[i] -= 4.0 * zr[s->map[i]] * inv;
        f1i[i] -= 4.0 * zi[s->map[i]] * inv;
      }
      f1r[ncoef - 1] -= 2.0 * zr[0] * inv;
    }
  }
  free(zr); free(zi);
  /* kinetic: cp-energy-ee-rho-stodft.c:308-320 */
  for (int is = 0; is < nstate; is++) {
    size_t o = (size_t)is * ncoef;
    for (int i = 0; i < ncoef - 1; i++) {
      fcre[o + i] -= 2.0 * s->ak2[i] * cre[o + i];
      fcim[o + i] -= 2.0 * s->ak2[i] * cim[o + i];
    }
    fcim[o + ncoef - 1] = 0.0;
  }
}

/* ------------------------------------------------------------------------ */
/* normHCheby (stodft/normh.c:182-344), normHNewtonHerm (:35-176)           */
/* ------------------------------------------------------------------------ */
void oracle_normh_cheby(const oracle_sys *s, int nstate, int ipoly, int cpy, double scale, double emean, double *cre,
                        double *cim, double *wf1re, double *wf1im, double *fcre, double *fcim) {
  const int ncoef = s->ncoef;
  const size_t tot = (size_t)nstate * ncoef;
  double prefact = -scale * emean, scale1 = -scale * 0.25, scale2 = -scale * 0.5;
  oracle_hpsi(s, nstate, cre, cim, fcre, fcim, NULL);
  if (ipoly == 1) {
    for (int is = 0; is < nstate; is++) {
      size_t o = (size_t)is * ncoef;
      for (int i = 0; i < ncoef - 1; i++) {
        fcre[o + i] = scale1 * fcre[o + i] + prefact * cre[o + i];
        fcim[o + i] = scale1 * fcim[o + i] + prefact * cim[o + i];
      }
      fcre[o + ncoef - 1] = scale2 * fcre[o + ncoef - 1] + prefact * cre[o + ncoef - 1];
    }
    if (cpy) { memcpy(cre, fcre, tot * 8); memcpy(cim, fcim, tot * 8); }
  } else {
    scale1 *= 2.0; scale2 *= 2.0; prefact *= 2.0;
    for (int is = 0; is < nstate; is++) {
      size_t o = (size_t)is * ncoef;
      for (int i = 0; i < ncoef - 1; i++) {
        fcre[o + i] = scale1 * fcre[o + i] + prefact * cre[o + i] - wf1re[o + i];
        fcim[o + i] = scale1 * fcim[o + i] + prefact * cim[o + i] - wf1im[o + i];
      }
      fcre[o + ncoef - 1] = scale2 * fcre[o + ncoef - 1] + prefact * cre[o + ncoef - 1] - wf1re[o + ncoef - 1];
    }
    if (cpy) {
      memcpy(wf1re, cre, tot * 8); memcpy(wf1im, cim, tot * 8);
      memcpy(cre, fcre, tot * 8); memcpy(cim, fcim, tot * 8);
    }
  }
}

void oracle_normh_newton(const oracle_sys *s, int nstate, double scale, double emean, double zn, double *cre,
                         double *cim, double *fcre, double *fcim) {
  const int ncoef = s->ncoef;
  const size_t tot = (size_t)nstate * ncoef;
  double prefact = -scale * emean - zn, scale1 = -scale * 0.25, scale2 = -scale * 0.5;
  oracle_hpsi(s, nstate, cre, cim, fcre, fcim, NULL);
  for (int is = 0; is < nstate; is++) {
    size_t o = (size_t)is * ncoef;
    for (int i = 0; i < ncoef - 1; i++) { fcre[o + i] *= scale1; fcim[o + i] *= scale1; }
    fcre[o + ncoef - 1] *= scale2;
  }
  for (size_t i = 0; i < tot; i++) { fcre[i] += prefact * cre[i]; fcim[i] += prefact * cim[i]; }
  memcpy(cre, fcre, tot * 8);
  memcpy(cim, fcim, tot * 8);
}

/* ------------------------------------------------------------------------ */
/* filterChebyPolyHerm (stodft/filter.c:318-706), filterNewtonPolyHerm (:33-312)
 * sto_re/sto_im: [nmu][nstate*ncoef]; moments (nullable): [L+1]          */
/* ------------------------------------------------------------------------ */
static double wdot(int ncoef, const double *ar, const double *ai, const double *br, const double *bi) {
  double d1 = 0.0, d2 = 0.0;
  for (int i = 0; i < ncoef; i++) { d1 += ar[i] * br[i]; d2 += ai[i] * bi[i]; }
  return 2.0 * d1 + 2.0 * d2 - ar[ncoef - 1] * br[ncoef - 1];
}

void oracle_filter_cheby(const oracle_sys *s, int nstate, const double *chire, const double *chiim, int L, int nmu,
                         const double *ec, double scale, double emean, double *sto_re, double *sto_im,
                         double *moments) {
  const int ncoef = s->ncoef;
  const size_t tot = (size_t)nstate * ncoef;
  double *cre = malloc(tot * 8), *cim = malloc(tot * 8), *w1r = malloc(tot * 8), *w1i = malloc(tot * 8);
  double *fr = malloc(tot * 8), *fi = malloc(tot * 8);
  memcpy(cre, chire, tot * 8); memcpy(cim, chiim, tot * 8);
  if (moments) {
    for (int k = 0; k <= L; k++) moments[k] = 0.0;
    for (int is = 0; is < nstate; is++) {
      size_t o = (size_t)is * ncoef;
      moments[0] += wdot(ncoef, chire + o, chiim + o, chire + o, chiim + o);
    }
  }
  for (int imu = 0; imu < nmu; imu++)
    for (size_t i = 0; i < tot; i++) {
      sto_re[imu * tot + i] = ec[imu] * cre[i];
      sto_im[imu * tot + i] = ec[imu] * cim[i];
    }
  memcpy(w1r, cre, tot * 8); memcpy(w1i, cim, tot * 8);
  for (int k = 1; k < L; k++) {
    oracle_normh_cheby(s, nstate, k, 1, scale, emean, cre, cim, w1r, w1i, fr, fi);
    if (moments)
      for (int is = 0; is < nstate; is++) {
        size_t o = (size_t)is * ncoef;
        moments[k] += wdot(ncoef, chire + o, chiim + o, cre + o, cim + o);
      }
    for (int imu = 0; imu < nmu; imu++) {
      double a = ec[k * nmu + imu];
      for (size_t i = 0; i < tot; i++) { sto_re[imu * tot + i] += a * cre[i]; sto_im[imu * tot + i] += a * cim[i]; }
    }
  }
  free(cre); free(cim); free(w1r); free(w1i); free(fr); free(fi);
}

void oracle_filter_newton(const oracle_sys *s, int nstate, const double *chire, const double *chiim, int L, int nmu,
                          const double *ec, const double *samp, double scale, double emean, double *sto_re,
                          double *sto_im) {
  const size_t tot = (size_t)nstate * s->ncoef;
  double *cre = malloc(tot * 8), *cim = malloc(tot * 8), *fr = malloc(tot * 8), *fi = malloc(tot * 8);
  memcpy(cre, chire, tot * 8); memcpy(cim, chiim, tot * 8);
  for (int imu = 0; imu < nmu; imu++)
    for (size_t i = 0; i < tot; i++) { sto_re[imu * tot + i] = ec[imu] * cre[i]; sto_im[imu * tot + i] = ec[imu] * cim[i]; }
  for (int k = 1; k < L; k++) {
    oracle_normh_newton(s, nstate, scale, emean, samp[k - 1], cre, cim, fr, fi);
    for (int imu = 0; imu < nmu; imu++) {
      double a = ec[k * nmu + imu];
      for (size_t i = 0; i < tot; i++) { sto_re[imu * tot + i] += a * cre[i]; sto_im[imu * tot + i] += a * cim[i]; }
    }
  }
  free(cre); free(cim); free(fr); free(fi);
}

/* ------------------------------------------------------------------------ */
/* calcChebyMoments (stodft/calc-chempot-chebyshev.c:596-912) on given chi  */
/* ------------------------------------------------------------------------ */
void oracle_cheby_moments(const oracle_sys *s, int nstate, const double *chire, const double *chiim, int L,
                          double scale, double emean, double *m) {
  const int ncoef = s->ncoef;
  const size_t tot = (size_t)nstate * ncoef;
  const int M = (L % 2 == 0) ? (L / 2 + 1) : ((L + 1) / 2);
  double *cre = malloc(tot * 8), *cim = malloc(tot * 8), *w1r = malloc(tot * 8), *w1i = malloc(tot * 8);
  double *fr = malloc(tot * 8), *fi = malloc(tot * 8);
  memcpy(cre, chire, tot * 8); memcpy(cim, chiim, tot * 8);
  memcpy(w1r, chire, tot * 8); memcpy(w1i, chiim, tot * 8);
  for (int k = 0; k <= L; k++) m[k] = 0.0;
  for (int is = 0; is < nstate; is++) {
    size_t o = (size_t)is * ncoef;
    m[0] += wdot(ncoef, chire + o, chiim + o, chire + o, chiim + o);
  }
  oracle_normh_cheby(s, nstate, 1, 0, scale, emean, cre, cim, w1r, w1i, fr, fi);
  for (int is = 0; is < nstate; is++) {
    size_t o = (size_t)is * ncoef;
    m[1] += wdot(ncoef, chire + o, chiim + o, fr + o, fi + o);
  }
  memcpy(cre, fr, tot * 8); memcpy(cim, fi, tot * 8);
  for (int n = 2; n < M; n++) {
    m[n] = 0.0; m[2 * n] = 0.0; m[2 * n - 1] = 0.0;
    oracle_normh_cheby(s, nstate, n, 0, scale, emean, cre, cim, w1r, w1i, fr, fi);
    for (int is = 0; is < nstate; is++) {
      size_t o = (size_t)is * ncoef;
      m[n] += wdot(ncoef, chire + o, chiim + o, fr + o, fi + o);
      m[2 * n - 1] += wdot(ncoef, fr + o, fi + o, cre + o, cim + o);
      m[2 * n] += wdot(ncoef, fr + o, fi + o, fr + o, fi + o);
    }
    m[2 * n] = 2.0 * m[2 * n] - m[0];
    m[2 * n - 1] = 2.0 * m[2 * n - 1] - m[1];
    memcpy(w1r, cre, tot * 8); memcpy(w1i, cim, tot * 8);
    memcpy(cre, fr, tot * 8); memcpy(cim, fi, tot * 8);
  }
  free(cre); free(cim); free(w1r); free(w1i); free(fr); free(fi);
}

/* ------------------------------------------------------------------------ */
/* rhoCalcRealStoHybrid (stodft/density.c:43-275): pack pairs, G -> r with
 * exp(+iGr) (FFTW_BACKWARD plans of the generic package,
 * mathlib/fft_create_package.c:1768-1810), sum_rho (fft_package.c:2502).
 * Output in package layout, a fastest.                                     */
/* ------------------------------------------------------------------------ */
void oracle_density(const oracle_sys *s, int nstate, const double *cre, const double *cim, double *rho) {
  const int ncoef = s->ncoef, N = s->N, n1 = s->n1, n2 = s->n2, n3 = s->n3;
  double *zr = malloc(sizeof(double) * N), *zi = malloc(sizeof(double) * N);
  memset(rho, 0, sizeof(double) * N);
  for (int is = 0; is < nstate; is += 2) {
    int pair = (is + 1 < nstate);
    const double *c1r = cre + (size_t)is * ncoef, *c1i = cim + (size_t)is * ncoef;
    const double *c2r = pair ? cre + (size_t)(is + 1) * ncoef : NULL, *c2i = pair ? cim + (size_t)(is + 1) * ncoef : NULL;
    memset(zr, 0, sizeof(double) * N);
    memset(zi, 0, sizeof(double) * N);
    for (int i = 0; i < ncoef - 1; i++) {
      double a = c1r[i], b = c1i[i], c = pair ? c2r[i] : 0.0, d = pair ? c2i[i] : 0.0;
      zr[s->map[i]] = a - d; zi[s->map[i]] = b + c;
      zr[s->mapc[i]] = a + d; zi[s->mapc[i]] = -b + c;
    }
    zr[0] = c1r[ncoef - 1];
    zi[0] = pair ? c2r[ncoef - 1] : c1i[ncoef - 1];
    fft3d(zr, zi, n1, n2, n3, +1);
    for (int a = 0; a < n1; a++)
      for (int b = 0; b < n2; b++)
        for (int c = 0; c < n3; c++) {
          long f = ((long)a * n2 + b) * n3 + c;
          long p = a + (long)n1 * (b + (long)n2 * c);
          rho[p] += zr[f] * zr[f] + zi[f] * zi[f];
        }
  }
  free(zr); free(zi);
}

/* ------------------------------------------------------------------------ */
/* Random numbers: DURAND (mathlib/blas_wrappers.f:39-69), ran_essl
 * (mathlib/mathlib.c:30-58), gaussran2 (mathlib/mathlib.c:118-165)         */
/* ------------------------------------------------------------------------ */
static double durand1(double *seed) {
  const double XM = 16807.0, XMP = 16807.0000078263692557811737060546875, SCALEU = 2147483648.0,
               SCALED = 4.656612873077392578125e-10, ONEPEP = 1.0000000004656612873077392578125,
               ONEMEP = 0.9999999995343387126922607421875;
  double t = (*seed) * SCALED;
  double s = trunc(t * XMP);
  t = t * XM;
  t = t - s * ONEMEP;
  double x = t * ONEPEP;
  *seed = t * SCALEU;
  return x;
}
double oracle_ran_essl(double *q) {
  if (*q < 1.0 || *q > 2147483646.0) *q = (sin(*q) + 1.0) * 2147483644.0 * 0.5 + 1.0;
  return durand1(q);
}
void oracle_gaussran2(int nran, double *q, double *gauss) {
  double twopi = 2.0 * M_PI, rad2 = sqrt(2.0);
  int loop = nran / 2;
  for (int i = 0; i < loop; i++) {
    double r = oracle_ran_essl(q);
    r = r > 1e-30 ? r : 1e-30;
    r = r < 1.0 ? r : 1.0;
    double phi = oracle_ran_essl(q);
    double al = sqrt(-log(r)) * rad2, arg = twopi * phi;
    gauss[2 * i] = al * cos(arg);
    gauss[2 * i + 1] = al * sin(arg);
  }
  if (nran % 2 != 0) {
    double r = oracle_ran_essl(q);
    r = r > 1e-30 ? r : 1e-30;
    r = r < 1.0 ? r : 1.0;
    double phi = oracle_ran_essl(q);
    double arg = twopi * phi, al = sqrt(-log(r)) * rad2;
    gauss[nran - 1] = al * cos(arg);
  }
}

/* genNoiseOrbitalReal (stodft/gen-noise.c:162-374), one state rank:
 * seeds (:219-234), +-sqrt(N) field in package layout (:297-302), r -> G
 * with exp(-iGr) and 1/N (generic bck_to_g, mathlib/fft_package.c:1098-1500),
 * sngl_upack_coef_sum (:1883-1915), scale 0.25 / 0.5 (:303-314).        */
void oracle_noise(const oracle_sys *s, int nstate, double seed, int np_states, int myid, double *cre, double *cim) {
  const int ncoef = s->ncoef, N = s->N, n1 = s->n1, n2 = s->n2, n3 = s->n3;
  double *seeds = malloc(sizeof(double) * (np_states + 1));
  double q = seed;
  oracle_gaussran2(np_states, &q, seeds);
  for (int p = 0; p < np_states; p++) {
    double x = seeds[p] * seeds[p];
    seeds[p] = (x >= 1.0) ? x * 100.0 : 100.0 / x;
  }
  double qn = seeds[myid];
  double *rnd = malloc(sizeof(double) * (size_t)nstate * N);
  oracle_gaussran2(nstate * N, &qn, rnd);
  double rv = sqrt((double)N);
  double *zr = malloc(sizeof(double) * N), *zi = malloc(sizeof(double) * N);
  memset(cre, 0, sizeof(double) * nstate * ncoef);
  memset(cim, 0, sizeof(double) * nstate * ncoef);
  for (int is = 0; is < nstate; is++) {
    for (int a = 0; a < n1; a++)
      for (int b = 0; b < n2; b++)
        for (int c = 0; c < n3; c++) {
          long f = ((long)a * n2 + b) * n3 + c, p = a + (long)n1 * (b + (long)n2 * c);
          zr[f] = rnd[(size_t)is * N + p] < 0.0 ? -rv : rv;
          zi[f] = 0.0;
        }
    fft3d(zr, zi, n1, n2, n3, -1);
    size_t o = (size_t)is * ncoef;
    for (int i = 0; i < ncoef - 1; i++) {
      cre[o + i] -= 4.0 * zr[s->map[i]] / N;
      cim[o + i] -= 4.0 * zi[s->map[i]] / N;
    }
    cre[o + ncoef - 1] -= 2.0 * zr[0] / N;
    for (int i = 0; i < ncoef - 1; i++) { cre[o + i] *= 0.25; cim[o + i] *= 0.25; }
    cre[o + ncoef - 1] *= 0.5;
    cim[o + ncoef - 1] = 0.0;
  }
  free(seeds); free(rnd); free(zr); free(zi);
}

/* ------------------------------------------------------------------------ */
/* Coefficients: roundFFT (stodft/coeff.c:1556-1603), calcChebyCoeff
 * (:1093-1223, funFlag 1/2), genSampNewtonHermit (:423-529),
 * genCoeffNewtonHermit (:199-290, SQRTFERMI)                               */
/* ------------------------------------------------------------------------ */
int oracle_round_fft(int n) {
  double ln2 = log(2.0), ln3 = log(3.0), lnn = log(n);
  int nmax = (int)(lnn / ln2) + 1;
  double mn = fabs(pow(2.0, nmax) - n);
  int a = nmax, b = 0;
  for (int i = 0; i < nmax; i++) {
    double x = fmax((lnn - i * ln2) / ln3, 0.0);
    int mnow = (int)(x) + 1;
    double diff = fabs(pow(2.0, i) * pow(3.0, mnow) - n);
    if (diff < mn) { b = mnow; a = i; mn = diff; }
  }
  int out = 1;
  for (int i = 0; i < a; i++) out *= 2;
  for (int i = 0; i < b; i++) out *= 3;
  return out;
}

void oracle_cheby_coeff(int L, int ngrid, double ediff, double emean, double beta, double mu, int fun, double *c) {
  double ed = ediff * 0.5, pre = 2.0 * M_PI;
  double *fr = malloc(sizeof(double) * ngrid), *fi = calloc(ngrid, sizeof(double));
  for (int j = 0; j < ngrid; j++) {
    double x = ed * cos(pre * (double)j / (double)ngrid) + emean;
    double v = 1.0 / (1.0 + exp(beta * (x - mu)));
    fr[j] = (fun == 2) ? sqrt(v) : v;
  }
  fft1d(fr, fi, ngrid, 1, -1);
  for (int k = 1; k < L; k++) c[k] = 2.0 * fr[k] / (double)ngrid;
  c[0] = fr[0] / (double)ngrid;
  free(fr); free(fi);
}

void oracle_newton_samp(int L, double smin, double smax, double scale, double emin, double *samp, double *unscale) {
  int nc = 32 * L;
  double delta = (smax - smin) / (double)(nc - 1);
  double *cand = malloc(sizeof(double) * nc), *obj = malloc(sizeof(double) * nc);
  for (int i = 0; i < nc; i++) cand[i] = smin + i * delta;
  samp[0] = cand[0];
  for (int i = 0; i < nc; i++) {
    double d = cand[i] - samp[0];
    d = d * d;
    obj[i] = d < 1.0e-20 ? -1.0e30 : log(d);
  }
  for (int p = 1; p < L; p++) {
    double om = -100000.0;
    int im = 0;
    for (int i = 0; i < nc; i++)
      if (obj[i] > om) { om = obj[i]; im = i; }
    samp[p] = cand[im];
    for (int i = 0; i < nc; i++) {
      double d = cand[i] - samp[p];
      d = d * d;
      if (d < 1.0e-20) obj[i] += -1.0e30; else obj[i] += log(d);
    }
  }
  for (int p = 0; p < L; p++) unscale[p] = (samp[p] - smin) * (1.0 / scale) + emin;
  free(cand); free(obj);
}

void oracle_newton_coeff(int L, int nmu, const double *mu, double beta, const double *samp, const double *unscale,
                         double *ec) {
  for (int im = 0; im < nmu; im++) {
    double f = sqrt(1.0 / (1.0 + exp(beta * (unscale[0] - mu[im]))));
    ec[im] = f;
    f = sqrt(1.0 / (1.0 + exp(beta * (unscale[1] - mu[im]))));
    ec[nmu + im] = (f - ec[im]) / (samp[1] - samp[0]);
    for (int p = 2; p < L; p++) {
      f = sqrt(1.0 / (1.0 + exp(beta * (unscale[p] - mu[im]))));
      double sum = f - ec[im], prod = 1.0;
      for (int q = 1; q < p; q++) {
        prod *= (samp[p] - samp[q - 1]);
        sum -= ec[q * nmu + im] * prod;
      }
      prod *= (samp[p] - samp[p - 1]);
      ec[p * nmu + im] = sum / prod;
    }
  }
}
