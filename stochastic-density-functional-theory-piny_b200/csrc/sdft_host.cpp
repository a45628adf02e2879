// sdft_host.cpp -- host-side FP64 pieces of the stochastic-DFT filter path:
// G-sphere generation and grid maps, kinetic table, Chebyshev / Newton
// expansion coefficients, chemical-potential bisection, and the reference's
// uniform/Gaussian random number chain used for noise orbitals.
//
// Compiled with -ffp-contract=off so that every floating-point step is the
// plain IEEE operation the reference C performs (no fused multiply-add).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <complex>
#include <algorithm>
#include "sdft_internal.h"

namespace sdft {

// ---------------------------------------------------------------------------
// G vectors.  Same scan as setkvec3d_sm (interface/cp_ewald/set_cp_ewald.c:
// 685-833): ka = 0..kamax; kb from the first in-sphere value of
// -kmax..0 (>= 0 when ka == 0) up to the last in-sphere value; kc likewise
// (>= 1 when ka == kb == 0).  Cutoff 0.5|G|^2 <= ecut with
// G_x = 2pi*(ka*hi[0] + kb*hi[1] + kc*hi[2]) etc. (hi = PINY hmati, 0-based).
// ---------------------------------------------------------------------------
static inline double g2_of(const double *hi, double a, double b, double c) {
  const double tpi = 2.0 * M_PI;
  double xk = (a * hi[0] + b * hi[1] + c * hi[2]) * tpi;
  double yk = (a * hi[3] + b * hi[4] + c * hi[5]) * tpi;
  double zk = (a * hi[6] + b * hi[7] + c * hi[8]) * tpi;
  return xk * xk + yk * yk + zk * zk;
}

// PINY hmat / hmati are column-major with 1-based index (i,j) -> 1+(i-1)+3(j-1).
// hmati[1],hmati[2],hmati[3] used with (aka,akb,akc) for xk => the x
// component uses entries 0,1,2 of the 0-based array, i.e. column 1 of hmati
// (h^-1_{11}, h^-1_{21}, h^-1_{31}).
void invert_cell(const double *h, double *hi) {
  // h, hi: 0-based PINY column-major arrays of 9.
  auto H = [&](int i, int j) { return h[i + 3 * j]; };
  double det = H(0, 0) * (H(1, 1) * H(2, 2) - H(1, 2) * H(2, 1)) -
               H(0, 1) * (H(1, 0) * H(2, 2) - H(1, 2) * H(2, 0)) +
               H(0, 2) * (H(1, 0) * H(2, 1) - H(1, 1) * H(2, 0));
  double inv[3][3];
  inv[0][0] = (H(1, 1) * H(2, 2) - H(1, 2) * H(2, 1)) / det;
  inv[0][1] = (H(0, 2) * H(2, 1) - H(0, 1) * H(2, 2)) / det;
  inv[0][2] = (H(0, 1) * H(1, 2) - H(0, 2) * H(1, 1)) / det;
  inv[1][0] = (H(1, 2) * H(2, 0) - H(1, 0) * H(2, 2)) / det;
  inv[1][1] = (H(0, 0) * H(2, 2) - H(0, 2) * H(2, 0)) / det;
  inv[1][2] = (H(0, 2) * H(1, 0) - H(0, 0) * H(1, 2)) / det;
  inv[2][0] = (H(1, 0) * H(2, 1) - H(1, 1) * H(2, 0)) / det;
  inv[2][1] = (H(0, 1) * H(2, 0) - H(0, 0) * H(2, 1)) / det;
  inv[2][2] = (H(0, 0) * H(1, 1) - H(0, 1) * H(1, 0)) / det;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) hi[i + 3 * j] = inv[i][j];
}

double cell_volume(const double *h) {
  auto H = [&](int i, int j) { return h[i + 3 * j]; };
  return std::fabs(H(0, 0) * (H(1, 1) * H(2, 2) - H(1, 2) * H(2, 1)) -
                   H(0, 1) * (H(1, 0) * H(2, 2) - H(1, 2) * H(2, 0)) +
                   H(0, 2) * (H(1, 0) * H(2, 1) - H(1, 1) * H(2, 0)));
}

// Scan of setkvec3d_sm.  When out arrays are null only counts.
static int gvec_scan(const double *hmat, double ecut, const int *kmax, int *ka_o,
                     int *kb_o, int *kc_o, int *ib1, int *ib2) {
  double hi[9];
  invert_cell(hmat, hi);
  int i, icount = 0;
  for (i = 1; i <= kmax[0]; ++i) {
    if (g2_of(hi, (double)i, 0.0, 0.0) * 0.5 > ecut) break;
  }
  int kamax = i - 1;
  for (int ka = 0; ka <= kamax; ++ka) {
    double aka = ka;
    int kbmin = -kmax[1];
    if (ka == 0) kbmin = 0;
    for (i = kbmin; i <= 0; ++i)
      if (g2_of(hi, aka, (double)i, 0.0) * 0.5 <= ecut) break;
    kbmin = i;
    for (i = 1; i <= kmax[1]; ++i)
      if (g2_of(hi, aka, (double)i, 0.0) * 0.5 > ecut) break;
    int kbmax = i - 1;
    for (int kb = kbmin; kb <= kbmax; ++kb) {
      double akb = kb;
      int kcmin = -kmax[2];
      if (ka == 0 && kb == 0) kcmin = 1;
      for (i = kcmin; i <= 0; ++i)
        if (g2_of(hi, aka, akb, (double)i) * 0.5 <= ecut) break;
      kcmin = i;
      for (i = 1; i <= kmax[2]; ++i)
        if (g2_of(hi, aka, akb, (double)i) * 0.5 > ecut) break;
      int kcmax = i - 1;
      for (int kc = kcmin; kc <= kcmax; ++kc) {
        if (ka_o) {
          ka_o[icount] = ka;
          kb_o[icount] = kb;
          kc_o[icount] = kc;
          ib1[icount] = (kc == kcmin) ? 1 : 0;
          ib2[icount] = (kc < kcmax) ? 1 : 0;
        }
        ++icount;
      }
    }
  }
  return icount;
}

}  // namespace sdft

using namespace sdft;

extern "C" int sdft_gvec_count(const double *hmat, double ecut, const int *kmax, int *nktot) {
  if (!hmat || !kmax || !nktot || ecut <= 0.0) return set_error(SDFT_ERR_ARG, "gvec_count: bad argument");
  *nktot = gvec_scan(hmat, ecut, kmax, nullptr, nullptr, nullptr, nullptr, nullptr);
  return SDFT_OK;
}

extern "C" int sdft_gvec_fill(const double *hmat, double ecut, const int *kmax, int nktot,
                              int *ka, int *kb, int *kc, int *ibreak1, int *ibreak2) {
  if (!hmat || !kmax || !ka || !kb || !kc) return set_error(SDFT_ERR_ARG, "gvec_fill: null");
  int n = gvec_scan(hmat, ecut, kmax, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (n != nktot) return set_error(SDFT_ERR_ARG, "gvec_fill: nktot mismatch");
  std::vector<int> b1(nktot + 1), b2(nktot + 1);
  gvec_scan(hmat, ecut, kmax, ka, kb, kc, b1.data(), b2.data());
  ka[nktot] = kb[nktot] = kc[nktot] = 0;  // G = 0 stored last
  if (ibreak1) std::memcpy(ibreak1, b1.data(), sizeof(int) * nktot);
  if (ibreak2) std::memcpy(ibreak2, b2.data(), sizeof(int) * nktot);
  return SDFT_OK;
}

// setfft_indx (mathlib/fft_create_package.c:981-1020) gives 1-based
// interleaved-double indices; the filter maps are (idx-1)/2, i.e. the
// complex index ((ka mod n1)*n2 + (kb mod n2))*n3 + (kc mod n3).  The G=0
// entry (last) maps to 0 for both (fft_create_package.c:241-247).
extern "C" int sdft_fft_maps(int n1, int n2, int n3, int ncoef, const int *ka, const int *kb,
                             const int *kc, int *map, int *mapc) {
  if (n1 <= 0 || n2 <= 0 || n3 <= 0 || ncoef <= 0 || !ka || !map || !mapc)
    return set_error(SDFT_ERR_ARG, "fft_maps: bad argument");
  auto wrap = [](int k, int n) { return k < 0 ? k + n : k; };
  for (int i = 0; i < ncoef - 1; i++) {
    map[i] = (wrap(ka[i], n1) * n2 + wrap(kb[i], n2)) * n3 + wrap(kc[i], n3);
    mapc[i] = (wrap(-ka[i], n1) * n2 + wrap(-kb[i], n2)) * n3 + wrap(-kc[i], n3);
  }
  map[ncoef - 1] = 0;
  mapc[ncoef - 1] = 0;  // (mapConFFTW = 0 -> (0-1)/2 = 0 in C integer division)
  return SDFT_OK;
}

extern "C" int sdft_ak2_kinetic(const double *hmat, int ncoef, const int *ka, const int *kb,
                                const int *kc, double gcut, double *ak2) {
  if (!hmat || !ka || !ak2 || ncoef <= 0) return set_error(SDFT_ERR_ARG, "ak2: bad argument");
  double hi[9];
  invert_cell(hmat, hi);
  double gcut2 = (gcut > 0.0) ? gcut * gcut : 1.0e30;
  for (int i = 0; i < ncoef - 1; i++) {
    double g2 = g2_of(hi, (double)ka[i], (double)kb[i], (double)kc[i]);
    ak2[i] = (g2 > gcut2) ? gcut2 : g2;
  }
  ak2[ncoef - 1] = 0.0;
  return SDFT_OK;
}

// ---------------------------------------------------------------------------
// Random numbers.  DURAND (mathlib/blas_wrappers.f:39-69) is the
// Park-Miller multiplicative generator x <- 16807 x mod (2^31-1) evaluated
// in double precision with the constants below; ran_essl
// (mathlib/mathlib.c:30-58) reseeds out-of-range seeds; gaussran2
// (mathlib/mathlib.c:118-165) is Box-Muller on pairs of uniforms.
// ---------------------------------------------------------------------------
namespace sdft {
static const double kXM = 16807.0;
static const double kXMP = 16807.0000078263692557811737060546875;  // 16807*(1+2^-31)
static const double kScaleU = 2147483648.0;                        // 2^31
static const double kScaleD = 4.656612873077392578125e-10;        // 2^-31
static const double kOnePEp = 1.0000000004656612873077392578125;   // 1+2^-31
static const double kOneMEp = 0.9999999995343387126922607421875;   // 1-2^-31

double ran_uniform(double *qseed) {
  if (*qseed < 1.0 || *qseed > 2147483646.0)
    *qseed = (std::sin(*qseed) + 1.0) * 2147483644.0 * 0.5 + 1.0;
  double t = (*qseed) * kScaleD;
  double s = std::trunc(t * kXMP);
  t = t * kXM;
  t = t - s * kOneMEp;
  double x = t * kOnePEp;
  *qseed = t * kScaleU;
  return x;
}

void gaussran2(int nran, double *qseed, double *gauss) {
  const double twopi = 2.0 * M_PI;
  const double rad2 = std::sqrt(2.0);
  int loop = nran / 2;
  for (int i = 0; i < loop; i++) {
    double r = ran_uniform(qseed);
    r = std::max(r, 1e-30);
    r = std::min(r, 1.0);
    double phi = ran_uniform(qseed);
    double al = std::sqrt(-std::log(r)) * rad2;
    double arg = twopi * phi;
    gauss[2 * i] = al * std::cos(arg);
    gauss[2 * i + 1] = al * std::sin(arg);
  }
  if (nran % 2 != 0) {
    double r = ran_uniform(qseed);
    r = std::max(r, 1e-30);
    r = std::min(r, 1.0);
    double phi = ran_uniform(qseed);
    double arg = twopi * phi;
    double al = std::sqrt(-std::log(r)) * rad2;
    gauss[nran - 1] = al * std::cos(arg);
  }
}

// Per-rank seeds of genNoiseOrbitalReal (stodft/gen-noise.c:219-234).
void noise_rank_seeds(double seed, int np_states, double *out) {
  gaussran2(np_states, &seed, out);
  for (int i = 0; i < np_states; i++) {
    double x = out[i] * out[i];
    out[i] = (x >= 1.0) ? x * 100.0 : 100.0 / x;
  }
}

// Signs of gaussran2(nran, seed) without forming the Gaussian: the value is
// al*cos(2 pi phi) (even slots) or al*sin(2 pi phi) (odd slots) with al >= 0,
// so "value < 0" is decided by the trig factor unless al == 0 (r == 1), in
// which case the value is +0 (not negative).  The trig sign is evaluated
// with the same libm calls as the Gaussian path, so the result matches it
// exactly; only sqrt/log are skipped.  neg[i] = 1 if value < 0.
// cos(2 pi phi) < 0 and sin(2 pi phi) < 0 for the uniform phi in (0, 1):
// away from the zero crossings (phi = 1/4, 1/2, 3/4, 1) by more than 1e-9 the
// sign is decided by comparing phi (the argument 2 pi phi is formed to
// ~1e-16, so libm cannot disagree there); within the margin the same libm
// call as the Gaussian path decides, so the result is identical to it.
static inline bool cos_neg(double phi, double arg) {
  const double d = 1e-9;
  if (phi > 0.25 + d && phi < 0.75 - d) return true;
  if (phi < 0.25 - d || (phi > 0.75 + d && phi < 1.0 - d)) return false;
  return std::cos(arg) < 0.0;
}
static inline bool sin_neg(double phi, double arg) {
  const double d = 1e-9;
  if (phi > 0.5 + d && phi < 1.0 - d) return true;
  if (phi > d && phi < 0.5 - d) return false;
  return std::sin(arg) < 0.0;
}

// One Box-Muller pair of gauss_signs: two draws from *qseed, the signs of
// the cos and sin slots into b[0], b[1] (b[1] only when `both`).
static inline void sign_pair(double *qseed, unsigned char *b, bool both) {
  const double twopi = 2.0 * M_PI;
  double r = ran_uniform(qseed);
  r = std::max(r, 1e-30);
  r = std::min(r, 1.0);
  double phi = ran_uniform(qseed);
  double arg = twopi * phi;
  bool zero_al = (r == 1.0);
  b[0] = (!zero_al && cos_neg(phi, arg)) ? 1 : 0;
  if (both) b[1] = (!zero_al && sin_neg(phi, arg)) ? 1 : 0;
}

void gauss_signs(long long nran, double *qseed, unsigned char *neg) {
  const long long npairs = (nran + 1) / 2;
  for (long long i = 0; i < npairs; i++) sign_pair(qseed, neg + 2 * i, 2 * i + 1 < nran);
}

bool durand_on_lattice(double q) {
  const double s = q * 128.0;
  return q >= 1.0 && q <= 2147483646.0 && s == std::floor(s);
}

long long gauss_signs_to_lattice(long long nran, long long p, long long pend, double *qseed, unsigned char *out) {
  long long i = p;
  while (i < pend) {
    sign_pair(qseed, out + 2 * (i - p), 2 * i + 1 < nran);
    ++i;
    if (durand_on_lattice(*qseed)) break;
  }
  return i;
}

void gauss_signs_from_phi(double phi, unsigned char *b) {
  const double arg = 2.0 * M_PI * phi;
  b[0] = cos_neg(phi, arg) ? 1 : 0;
  b[1] = sin_neg(phi, arg) ? 1 : 0;
}
}  // namespace sdft

extern "C" int sdft_gaussran2(int nran, double *qseed, double *gauss) {
  if (nran < 0 || !qseed || (nran > 0 && !gauss)) return set_error(SDFT_ERR_ARG, "gaussran2: bad argument");
  gaussran2(nran, qseed, gauss);
  return SDFT_OK;
}

// ---------------------------------------------------------------------------
// Polynomial coefficients.
// ---------------------------------------------------------------------------

// roundFFT (stodft/coeff.c:1556-1603): 2^n 3^m closest to numGridIn.
extern "C" int sdft_round_fft(int num_grid_in) {
  if (num_grid_in <= 0) return 1;
  double ln2 = std::log(2.0), ln3 = std::log(3.0), lnn = std::log((double)num_grid_in);
  int nmax = (int)(lnn / ln2) + 1;
  double mn = std::fabs(std::pow(2.0, nmax) - num_grid_in);
  int n = nmax, m = 0;
  for (int i = 0; i < nmax; i++) {
    double x = std::fmax((lnn - i * ln2) / ln3, 0.0);
    int mnow = (int)(x) + 1;
    double diff = std::fabs(std::pow(2.0, i) * std::pow(3.0, mnow) - num_grid_in);
    if (diff < mn) {
      m = mnow;
      n = i;
      mn = diff;
    }
  }
  int out = 1;
  for (int i = 0; i < n; i++) out *= 2;
  for (int i = 0; i < m; i++) out *= 3;
  return out;
}

namespace sdft {
// In-place mixed radix (2,3) complex FFT, forward sign exp(-2 pi i jk/N),
// recursive decimation in time.  N must be 2^a 3^b.
static void fft_rec(std::complex<double> *x, int n, int stride, std::complex<double> *out,
                    const std::vector<std::complex<double>> &tw, int twstride) {
  if (n == 1) {
    out[0] = x[0];
    return;
  }
  int r = (n % 3 == 0) ? 3 : 2;
  int m = n / r;
  std::vector<std::complex<double>> sub(n);
  for (int q = 0; q < r; q++) fft_rec(x + q * stride, m, stride * r, sub.data() + q * m, tw, twstride * r);
  for (int k = 0; k < m; k++) {
    std::complex<double> v[3];
    for (int q = 0; q < r; q++) v[q] = sub[q * m + k] * tw[(size_t)q * k * twstride];
    if (r == 2) {
      out[k] = v[0] + v[1];
      out[k + m] = v[0] - v[1];
    } else {
      const std::complex<double> w1 = tw[(size_t)m * twstride];      // exp(-2pi i/3)
      const std::complex<double> w2 = tw[(size_t)2 * m * twstride];  // exp(-4pi i/3)
      out[k] = v[0] + v[1] + v[2];
      out[k + m] = v[0] + w1 * v[1] + w2 * v[2];
      out[k + 2 * m] = v[0] + w2 * v[1] + w1 * v[2];
    }
  }
}

void fft_forward_1d(std::vector<std::complex<double>> &x) {
  int n = (int)x.size();
  std::vector<std::complex<double>> tw(n);
  for (int t = 0; t < n; t++) tw[t] = std::polar(1.0, -2.0 * M_PI * t / n);
  std::vector<std::complex<double>> out(n);
  fft_rec(x.data(), n, 1, out.data(), tw, 1);
  x.swap(out);
}

static inline double fermi_exp(double x, double mu, double beta) {
  return 1.0 / (1.0 + std::exp(beta * (x - mu)));  // fermiExpReal mathlib/mathlib.c:781
}

// calcChebyCoeff (stodft/coeff.c:1093-1223) for funFlag 1 (F) and 2 (sqrt F).
int cheby_coeff(int L, int ngrid, double energy_diff, double energy_mean, double beta,
                double chem_pot, int fun_flag, double *coeffs) {
  double ed = energy_diff * 0.5;
  double pre = 2.0 * M_PI;
  std::vector<std::complex<double>> f(ngrid);
  for (int j = 0; j < ngrid; j++) {
    double x = ed * std::cos(pre * (double)j / (double)ngrid) + energy_mean;
    double v = fermi_exp(x, chem_pot, beta);
    f[j] = (fun_flag == 2) ? std::sqrt(v) : v;
  }
  fft_forward_1d(f);
  for (int k = 1; k < L; k++) coeffs[k] = 2.0 * f[k].real() / (double)ngrid;
  coeffs[0] = f[0].real() / (double)ngrid;
  return 0;
}

double num_elec_cheby(int L, int ngrid, double energy_diff, double energy_mean, double beta,
                      double chem_pot, double occ, const double *moments) {
  std::vector<double> c(L);
  cheby_coeff(L, ngrid, energy_diff, energy_mean, beta, chem_pot, 1, c.data());
  double s = 0.0;
  for (int k = 0; k < L; k++) s += c[k] * moments[k];
  return s * occ;
}
}  // namespace sdft

extern "C" int sdft_cheby_coeff(int L, int num_cheby_grid, double energy_diff, double energy_mean,
                                double beta, double chem_pot, int fun_flag, double *coeffs) {
  if (L <= 0 || num_cheby_grid < L || !coeffs || (fun_flag != 1 && fun_flag != 2))
    return set_error(SDFT_ERR_ARG, "cheby_coeff: bad argument");
  int n = num_cheby_grid;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  if (n != 1) return set_error(SDFT_ERR_ARG, "cheby_coeff: grid must be 2^a 3^b");
  cheby_coeff(L, num_cheby_grid, energy_diff, energy_mean, beta, chem_pot, fun_flag, coeffs);
  return SDFT_OK;
}

extern "C" double sdft_num_elec_cheby(int L, int num_cheby_grid, double energy_diff,
                                      double energy_mean, double beta, double chem_pot, double occ,
                                      const double *moments) {
  return num_elec_cheby(L, num_cheby_grid, energy_diff, energy_mean, beta, chem_pot, occ, moments);
}

// Bisection of calcChemPotCheby (stodft/calc-chempot-chebyshev.c:212-251):
// bracket [mu0-gap/2, mu0+gap/2], widen by gap until it brackets Ne, one
// secant step, then halve until |N - Ne| <= 1e-11 Ne.
extern "C" int sdft_chempot_cheby(int L, double energy_diff, double energy_mean, double beta,
                                  double occ, const double *moments, double num_elec_true,
                                  double chem_pot_init, double gap_init, double *chem_pot,
                                  double *num_elec) {
  if (L <= 0 || !moments || !chem_pot || gap_init <= 0.0) return set_error(SDFT_ERR_ARG, "chempot: bad argument");
  int ngrid = sdft_round_fft(L * 32);
  double tol = 1.0e-11 * num_elec_true;
  auto N = [&](double mu) { return num_elec_cheby(L, ngrid, energy_diff, energy_mean, beta, mu, occ, moments); };
  double mumin = chem_pot_init - gap_init * 0.5, mumax = chem_pot_init + gap_init * 0.5;
  double nmin = N(mumin), nmax = N(mumax);
  int guard = 0;
  while (nmax < num_elec_true && guard++ < 10000) {
    mumin = mumax;
    mumax += gap_init;
    nmin = N(mumin);
    nmax = N(mumax);
  }
  while (nmin > num_elec_true && guard++ < 20000) {
    mumax = mumin;
    mumin -= gap_init;
    nmin = N(mumin);
    nmax = N(mumax);
  }
  double munew = (num_elec_true - nmin) * (mumax - mumin) / (nmax - nmin) + mumin;
  double nnew = N(munew);
  int it = 0;
  while (std::fabs(nnew - num_elec_true) > tol && it++ < 2000) {
    if (nnew > num_elec_true) { mumax = munew; nmax = nnew; }
    if (nnew < num_elec_true) { mumin = munew; nmin = nnew; }
    munew = 0.5 * (mumin + mumax);
    nnew = N(munew);
  }
  *chem_pot = munew;
  if (num_elec) *num_elec = nnew;
  if (std::fabs(nnew - num_elec_true) > tol) return set_error(SDFT_ERR_ARG, "chempot: bisection did not converge");
  return SDFT_OK;
}

// genSampNewtonHermit (stodft/coeff.c:423-529): greedy Leja-type points from
// 32L equispaced candidates on [smin,smax]; first maximum wins.
extern "C" int sdft_newton_samp(int L, double smin, double smax, double scale, double energy_min,
                                double *samp, double *samp_unscale) {
  if (L < 2 || !samp || !samp_unscale || scale == 0.0) return set_error(SDFT_ERR_ARG, "newton_samp: bad argument");
  int ncand = 32 * L;
  double delta = (smax - smin) / (double)(ncand - 1);
  std::vector<double> cand(ncand), obj(ncand);
  for (int i = 0; i < ncand; i++) cand[i] = smin + i * delta;
  samp[0] = cand[0];
  for (int i = 0; i < ncand; i++) {
    double d = cand[i] - samp[0];
    d = d * d;
    obj[i] = (d < 1.0e-20) ? -1.0e30 : std::log(d);
  }
  for (int ip = 1; ip < L; ip++) {
    double omax = -100000.0;
    int imax = 0;
    for (int i = 0; i < ncand; i++)
      if (obj[i] > omax) { omax = obj[i]; imax = i; }
    samp[ip] = cand[imax];
    for (int i = 0; i < ncand; i++) {
      double d = cand[i] - samp[ip];
      d = d * d;
      if (d < 1.0e-20) obj[i] += -1.0e30;
      else obj[i] += std::log(d);
    }
  }
  double inv = 1.0 / scale;
  for (int ip = 0; ip < L; ip++) samp_unscale[ip] = (samp[ip] - smin) * inv + energy_min;
  return SDFT_OK;
}

// genCoeffNewtonHermit (stodft/coeff.c:199-290, energy window off, SQRTFERMI):
// divided differences of sqrt(F) on the Newton points.
extern "C" int sdft_newton_coeff(int L, int num_chem_pot, const double *chem_pot, double beta,
                                 const double *samp, const double *samp_unscale, double *ec) {
  if (L < 2 || num_chem_pot < 1 || !chem_pot || !samp || !samp_unscale || !ec)
    return set_error(SDFT_ERR_ARG, "newton_coeff: bad argument");
  for (int imu = 0; imu < num_chem_pot; imu++) {
    double f = std::sqrt(fermi_exp(samp_unscale[0], chem_pot[imu], beta));
    ec[imu] = f;
    f = std::sqrt(fermi_exp(samp_unscale[1], chem_pot[imu], beta));
    ec[num_chem_pot + imu] = (f - ec[imu]) / (samp[1] - samp[0]);
    for (int ip = 2; ip < L; ip++) {
      f = std::sqrt(fermi_exp(samp_unscale[ip], chem_pot[imu], beta));
      double sum = f - ec[imu], prod = 1.0;
      for (int jp = 1; jp < ip; jp++) {
        prod *= (samp[ip] - samp[jp - 1]);
        sum -= ec[jp * num_chem_pot + imu] * prod;
      }
      prod *= (samp[ip] - samp[ip - 1]);
      ec[ip * num_chem_pot + imu] = sum / prod;
    }
  }
  return SDFT_OK;
}
