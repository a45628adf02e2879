/* sdft_oracle.h -- CPU oracle of the stochastic-DFT filter path.
 * TEST INFRASTRUCTURE ONLY (checker for tests/, smoke() and bench.py's
 * CPU baseline); the product library never calls it. */
#ifndef SDFT_ORACLE_H
#define SDFT_ORACLE_H
typedef struct oracle_sys oracle_sys;
int oracle_gvec(const double *hmat, double ecut, const int *kmax, int cap, int *ka, int *kb, int *kc, int *ib1,
                int *ib2);
oracle_sys *oracle_create(int n1, int n2, int n3, int ncoef, const int *ka, const int *kb, const int *kc,
                          const int *ib1, const int *ib2, const double *hmat);
void oracle_destroy(oracle_sys *s);
void oracle_set_vks(oracle_sys *s, const double *v);
void oracle_set_kinetic_cap(oracle_sys *s, double gcut);
void oracle_set_kb(oracle_sys *s, int natm, const double *pos, const int *type, int ntype, int lmax,
                   const int *lmax_type, int nsplin, double gmin, double dg, const double *vps,
                   const double *vpsnorm, const double *gzvps0);
/* KB nonlocal atomic forces f[natm*3] and energy of nstate orbitals (raw sums) */
void oracle_nl_force(const oracle_sys *s, int nstate, const double *cre, const double *cim, double *f, double *enl);
void oracle_hpsi(const oracle_sys *s, int nstate, const double *cre, const double *cim, double *fcre, double *fcim,
                 double *enl);
void oracle_normh_cheby(const oracle_sys *s, int nstate, int ipoly, int cpy, double scale, double emean, double *cre,
                        double *cim, double *wf1re, double *wf1im, double *fcre, double *fcim);
void oracle_normh_newton(const oracle_sys *s, int nstate, double scale, double emean, double zn, double *cre,
                         double *cim, double *fcre, double *fcim);
void oracle_filter_cheby(const oracle_sys *s, int nstate, const double *chire, const double *chiim, int L, int nmu,
                         const double *ec, double scale, double emean, double *sto_re, double *sto_im,
                         double *moments);
void oracle_filter_newton(const oracle_sys *s, int nstate, const double *chire, const double *chiim, int L, int nmu,
                          const double *ec, const double *samp, double scale, double emean, double *sto_re,
                          double *sto_im);
void oracle_cheby_moments(const oracle_sys *s, int nstate, const double *chire, const double *chiim, int L,
                          double scale, double emean, double *m);
void oracle_density(const oracle_sys *s, int nstate, const double *cre, const double *cim, double *rho);
double oracle_ran_essl(double *q);
void oracle_gaussran2(int nran, double *q, double *gauss);
void oracle_noise(const oracle_sys *s, int nstate, double seed, int np_states, int myid, double *cre, double *cim);
int oracle_round_fft(int n);
void oracle_cheby_coeff(int L, int ngrid, double ediff, double emean, double beta, double mu, int fun, double *c);
void oracle_newton_samp(int L, double smin, double smax, double scale, double emin, double *samp, double *unscale);
void oracle_newton_coeff(int L, int nmu, const double *mu, double beta, const double *samp, const double *unscale,
                         double *ec);
#endif
