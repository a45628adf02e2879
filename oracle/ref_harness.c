/*
 * ref_harness.c -- drives the reference's OWN hot-path C sources (compiled
 * from the read-only reference tree by oracle/build_ref.sh into
 * oracle/_ref/libpinyref.so).  TEST INFRASTRUCTURE ONLY: used by
 * tests/test_oracle_pin.py to pin the CPU restatement (sdft_oracle.c).
 *
 * What is the reference's code: setkvec3d_sm, calcCoefForceWrapSCF and
 * everything below it (KB projection / energy / back projection, the
 * filter-path FFT wrappers, cp_vpsi, kinetic term), normHCheby,
 * normHNewtonHerm, filterChebyPolyHerm, filterNewtonPolyHerm,
 * calcChebyMoments, calcChebyCoeff, genSampNewtonHermit,
 * genCoeffNewtonHermit, gaussran2/ran_essl.
 * What this file supplies: the PINY data structures filled for one
 * single-rank, spin-unpolarised system with one atom type and one radial
 * KB projector per l channel; single-rank MPI wrappers; BLAS ddot/daxpy;
 * an FP64 DFT behind the FFTW3 API subset the sources call (FFTW is not
 * installed here); DURAND (Fortran, no Fortran compiler here) restated from
 * mathlib/blas_wrappers.f:39-69; abort stubs for routines off this path.
 */
#include "standard_include.h"
#include "../typ_defs/typedefs_gen.h"
#include "../typ_defs/typedefs_class.h"
#include "../typ_defs/typedefs_bnd.h"
#include "../typ_defs/typedefs_cp.h"
#include <time.h>
#include <unistd.h>

/* reference prototypes used here */
void create_para_fft_pkg3d(PARA_FFT_PKG3D *, int *, int *, int *, int);
void para_fft_gen3d_init(PARA_FFT_PKG3D *);
void ref_genNoiseOrbitalReal(CP *, CPCOEFFS_POS *);
void rhoCalcRealStoHybrid(CPSCR *, CPCOEFFS_INFO *, CELL *, STODFTINFO *, double *, double *, double *, int, int,
                          int, int, int, COMMUNICATE *, PARA_FFT_PKG3D *, PARA_FFT_PKG3D *, PARA_FFT_PKG3D *,
                          PARA_FFT_PKG3D *, PARA_FFT_PKG3D *);
void setkvec3d_sm(int, double, int *, double *, int *, int *, int *, int *, int *, double *, double *);
void calcCoefForceWrapSCF(CLASS *, GENERAL_DATA *, CP *, CPCOEFFS_POS *, CLATOMS_POS *);
void normHCheby(CP *, CLASS *, GENERAL_DATA *, CPCOEFFS_POS *, CLATOMS_POS *, int, int);
void normHNewtonHerm(CP *, CLASS *, GENERAL_DATA *, CPCOEFFS_POS *, CLATOMS_POS *, double);
void filterChebyPolyHerm(CP *, CLASS *, GENERAL_DATA *, int);
void filterNewtonPolyHerm(CP *, CLASS *, GENERAL_DATA *, int);
void calcChebyMoments(CP *, CLASS *, GENERAL_DATA *, int);
void calcChemPotCheby(CP *, CLASS *, GENERAL_DATA *, int);
double calcNumElecCheby(CP *, double, double *);
void countkvec3d(int *, double, int *, double *);
void setkvec3d(int, double, int *, double *, int *, int *, int *, int *, int *, int, double *, double *, double *);
void controlEwdLocPreScf(CLATOMS_INFO *, CLATOMS_POS *, CELL *, PTENS *, EWALD *, CPEWALD *, CPSCR *, PSEUDO *,
                         EWD_SCR *, CPOPTS *, ATOMMAPS *, double *, double *, COMMUNICATE *, FOR_SCR *, int, int);
void calcRhoStoRecipFullg(CPEWALD *, CPSCR *, CPCOEFFS_INFO *, EWALD *, CELL *, double *, double *, double *,
                          double *, double *, double *, double *, double *, double *, int, int, int, COMMUNICATE *,
                          PARA_FFT_PKG3D *, PARA_FFT_PKG3D *);
void control_ewd_loc(CLATOMS_INFO *, CLATOMS_POS *, CELL *, PTENS *, EWALD *, CPEWALD *, CPSCR *, PSEUDO *, EWD_SCR *,
                     CPOPTS *, ATOMMAPS *, double *, double *, COMMUNICATE *, FOR_SCR *, int, int);
void ewald3d_selfbgr_cp(CLATOMS_INFO *, EWALD *, PTENS *, double, double *, double *, int);
double getdeth(double *);
void spline_vdv(double, double, double *, double *, int, double *, double *, double, double, double, double, double,
                double, double, double, double, double, double, double, int, int, int, double, int, double, double,
                double);
void cpGetVksStodft(CPOPTS *, CPSCR *, CPEWALD *, EWALD *, COMMUNICATE *, CP_COMM_STATE_PKG *, CP_COMM_STATE_PKG *,
                    STAT_AVG *, double *, CELL *, char *, double *, double, double, int, int, int, int, int, int,
                    PARA_FFT_PKG3D *, PARA_FFT_PKG3D *, PARA_FFT_PKG3D *, PARA_FFT_PKG3D *, int);
void calcChebyCoeff(STODFTINFO *, STODFTCOEFPOS *, double *, double *, int, double);
void genSampNewtonHermit(STODFTINFO *, STODFTCOEFPOS *);
void genCoeffNewtonHermit(STODFTINFO *, STODFTCOEFPOS *);
int roundFFT(int);
void gaussran2(int, int *, int *, double *, double[]);
double fermiExpReal(double, double, double);

/* ====================================================================== */
/* FFTW3 subset: plain O(N^2)-per-dimension-free mixed radix DFT         */
/* ====================================================================== */
struct sdft_fftw_plan_s {
  int rank, n[3], howmany, istride, idist, sign;
  fftw_complex *in, *out;
};

static void dft1(fftw_complex *x, int n, long st, int sign, fftw_complex *tmp) {
  /* recursive mixed radix on a gathered copy */
  for (int j = 0; j < n; j++) tmp[j] = x[j * st];
  /* iterative: naive for small factors via recursion helper */
  fftw_complex *y = tmp + n;
  /* decimation: use simple recursive function */
  extern void sdft_ref_fft_rec(const fftw_complex *, int, int, fftw_complex *, int, fftw_complex *);
  sdft_ref_fft_rec(tmp, n, 1, y, sign, y + n);
  for (int j = 0; j < n; j++) x[j * st] = y[j];
}

void sdft_ref_fft_rec(const fftw_complex *x, int n, int stride, fftw_complex *y, int sign, fftw_complex *scr) {
  if (n == 1) { y[0] = x[0]; return; }
  int r = (n % 3 == 0) ? 3 : ((n % 2 == 0) ? 2 : n);
  int m = n / r;
  fftw_complex *sub = scr, *nscr = scr + n;
  for (int q = 0; q < r; q++) sdft_ref_fft_rec(x + q * stride, m, stride * r, sub + q * m, sign, nscr);
  for (int k = 0; k < m; k++) {
    fftw_complex v[8];
    for (int q = 0; q < r; q++) v[q] = sub[q * m + k] * cexp(sign * 2.0 * M_PI * I * (double)(q * k) / n);
    for (int t = 0; t < r; t++) {
      fftw_complex a = 0;
      for (int q = 0; q < r; q++) a += v[q] * cexp(sign * 2.0 * M_PI * I * (double)(q * t) / r);
      y[k + t * m] = a;
    }
  }
}

static fftw_plan mkplan(int rank, const int *n, int howmany, fftw_complex *in, int istride, int idist,
                        fftw_complex *out, int sign) {
  fftw_plan p = calloc(1, sizeof(*p));
  p->rank = rank;
  for (int i = 0; i < rank; i++) p->n[i] = n[i];
  p->howmany = howmany; p->istride = istride; p->idist = idist; p->sign = sign; p->in = in; p->out = out;
  return p;
}
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned f) {
  int n[3] = {n0, n1, n2};
  (void)f;
  return mkplan(3, n, 1, in, 1, 0, out, sign);
}
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned f) {
  (void)f;
  return mkplan(1, &n, 1, in, 1, n, out, sign);
}
fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *ie, int is, int id,
                             fftw_complex *out, const int *oe, int os, int od, int sign, unsigned f) {
  (void)ie; (void)oe; (void)os; (void)od; (void)f;
  return mkplan(rank, n, howmany, in, is, id, out, sign);
}
static void exec(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
  int nmax = 1;
  for (int i = 0; i < p->rank; i++) nmax = p->n[i] > nmax ? p->n[i] : nmax;
  fftw_complex *tmp = malloc(sizeof(fftw_complex) * nmax * 16);
  if (p->rank == 3) {
    int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    long N = (long)n0 * n1 * n2;
    if (out != in) memcpy(out, in, sizeof(fftw_complex) * N);
    for (long a = 0; a < (long)n0 * n1; a++) dft1(out + a * n2, n2, 1, p->sign, tmp);
    for (int a = 0; a < n0; a++)
      for (int c = 0; c < n2; c++) dft1(out + (long)a * n1 * n2 + c, n1, n2, p->sign, tmp);
    for (long bc = 0; bc < (long)n1 * n2; bc++) dft1(out + bc, n0, (long)n1 * n2, p->sign, tmp);
  } else {
    int n = p->n[0];
    for (int h = 0; h < p->howmany; h++) {
      /* many_dft with data given as interleaved doubles through the reference's
         1-based zfft pointers: in == out in every call on this path */
      fftw_complex *b = out + (long)h * p->idist;
      if (out != in) memcpy(b, in + (long)h * p->idist, sizeof(fftw_complex) * n);  /* contiguous only */
      dft1(b, n, p->istride, p->sign, tmp);
    }
  }
  free(tmp);
}
void fftw_execute(const fftw_plan p) { exec(p, p->in, p->out); }
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) { exec(p, in, out); }
void fftw_destroy_plan(fftw_plan p) { free(p); }
void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int n) { (void)n; }
void fftw_cleanup_threads(void) {}

/* ====================================================================== */
/* OpenMP / MKL / MPI single-rank stand-ins                              */
/* ====================================================================== */
double omp_get_wtime(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}
void omp_set_num_threads(int n) { (void)n; }
int omp_get_thread_num(void) { return 0; }
int omp_get_num_threads(void) { return 1; }
int omp_get_max_threads(void) { return 1; }
void omp_set_max_active_levels(int n) { (void)n; }
void mkl_set_num_threads(int n) { (void)n; }
void mkl_set_dynamic(int n) { (void)n; }

static void sdft_ref_abort(const char *f) {
  fprintf(stderr, "reference harness: off-path routine %s called\n", f);
  abort();
}
#define ABORT_STUB(name) \
  void name(void) { sdft_ref_abort(#name); }
ABORT_STUB(Allgather) ABORT_STUB(Allgatherv) ABORT_STUB(Allreduce) ABORT_STUB(Alltoall) ABORT_STUB(Alltoallv)
ABORT_STUB(Finalize) ABORT_STUB(Gatherv) ABORT_STUB(Reduce) ABORT_STUB(Reduce_scatter) ABORT_STUB(Scatterv)
ABORT_STUB(Bcast) ABORT_STUB(Send) ABORT_STUB(Recv) ABORT_STUB(DGEMV) ABORT_STUB(DSYMV) ABORT_STUB(dsysv_) ABORT_STUB(rs_)
ABORT_STUB(calcChemPotInterp) ABORT_STUB(coef_force_calc_hybrid_threads_state)
ABORT_STUB(coef_force_tau_fun_full_g) ABORT_STUB(coef_force_tau_fun_hybrid)
ABORT_STUB(controlEnergyNlppRealThreads) ABORT_STUB(controlPotentialEnergyFilter) ABORT_STUB(control_contract_rho)
ABORT_STUB(control_grad_rho) ABORT_STUB(control_nonloc_gh) ABORT_STUB(control_spread_rho)
ABORT_STUB(cp_condiag_ksmat) ABORT_STUB(cp_rotate_vector) ABORT_STUB(dcfftb_generic_) ABORT_STUB(dcfftf_generic_)
ABORT_STUB(dcffti_generic_) 

ABORT_STUB(getnl_fcoef_gh) ABORT_STUB(getnl_pot_pv_fatm_gh) ABORT_STUB(grad_corr_lda) ABORT_STUB(grad_corr_lsda)
ABORT_STUB(cfopen)
void Barrier(int c) { (void)c; }

/* BLAS level-1 used by the filter/moment code (mathlib/mathlib.c:518-570) */
double ddot_(int *n, double *x, int *incx, double *y, int *incy) {
  double s = 0.0;
  for (int i = 0; i < *n; i++) s += x[i * *incx] * y[i * *incy];
  return s;
}
void daxpy_(int *n, double *a, double *x, int *incx, double *y, int *incy) {
  for (int i = 0; i < *n; i++) y[i * *incy] += *a * x[i * *incx];
}
/* DURAND, mathlib/blas_wrappers.f:39-69 (Park-Miller in FP64) */
void durand_(double *seed, int *n, double *x, int *ierr) {
  const double XM = 16807.0, XMP = 16807.0000078263692557811737060546875, SCALEU = 2147483648.0,
               SCALED = 4.656612873077392578125e-10, ONEPEP = 1.0000000004656612873077392578125,
               ONEMEP = 0.9999999995343387126922607421875;
  *ierr = 0;
  if (*n < 0 || *seed < 1.0 || *seed > 2147483646.0) { *ierr = 1; return; }
  double t = *seed * SCALED;
  for (int j = 0; j < *n; j++) {
    double s = trunc(t * XMP);
    t = t * XM;
    t = t - s * ONEMEP;
    x[j] = t * ONEPEP;
  }
  *seed = t * SCALEU;
}

/* ====================================================================== */
/* PINY data structures for one system                                    */
/* ====================================================================== */
typedef struct {
  CP cp;
  CLASS cls;
  GENERAL_DATA gd;
  CPCOEFFS_POS cpos;
  CLATOMS_POS apos;
  STODFTINFO sinfo;
  STODFTCOEFPOS scoef;
  NEWTONINFO newton;
  CHEBYSHEVINFO cheby;
  int ncoef, N, nmax, natm;
  fftw_complex *fin, *fout, *bin, *bout;
  fftw_plan pfwd, pbwd;
  fftw_complex *fin_arr[1], *fout_arr[1], *bin_arr[1], *bout_arr[1];
  fftw_plan pfwd_arr[1], pbwd_arr[1];
} RefSys;

static double *d1(long n) { return (double *)calloc(n + 2, sizeof(double)); }  /* 1-based ready */
static int *i1(long n) { return (int *)calloc(n + 2, sizeof(int)); }

RefSys *ref_create(int n1, int n2, int n3, int ncoef, const int *ka, const int *kb, const int *kc, const int *ib1,
                   const int *ib2, const double *hmat, const double *vks, int natm, const double *pos, int nsplin,
                   double gmin, double dg, const double *vps /*[2][4][nsplin]*/, const double *vpsnorm /*[2]*/,
                   double gzvps0, int nmax) {
  RefSys *r = calloc(1, sizeof(RefSys));
  CP *cp = &r->cp;
  CLASS *cl = &r->cls;
  GENERAL_DATA *gd = &r->gd;
  const int N = n1 * n2 * n3, nk = ncoef - 1;
  r->ncoef = ncoef; r->N = N; r->nmax = nmax; r->natm = natm;
  /* cell: hmat / hmati 1-based column-major; CP box = full box */
  CELL *cell = &gd->cell;
  double hi[9];
  {
    const double *h = hmat;
    double det = h[0] * (h[4] * h[8] - h[7] * h[5]) - h[3] * (h[1] * h[8] - h[7] * h[2]) + h[6] * (h[1] * h[5] - h[4] * h[2]);
    hi[0] = (h[4] * h[8] - h[5] * h[7]) / det; hi[3] = (h[5] * h[6] - h[3] * h[8]) / det; hi[6] = (h[3] * h[7] - h[4] * h[6]) / det;
    hi[1] = (h[7] * h[2] - h[1] * h[8]) / det; hi[4] = (h[0] * h[8] - h[2] * h[6]) / det; hi[7] = (h[1] * h[6] - h[0] * h[7]) / det;
    hi[2] = (h[1] * h[5] - h[2] * h[4]) / det; hi[5] = (h[2] * h[3] - h[0] * h[5]) / det; hi[8] = (h[0] * h[4] - h[1] * h[3]) / det;
  }
  cell->hmat = d1(9); cell->hmati = d1(9); cell->hmat_cp = d1(9); cell->hmati_cp = d1(9);
  for (int i = 0; i < 9; i++) {
    cell->hmat[i + 1] = cell->hmat_cp[i + 1] = hmat[i];
    cell->hmati[i + 1] = cell->hmati_cp[i + 1] = hi[i];
  }
  cell->cp_box_center = d1(3); cell->cp_box_center_rel = d1(3);
  cell->iperd = 3;
  gd->ptens.pvten_tmp = d1(9);
  /* options / info */
  cp->cpopts.cp_lsda = 0; cp->cpopts.cp_dual_grid_opt = 0; cp->cpopts.cp_ptens_calc = 0; cp->cpopts.cp_hess_calc = 0;
  cp->cpcoeffs_info.ncoef = ncoef;
  cp->cpcoeffs_info.nstate_up_proc = nmax; cp->cpcoeffs_info.nstate_up = nmax;
  cp->communicate.myid_state = 0; cp->communicate.np_states = 1; cp->communicate.numThreads = 1;
  cp->communicate.np_forc = 1;
  /* coefficients */
  r->cpos.cre_up = d1((long)nmax * ncoef); r->cpos.cim_up = d1((long)nmax * ncoef);
  r->cpos.fcre_up = d1((long)nmax * ncoef); r->cpos.fcim_up = d1((long)nmax * ncoef);
  r->cpos.icoef_orth_up = 1;
  cp->cpcoeffs_pos = &r->cpos;
  cl->clatoms_pos = &r->apos;
  /* k vectors (1-based) */
  CPEWALD *ew = &cp->cpewald;
  ew->nktot_sm = nk;
  ew->kastr_sm = i1(ncoef); ew->kbstr_sm = i1(ncoef); ew->kcstr_sm = i1(ncoef);
  ew->ibrk1_sm = i1(ncoef); ew->ibrk2_sm = i1(ncoef);
  ew->ak2_sm = d1(ncoef); ew->ak2Kinetic = d1(ncoef);
  for (int i = 0; i < ncoef; i++) {
    ew->kastr_sm[i + 1] = ka[i]; ew->kbstr_sm[i + 1] = kb[i]; ew->kcstr_sm[i + 1] = kc[i];
  }
  for (int i = 0; i < nk; i++) { ew->ibrk1_sm[i + 1] = ib1[i]; ew->ibrk2_sm[i + 1] = ib2[i]; }
  ew->fftw3dFlag = 1;
  ew->eCutoffKe = -1.0;
  {
    double tpi = 2.0 * M_PI;
    for (int i = 1; i <= nk; i++) {
      double a = ew->kastr_sm[i], b = ew->kbstr_sm[i], c = ew->kcstr_sm[i];
      double *h = cell->hmati_cp;
      double xk = (a * h[1] + b * h[2] + c * h[3]) * tpi, yk = (a * h[4] + b * h[5] + c * h[6]) * tpi,
             zk = (a * h[7] + b * h[8] + c * h[9]) * tpi;
      ew->ak2_sm[i] = ew->ak2Kinetic[i] = xk * xk + yk * yk + zk * zk; /* get_ak2_sm, no cap */
    }
  }
  /* V_KS (1-based, filter layout) */
  cp->cpscr.cpscr_rho.v_ks_up = d1(N);
  memcpy(&cp->cpscr.cpscr_rho.v_ks_up[1], vks, sizeof(double) * N);
  cp->cpscr.cpscr_wave.zfft = d1(2 * (long)N + 2);
  cp->cpscr.cpscr_wave.zfft_tmp = d1(2 * (long)N + 2);
  /* FFT package built by the reference itself (create_para_fft_pkg3d +
     para_fft_gen3d_init, mathlib/fft_create_package.c:41,1571): filter maps,
     3-D FFTW plans and the generic pencil transforms */
  PARA_FFT_PKG3D *pk = &cp->cp_sclr_fft_pkg3d_sm;
  pk->comm = 0; pk->num_proc = 1; pk->myid = 0;
  pk->nktot = nk; pk->ncoef = ncoef; pk->nkf1 = n1; pk->nkf2 = n2; pk->nkf3 = n3;
  pk->threadFlag = 2; pk->igeneric_opt = 0; pk->numThreads = 1; pk->numThreadsFFTW3 = 1;
  create_para_fft_pkg3d(pk, ew->kastr_sm, ew->kbstr_sm, ew->kcstr_sm, 0);
  para_fft_gen3d_init(pk);
  cp->cp_sclr_fft_pkg3d_lg = *pk;
  cp->cp_para_fft_pkg3d_lg.nfft = pk->nfft;
  cp->cp_para_fft_pkg3d_lg.nfft_proc = pk->nfft_proc;
  r->sinfo.fragInfo = (FRAGINFO *)calloc(1, sizeof(FRAGINFO));
  r->sinfo.randSeedTot = d1(2);
  cp->cp_para_fft_pkg3d_lg.ncoef_proc = 0;
  cp->cp_para_fft_pkg3d_dens_cp_box.ncoef_proc = 0;
  cp->cpscr.cpscr_loc.vextr = d1(1); cp->cpscr.cpscr_loc.vexti = d1(1);
  cp->cpscr.cpscr_loc.vextr_loc = d1(1); cp->cpscr.cpscr_loc.vexti_loc = d1(1);
  /* atoms + KB pseudopotential: one type, s and p, one radial projector */
  CLATOMS_INFO *ci = &cl->clatoms_info;
  ci->natm_tot = natm; ci->hess_calc = 0; ci->pi_beads = 1; ci->q = d1(natm);
  CLATOMS_POS *ap = &r->apos;
  ap->x = d1(natm); ap->y = d1(natm); ap->z = d1(natm); ap->fx = d1(natm); ap->fy = d1(natm); ap->fz = d1(natm);
  for (int i = 0; i < natm; i++) { ap->x[i + 1] = pos[3 * i]; ap->y[i + 1] = pos[3 * i + 1]; ap->z[i + 1] = pos[3 * i + 2]; }
  ATOMMAPS *am = &cl->atommaps;
  am->natm_typ = 1;
  am->iatm_atm_typ = i1(natm); am->iatm_atm_typ_nl = i1(natm); am->iatm_atm_typ_nl_rev = i1(natm);
  am->imap_atm_typ_nl = i1(2);
  for (int i = 1; i <= natm; i++) am->iatm_atm_typ[i] = am->iatm_atm_typ_nl[i] = am->iatm_atm_typ_nl_rev[i] = 1;
  am->imap_atm_typ_nl[1] = 1;
  PSEUDO *ps = &cp->pseudo;
  ps->n_ang_max = 1; ps->n_ang_max_kb = 1; ps->n_ang_max_gh = 0; ps->n_rad_max = 1; ps->natm_typ_nl = 1;
  ps->np_nl = i1(4); ps->np_nl_gh = i1(4);
  ps->np_nl[1] = natm; ps->np_nl[2] = natm;
  ps->np_nonloc_cp_box_kb = natm; ps->np_nonloc_cp_box_gh = 0;
  /* ip_nl / ip_nl_rev are indexed (ipart + l*natm) for each open l channel */
  ps->ip_nl = i1(2 * natm + 2); ps->ip_nl_rev = i1(2 * natm + 2);
  for (int i = 1; i <= natm; i++) {
    ps->ip_nl[i] = ps->ip_nl[i + natm] = i;
    ps->ip_nl_rev[i] = ps->ip_nl_rev[i + natm] = i;
  }
  ps->nrad_max_l = i1(4); ps->nrad_max_l[1] = 1; ps->nrad_max_l[2] = 1;
  ps->np_nl_rad_str = (int **)calloc(4, sizeof(int *));
  for (int l = 1; l <= 3; l++) { ps->np_nl_rad_str[l] = i1(2); ps->np_nl_rad_str[l][1] = 1; }
  ps->nsplin_g = nsplin; ps->gmin_spl = gmin; ps->dg_spl = dg;
  ps->vps0 = d1(2 * nsplin); ps->vps1 = d1(2 * nsplin); ps->vps2 = d1(2 * nsplin); ps->vps3 = d1(2 * nsplin);
  ps->dvps0 = d1(2 * nsplin); ps->dvps1 = d1(2 * nsplin); ps->dvps2 = d1(2 * nsplin); ps->dvps3 = d1(2 * nsplin);
  for (int l = 0; l < 2; l++)
    for (int i = 0; i < nsplin; i++) {
      ps->vps0[1 + l * nsplin + i] = vps[(l * 4 + 0) * nsplin + i];
      ps->vps1[1 + l * nsplin + i] = vps[(l * 4 + 1) * nsplin + i];
      ps->vps2[1 + l * nsplin + i] = vps[(l * 4 + 2) * nsplin + i];
      ps->vps3[1 + l * nsplin + i] = vps[(l * 4 + 3) * nsplin + i];
    }
  ps->vpsnorm = d1(2); ps->vpsnorm[1] = vpsnorm[0]; ps->vpsnorm[2] = vpsnorm[1];
  ps->gzvps0 = d1(1); ps->gzvps0[1] = gzvps0; ps->gzvps = d1(1);
  ps->pseudoReal.pseudoRealFlag = 0;
  /* nonlocal scratch: ntot = nstate * np_nlmax * nlm * nrad */
  long ntot = (long)nmax * natm * 4 + 2;
  CPSCR_NONLOC *nl = &cp->cpscr.cpscr_nonloc;
  nl->vnlre_up = d1(ntot); nl->vnlim_up = d1(ntot);
  nl->dvnlre_x_up = d1(ntot); nl->dvnlre_y_up = d1(ntot); nl->dvnlre_z_up = d1(ntot);
  nl->dvnlim_x_up = d1(ntot); nl->dvnlim_y_up = d1(ntot); nl->dvnlim_z_up = d1(ntot);
  EWD_SCR *es = &cl->ewd_scr;
  long na = natm + 4;
  es->cossc = d1(na); es->sinsc = d1(na); es->helr = d1(na); es->heli = d1(na); es->fx2 = d1(na); es->fy2 = d1(na);
  es->fz2 = d1(na); es->vtemp_now = d1(na); es->q = d1(na); es->x = d1(na); es->y = d1(na); es->z = d1(na);
  es->fx = d1(na); es->fy = d1(na); es->fz = d1(na); es->helr_now = d1(na); es->heli_now = d1(na); es->temp = d1(na);
  cl->for_scr.iexcl = i1(na);
  /* stochastic DFT info */
  cp->stodftInfo = &r->sinfo;
  cp->stodftCoefPos = &r->scoef;
  r->sinfo.newtonInfo = &r->newton;
  r->sinfo.chebyshevInfo = &r->cheby;
  r->sinfo.filterFlag = 1;
  r->sinfo.numThreads = 1;
  r->sinfo.fermiFunctionReal = fermiExpReal;
  r->scoef.stoWfUpRe = (double **)calloc(8, sizeof(double *));
  r->scoef.stoWfUpIm = (double **)calloc(8, sizeof(double *));
  return r;
}

void ref_destroy(RefSys *r) { (void)r; /* process-lifetime test object */ }

static void load_states(RefSys *r, int ns, const double *re, const double *im) {
  r->cp.cpcoeffs_info.nstate_up_proc = ns;
  r->cp.cpcoeffs_info.nstate_up = ns;
  memcpy(&r->cpos.cre_up[1], re, sizeof(double) * ns * r->ncoef);
  memcpy(&r->cpos.cim_up[1], im, sizeof(double) * ns * r->ncoef);
}

int ref_hpsi(RefSys *r, int ns, const double *re, const double *im, double *fre, double *fim, double *enl) {
  load_states(r, ns, re, im);
  r->gd.stat_avg.cp_enl = 0.0;
  calcCoefForceWrapSCF(&r->cls, &r->gd, &r->cp, &r->cpos, &r->apos);
  memcpy(fre, &r->cpos.fcre_up[1], sizeof(double) * ns * r->ncoef);
  memcpy(fim, &r->cpos.fcim_up[1], sizeof(double) * ns * r->ncoef);
  if (enl) *enl = r->gd.stat_avg.cp_enl;
  return 0;
}

/* KB nonlocal atomic forces and energy of the loaded states through the
 * reference's calcNlPseudoPostScf (stodft/reduced-energy/energy-wrapper-post-scf.c:224):
 * control_ewd_non_loc / get_nlmat (Z and dZ/dR) then getnl_pot_pv_fatm.
 * f[3a+d]: the raw per-atom sums, before calcEnergyForce's occ / numStateStoUp. */
void calcNlPseudoPostScf(CLASS *, GENERAL_DATA *, CP *, CPCOEFFS_POS *, CLATOMS_POS *);
int ref_nl_force(RefSys *r, int ns, const double *re, const double *im, double *f, double *enl) {
  load_states(r, ns, re, im);
  memset(&r->cpos.fcre_up[1], 0, sizeof(double) * ns * r->ncoef);
  memset(&r->cpos.fcim_up[1], 0, sizeof(double) * ns * r->ncoef);
  for (int a = 1; a <= r->natm; a++) r->apos.fx[a] = r->apos.fy[a] = r->apos.fz[a] = 0.0;
  r->gd.stat_avg.cp_enl = 0.0;
  calcNlPseudoPostScf(&r->cls, &r->gd, &r->cp, &r->cpos, &r->apos);
  for (int a = 0; a < r->natm; a++) {
    f[3 * a] = r->apos.fx[a + 1];
    f[3 * a + 1] = r->apos.fy[a + 1];
    f[3 * a + 2] = r->apos.fz[a + 1];
  }
  if (enl) *enl = r->gd.stat_avg.cp_enl;
  return 0;
}

static void set_poly(RefSys *r, int L, int nmu, const double *ec, double scale, double emean, int cheby) {
  STODFTINFO *si = &r->sinfo;
  si->polynormLength = L;
  si->numChemPot = nmu;
  si->energyMean = emean;
  si->expanType = cheby ? 1 : 2;
  r->cheby.scale = scale; r->cheby.Smin = -1.0; r->cheby.Smax = 1.0;
  r->newton.scale = scale; r->newton.Smin = -2.0; r->newton.Smax = 2.0;
  r->scoef.expanCoeff = (double *)ec;
}

int ref_filter(RefSys *r, int cheby, int ns, const double *re, const double *im, int L, int nmu, const double *ec,
               const double *samp, double scale, double emean, double *out_re, double *out_im, double *moments) {
  load_states(r, ns, re, im);
  set_poly(r, L, nmu, ec, scale, emean, cheby);
  for (int imu = 0; imu < nmu; imu++) {
    r->scoef.stoWfUpRe[imu] = d1((long)ns * r->ncoef);
    r->scoef.stoWfUpIm[imu] = d1((long)ns * r->ncoef);
  }
  if (cheby) {
    r->sinfo.storeChebyMomentsFlag = moments ? 1 : 0;
    filterChebyPolyHerm(&r->cp, &r->cls, &r->gd, 0);
    if (moments) memcpy(moments, r->scoef.chebyMomentsUp, sizeof(double) * L);
  } else {
    r->newton.sampPoint = (void *)samp;
    filterNewtonPolyHerm(&r->cp, &r->cls, &r->gd, 0);
  }
  for (int imu = 0; imu < nmu; imu++) {
    memcpy(out_re + (long)imu * ns * r->ncoef, &r->scoef.stoWfUpRe[imu][1], sizeof(double) * ns * r->ncoef);
    memcpy(out_im + (long)imu * ns * r->ncoef, &r->scoef.stoWfUpIm[imu][1], sizeof(double) * ns * r->ncoef);
    free(r->scoef.stoWfUpRe[imu]);
    free(r->scoef.stoWfUpIm[imu]);
  }
  return 0;
}

/* calcChebyMoments draws its noise through genNoiseOrbitalReal; the
 * harness supplies that routine and hands it the injected chi. */
static const double *g_inj_re, *g_inj_im;
static int g_inj_n;
void genNoiseOrbitalReal(CP *cp, CPCOEFFS_POS *pos) {
  (void)cp;
  memcpy(&pos->cre_up[1], g_inj_re, sizeof(double) * g_inj_n);
  memcpy(&pos->cim_up[1], g_inj_im, sizeof(double) * g_inj_n);
}

int ref_moments(RefSys *r, int ns, const double *re, const double *im, int L, double scale, double emean,
                double *moments) {
  load_states(r, ns, re, im);
  g_inj_re = re; g_inj_im = im; g_inj_n = ns * r->ncoef;
  set_poly(r, L, 1, NULL, scale, emean, 1);
  r->sinfo.numChebyMoments = (L % 2 == 0) ? (L / 2 + 1) : ((L + 1) / 2);
  r->scoef.chebyMomentsUp = d1(L + 1);
  calcChebyMoments(&r->cp, &r->cls, &r->gd, 0);
  memcpy(moments, r->scoef.chebyMomentsUp, sizeof(double) * (L + 1));
  return 0;
}

/* The stodftInfo fields that calcChemPotCheby and calcNumElecCheby read
 * (stodft/calc-chempot-chebyshev.c:30-95, :918-930), spin-unpolarised. */
static void set_chempot_info(RefSys *r, int ns, int L, double emin, double emax, double beta, double occ,
                             double num_elec, double chem_pot_init, double gap_init) {
  STODFTINFO *si = &r->sinfo;
  set_poly(r, L, 1, NULL, 2.0 / (emax - emin), 0.5 * (emin + emax), 1);
  si->energyDiff = emax - emin;
  si->energyMin = emin;
  si->energyMax = emax;
  si->beta = beta;
  si->occNumber = (int)occ;
  si->numElecTrue = num_elec;
  si->chemPotInit = chem_pot_init;
  si->gapInit = gap_init;
  si->numStateStoUp = ns;
  si->numStateStoDn = 0;
  si->printChebyMoment = 0;
  si->iScf = 1;
  if (!r->scoef.chemPot) r->scoef.chemPot = (double *)calloc(4, sizeof(double));
}

/* calcNumElecCheby (stodft/calc-chempot-chebyshev.c:918) at mu with the
 * moments in cp->stodftCoefPos->chebyMomentsUp: the Chebyshev grid and the
 * forward FFT plan that calcChemPotCheby sets up around it (:109-116). */
static double num_elec_with(CP *cp, int L, double mu) {
  STODFTINFO *si = cp->stodftInfo;
  STODFTCOEFPOS *sc = cp->stodftCoefPos;
  si->numChebyGrid = roundFFT(32 * L);
  sc->funValGridFFT = fftw_malloc(sizeof(fftw_complex) * si->numChebyGrid);
  sc->chebyCoeffsFFT = fftw_malloc(sizeof(fftw_complex) * si->numChebyGrid);
  si->fftwPlanForward = fftw_plan_dft_1d(si->numChebyGrid, sc->funValGridFFT, sc->chebyCoeffsFFT, FFTW_FORWARD, 0);
  double *coeffs = (double *)calloc(L, sizeof(double));
  double n = calcNumElecCheby(cp, mu, coeffs);
  free(coeffs);
  fftw_destroy_plan(si->fftwPlanForward);
  fftw_free(sc->funValGridFFT);
  fftw_free(sc->chebyCoeffsFFT);
  return n;
}

static double ref_num_elec_on(RefSys *r, int L, double mu) { return num_elec_with(&r->cp, L, mu); }

/* calcNumElecCheby on given normalised moments (moments[0..L-1] enter the
 * sum), without a system: only the fields it reads are set. */
double ref_num_elec(int L, double emin, double emax, double beta, double occ, const double *moments, double mu) {
  CP cp;
  STODFTINFO si;
  STODFTCOEFPOS sc;
  CHEBYSHEVINFO ch;
  memset(&cp, 0, sizeof cp); memset(&si, 0, sizeof si); memset(&sc, 0, sizeof sc); memset(&ch, 0, sizeof ch);
  cp.stodftInfo = &si;
  cp.stodftCoefPos = &sc;
  cp.communicate.numThreads = 1;
  si.chebyshevInfo = &ch;
  si.polynormLength = L;
  si.energyDiff = emax - emin;
  si.energyMean = 0.5 * (emin + emax);
  si.beta = beta;
  si.occNumber = (int)occ;
  si.fermiFunctionReal = fermiExpReal;
  sc.chebyMomentsUp = (double *)moments;
  return num_elec_with(&cp, L, mu);
}

/* calcChemPotCheby (stodft/calc-chempot-chebyshev.c:30) on the loaded
 * states: the routine computes their Chebyshev moments itself
 * (calcChebyMoments, whose noise call the harness answers with the injected
 * chi), divides them by numStateStoUp, brackets N(mu) = Ne from
 * chemPotInit +- gapInit/2 (widening by gapInit), takes one secant step and
 * bisects to 1e-11 Ne.  Out: chemPot[0] and N(mu) at that mu. */
int ref_chempot(RefSys *r, int ns, const double *re, const double *im, int L, double emin, double emax,
                double beta, double occ, double num_elec, double chem_pot_init, double gap_init, double *mu,
                double *ne) {
  load_states(r, ns, re, im);
  g_inj_re = re; g_inj_im = im; g_inj_n = ns * r->ncoef;
  set_chempot_info(r, ns, L, emin, emax, beta, occ, num_elec, chem_pot_init, gap_init);
  calcChemPotCheby(&r->cp, &r->cls, &r->gd, 0);
  *mu = r->scoef.chemPot[0];
  if (ne) {
    /* N(mu) through calcNumElecCheby on the routine's own normalised moments:
     * recomputed here, since calcChemPotCheby frees them */
    double *m = d1(L + 1);
    r->scoef.chebyMomentsUp = m;
    r->sinfo.numChebyMoments = (L % 2 == 0) ? (L / 2 + 1) : ((L + 1) / 2);
    calcChebyMoments(&r->cp, &r->cls, &r->gd, 0);
    for (int i = 0; i <= L; i++) m[i] /= (double)ns;
    *ne = ref_num_elec_on(r, L, *mu);
    free(m);
    r->scoef.chebyMomentsUp = NULL;
  }
  return 0;
}

/* --- host pieces ------------------------------------------------------- */
int ref_gvec(const double *hmat, double ecut, const int *kmax, int cap, int *ka, int *kb, int *kc, int *ib1, int *ib2) {
  double h[10], hi[10], gmin, gmax;
  double det = hmat[0] * (hmat[4] * hmat[8] - hmat[7] * hmat[5]) - hmat[3] * (hmat[1] * hmat[8] - hmat[7] * hmat[2]) +
               hmat[6] * (hmat[1] * hmat[5] - hmat[4] * hmat[2]);
  (void)h;
  hi[1] = (hmat[4] * hmat[8] - hmat[5] * hmat[7]) / det; hi[4] = (hmat[5] * hmat[6] - hmat[3] * hmat[8]) / det;
  hi[7] = (hmat[3] * hmat[7] - hmat[4] * hmat[6]) / det; hi[2] = (hmat[7] * hmat[2] - hmat[1] * hmat[8]) / det;
  hi[5] = (hmat[0] * hmat[8] - hmat[2] * hmat[6]) / det; hi[8] = (hmat[1] * hmat[6] - hmat[0] * hmat[7]) / det;
  hi[3] = (hmat[1] * hmat[5] - hmat[2] * hmat[4]) / det; hi[6] = (hmat[2] * hmat[3] - hmat[0] * hmat[5]) / det;
  hi[9] = (hmat[0] * hmat[4] - hmat[1] * hmat[3]) / det;
  int km[4] = {0, kmax[0], kmax[1], kmax[2]};
  int nk = cap - 1;
  int *a = i1(cap), *b = i1(cap), *c = i1(cap), *b1 = i1(cap), *b2 = i1(cap);
  setkvec3d_sm(nk, ecut, km, hi, a, b, c, b1, b2, &gmin, &gmax);
  for (int i = 0; i < cap; i++) { ka[i] = a[i + 1]; kb[i] = b[i + 1]; kc[i] = c[i + 1]; }
  for (int i = 0; i < nk; i++) { ib1[i] = b1[i + 1]; ib2[i] = b2[i + 1]; }
  free(a); free(b); free(c); free(b1); free(b2);
  return 0;
}

int ref_round_fft(int n) { return roundFFT(n); }

int ref_cheby_coeff(int L, double ediff, double emean, double beta, double mu, int fun, double *out) {
  STODFTINFO si;
  STODFTCOEFPOS sc;
  CHEBYSHEVINFO ch;
  memset(&si, 0, sizeof si); memset(&sc, 0, sizeof sc); memset(&ch, 0, sizeof ch);
  si.chebyshevInfo = &ch;
  si.polynormLength = L;
  si.energyDiff = ediff;
  si.energyMean = emean;
  si.beta = beta;
  si.fermiFunctionReal = fermiExpReal;
  si.numChebyGrid = roundFFT(32 * L);
  sc.funValGridFFT = fftw_malloc(sizeof(fftw_complex) * si.numChebyGrid);
  sc.chebyCoeffsFFT = fftw_malloc(sizeof(fftw_complex) * si.numChebyGrid);
  si.fftwPlanForward = fftw_plan_dft_1d(si.numChebyGrid, sc.funValGridFFT, sc.chebyCoeffsFFT, FFTW_FORWARD, 0);
  calcChebyCoeff(&si, &sc, &mu, out, fun, 0.0);
  fftw_destroy_plan(si.fftwPlanForward);
  fftw_free(sc.funValGridFFT); fftw_free(sc.chebyCoeffsFFT);
  return 0;
}

int ref_newton(int L, double scale, double emin, double beta, double mu, double *samp, double *unsc, double *ec) {
  STODFTINFO si;
  STODFTCOEFPOS sc;
  NEWTONINFO nw;
  memset(&si, 0, sizeof si); memset(&sc, 0, sizeof sc); memset(&nw, 0, sizeof nw);
  si.newtonInfo = &nw;
  si.polynormLength = L; si.numChemPot = 1; si.numThreads = 1; si.energyMin = emin; si.beta = beta;
  si.fermiFunctionReal = fermiExpReal;
  nw.Smin = -2.0; nw.Smax = 2.0; nw.scale = scale;
  nw.sampPoint = samp; nw.sampPointUnscale = unsc;
  sc.expanCoeff = ec;
  sc.chemPot = &mu;
  genSampNewtonHermit(&si, &sc);
  genCoeffNewtonHermit(&si, &sc);
  return 0;
}

/* genNoiseOrbitalReal (stodft/gen-noise.c:162) of the reference */
int ref_noise(RefSys *r, int ns, double seed, double *re, double *im) {
  r->cp.cpcoeffs_info.nstate_up_proc = ns;
  r->cp.cpcoeffs_info.nstate_up = ns;
  r->sinfo.randSeed = seed;
  ref_genNoiseOrbitalReal(&r->cp, &r->cpos);
  memcpy(re, &r->cpos.cre_up[1], sizeof(double) * ns * r->ncoef);
  memcpy(im, &r->cpos.cim_up[1], sizeof(double) * ns * r->ncoef);
  return 0;
}

/* The product adapter's genNoiseOrbitalReal body (present only in the
 * adapter test library) on the same structures as ref_noise. */
void sdft_piny_noise(CP *, CPCOEFFS_POS *) __attribute__((weak));
int ref_noise_adapter(RefSys *r, int ns, double seed, double *re, double *im) {
  if (!sdft_piny_noise) return -1;
  r->cp.cpcoeffs_info.nstate_up_proc = ns;
  r->cp.cpcoeffs_info.nstate_up = ns;
  r->sinfo.randSeed = seed;
  sdft_piny_noise(&r->cp, &r->cpos);
  memcpy(re, &r->cpos.cre_up[1], sizeof(double) * ns * r->ncoef);
  memcpy(im, &r->cpos.cim_up[1], sizeof(double) * ns * r->ncoef);
  return 0;
}

/* rhoCalcRealStoHybrid (stodft/density.c:43): sum_s |psi_s(r)|^2 */
int ref_density(RefSys *r, int ns, const double *re, const double *im, double *rho) {
  load_states(r, ns, re, im);
  double *rs = d1(r->N);
  CP *cp = &r->cp;
  rhoCalcRealStoHybrid(&cp->cpscr, &cp->cpcoeffs_info, &r->gd.cell, &r->sinfo, r->cpos.cre_up, r->cpos.cim_up, rs,
                       0, 1, ns, r->ncoef, 0, &cp->communicate, &cp->cp_para_fft_pkg3d_lg, &cp->cp_sclr_fft_pkg3d_lg,
                       &cp->cp_para_fft_pkg3d_dens_cp_box, &cp->cp_sclr_fft_pkg3d_dens_cp_box,
                       &cp->cp_sclr_fft_pkg3d_sm);
  memcpy(rho, &rs[1], sizeof(double) * r->N);
  free(rs);
  return 0;
}

void ref_gaussran2(int n, double *seed, double *out) {
  int is = 0;
  gaussran2(n, &is, &is, seed, out);
}

/* ====================================================================== */
/* Density mixing (stodft/diis.c: genDensityMix) and checkpoint output     */
/* (stodft/checkpointIO.c: checkpointOutput), single rank, spin-unpolarised */
/* ====================================================================== */
void genDensityMix(CP *, int);
void checkpointOutput(CP *, GENERAL_DATA *);

/* LAPACK dgesvd (A = U S V^T, column-major, square) by one-sided Jacobi
 * (Hestenes) rotations; singular values in descending order.  Project-
 * written stand-in for MKL: only diis.c's matrixInvSVD calls it. */
void dgesvd_(char *jobu, char *jobvt, int *m, int *n, double *a, int *lda, double *s, double *u, int *ldu,
             double *vt, int *ldvt, double *work, int *lwork, int *info) {
  (void)jobu; (void)jobvt; (void)work; (void)lwork;
  const int nn = *n, ld = *lda;
  *info = 0;
  if (*m != nn) { *info = -2; return; }
  double *w = malloc(sizeof(double) * nn * nn), *v = calloc((size_t)nn * nn, sizeof(double));
  for (int c = 0; c < nn; c++) {
    for (int r = 0; r < nn; r++) w[r + c * nn] = a[r + c * ld];
    v[c + c * nn] = 1.0;
  }
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int p = 0; p < nn - 1; p++)
      for (int q = p + 1; q < nn; q++) {
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int r = 0; r < nn; r++) {
          al += w[r + p * nn] * w[r + p * nn];
          be += w[r + q * nn] * w[r + q * nn];
          ga += w[r + p * nn] * w[r + q * nn];
        }
        if (ga == 0.0 || fabs(ga) <= 1e-15 * sqrt(al * be)) continue;
        off = fmax(off, fabs(ga) / sqrt(al * be));
        const double ze = (be - al) / (2.0 * ga);
        const double tt = (ze >= 0.0 ? 1.0 : -1.0) / (fabs(ze) + sqrt(1.0 + ze * ze));
        const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
        for (int r = 0; r < nn; r++) {
          const double x = w[r + p * nn], y = w[r + q * nn];
          w[r + p * nn] = cs * x - sn * y;
          w[r + q * nn] = sn * x + cs * y;
          const double vx = v[r + p * nn], vy = v[r + q * nn];
          v[r + p * nn] = cs * vx - sn * vy;
          v[r + q * nn] = sn * vx + cs * vy;
        }
      }
    if (off == 0.0) break;
  }
  int *ord = malloc(sizeof(int) * nn);
  double *sv = malloc(sizeof(double) * nn);
  for (int c = 0; c < nn; c++) {
    double t2 = 0.0;
    for (int r = 0; r < nn; r++) t2 += w[r + c * nn] * w[r + c * nn];
    sv[c] = sqrt(t2);
    ord[c] = c;
  }
  for (int i = 1; i < nn; i++)
    for (int j = i; j > 0 && sv[ord[j]] > sv[ord[j - 1]]; j--) { int x = ord[j]; ord[j] = ord[j - 1]; ord[j - 1] = x; }
  for (int k = 0; k < nn; k++) {
    const int c = ord[k];
    s[k] = sv[c];
    for (int r = 0; r < nn; r++) {
      u[r + k * *ldu] = sv[c] > 0.0 ? w[r + c * nn] / sv[c] : 0.0;
      vt[k + r * *ldvt] = v[r + c * nn];
    }
  }
  free(w); free(v); free(ord); free(sv);
}

/* BLAS dgemv: y = alpha op(A) x + beta y, column-major */
void dgemv_(char *trans, int *m, int *n, double *alpha, double *a, int *lda, double *x, int *incx, double *beta,
            double *y, int *incy) {
  const int tr = (*trans == 't' || *trans == 'T');
  const int ny = tr ? *n : *m, nx = tr ? *m : *n;
  for (int i = 0; i < ny; i++) {
    double acc = 0.0;
    for (int j = 0; j < nx; j++) acc += (tr ? a[j + i * *lda] : a[i + j * *lda]) * x[j * *incx];
    y[i * *incy] = *alpha * acc + *beta * y[i * *incy];
  }
}

typedef struct {
  CP cp;
  GENERAL_DATA gd;
  STODFTINFO si;
  STODFTCOEFPOS sp;
  double *rho1;  /* rho_up, 1-based */
  double hmat[10];
} RefMix;

RefMix *ref_mix_create(int n, int num_diis, int num_step_mix, double r_big, double r_sm, double r_sm2) {
  RefMix *m = calloc(1, sizeof(RefMix));
  m->cp.stodftInfo = &m->si;
  m->cp.stodftCoefPos = &m->sp;
  m->cp.cpopts.cp_lsda = 0;
  m->cp.communicate.myid_state = 0;
  m->cp.communicate.np_states = 1;
  m->si.rhoRealGridNum = n;
  m->si.rhoRealGridTot = n;
  m->si.numDiis = num_diis;
  m->si.numStepMix = num_step_mix;
  m->si.mixRatioBig = r_big;
  m->si.mixRatioSM = r_sm;
  m->si.mixRatioSM2 = r_sm2;
  m->sp.rhoUpCorrect = malloc(sizeof(double) * n);
  m->sp.rhoUpOld = malloc(sizeof(double) * n);
  m->sp.rhoUpBank = calloc(num_diis + 1, sizeof(double *));
  m->sp.rhoUpErr = calloc(num_diis + 1, sizeof(double *));
  m->sp.diisCoeff = calloc(num_diis + 1, sizeof(double));
  m->rho1 = calloc(n + 1, sizeof(double));
  m->cp.cpscr.cpscr_rho.rho_up = m->rho1;
  m->gd.cell.hmat_cp = m->hmat;
  return m;
}

/* one SCF step of genDensityMix: rho_out = the mixed rho_up (unchanged from
 * the previous step's value at iscf == 0, as in the reference) */
void ref_mix_step(RefMix *m, int iscf, const double *rho_correct, double *rho_out) {
  memcpy(m->sp.rhoUpCorrect, rho_correct, sizeof(double) * m->si.rhoRealGridNum);
  m->si.iScf = iscf;
  genDensityMix(&m->cp, iscf);
  memcpy(rho_out, &m->rho1[1], sizeof(double) * m->si.rhoRealGridNum);
}

void ref_mix_set_rho(RefMix *m, const double *rho) { memcpy(&m->rho1[1], rho, sizeof(double) * m->si.rhoRealGridNum); }

/* checkpointOutput into dir/density-checkpoint (the reference writes to the
 * working directory); cell = diag(l1, l2, l3) for the volume factor */
int ref_mix_checkpoint(RefMix *m, const char *dir, double l1, double l2, double l3) {
  char cwd[4096];
  if (!getcwd(cwd, sizeof cwd) || chdir(dir) != 0) return 1;
  memset(m->hmat, 0, sizeof m->hmat);
  m->hmat[1] = l1; m->hmat[5] = l2; m->hmat[9] = l3;
  checkpointOutput(&m->cp, &m->gd);
  return chdir(cwd) != 0;
}

/* ====================================================================== */
/* LDA exchange-correlation (energy/cp/xc_functionals.c): kind 1 = PZ81,  */
/* 2 = PW92; rho and vks 0-based (vks += V_xc)                            */
/* ====================================================================== */
void excpot_pz_lda(double *, double *, double *, double *, int, int, double, int, int, double *, int);
void excpot_pw_lda(double *, double *, double *, double *, int, int, double, int, int, double *, int);

void ref_xc_lda(int kind, int n, double *rho, double *vks, double vol, double *exc, double *muxc) {
  double pvten[10] = {0};
  *exc = 0.0;
  *muxc = 0.0;
  if (kind == 1) excpot_pz_lda(vks - 1, rho - 1, exc, muxc, 2 * n, 2 * n, vol, 0, 0, pvten, 0);
  else excpot_pw_lda(vks - 1, rho - 1, exc, muxc, 2 * n, 2 * n, vol, 0, 0, pvten, 0);
}

/* ====================================================================== */
/* The density side of the SCF step: vext, rho(G), V_KS                   */
/* ====================================================================== */
/* On the system's cell, atoms and grid (the reference uses one grid for the
 * wave functions and the density when cp_dual_grid_opt is 0):
 *   1. the density sphere 0.5|G|^2 <= 4 ecut by the reference's own
 *      countkvec3d / setkvec3d (interface/cp_ewald/set_cp_ewald.c:401,525),
 *      G = 0 appended last, and the FFT package on it
 *      (create_para_fft_pkg3d / para_fft_gen3d_init);
 *   2. controlEwdLocPreScf (stodft/reduced-energy/cp-energy-eext-stodft.c:35)
 *      for vext(G): the local channel is stored as the l = 2 block of the
 *      spline tables (loc_opt 2), charges zero (no charge correction);
 *   3. calcRhoStoRecipFullg (stodft/density.c:699) on rho_in (the density
 *      times the volume, package layout) and cpGetVksStodft
 *      (stodft/reduced-energy/cp-energy-ee-rho-stodft.c:644) with
 *      cp_dual_grid_opt 0, periodic, LDA (xc 1 pz_lda, 2 pw_lda).
 * The system's own V_KS array is left as it was.  Outputs (cap >= ncoef_l):
 * the sphere, vext, rho(G), V_KS in the filter layout and
 * energies = {cp_ehart, cp_eext, cp_exc, cp_muxc}. */
int ref_vks(RefSys *r, double ecut, int nsp_loc, double gmin_loc, double dg_loc,
            const double *vloc /*[4][nsp_loc]*/, double gzvps_loc, int xc,
            const double *rho_in, int cap, int *ncoef_out, int *ka, int *kb, int *kc, double *vext_re,
            double *vext_im, double *rhog_re, double *rhog_im, double *vks, double *energies,
            const double *q, double q_pseud, double alp_ewd, double *force, double *ewald_e) {
  CP *cp = &r->cp;
  CELL *cell = &r->gd.cell;
  PARA_FFT_PKG3D *sm = &cp->cp_sclr_fft_pkg3d_sm;
  const int n1 = sm->nkf1, n2 = sm->nkf2, n3 = sm->nkf3, N = n1 * n2 * n3;
  /* 1. density sphere */
  int kmaxv[4] = {0, n1, n2, n3};
  int nktot = 0;
  countkvec3d(&nktot, ecut, kmaxv, cell->hmati);
  const int ncoef = nktot + 1;
  *ncoef_out = ncoef;
  if (ncoef > cap) return 1;
  EWALD *ew = &r->gd.ewald;
  ew->nktot = nktot;
  ew->kastr = i1(ncoef); ew->kbstr = i1(ncoef); ew->kcstr = i1(ncoef);
  ew->ibrk1 = i1(ncoef); ew->ibrk2 = i1(ncoef);
  double gmin_spl, gmin_true, gmax_spl;
  setkvec3d(nktot, ecut, kmaxv, cell->hmati, ew->kastr, ew->kbstr, ew->kcstr, ew->ibrk1, ew->ibrk2, 1, &gmin_spl,
            &gmin_true, &gmax_spl);
  ew->kastr[ncoef] = ew->kbstr[ncoef] = ew->kcstr[ncoef] = 0;
  for (int i = 0; i < ncoef; i++) { ka[i] = ew->kastr[i + 1]; kb[i] = ew->kbstr[i + 1]; kc[i] = ew->kcstr[i + 1]; }
  PARA_FFT_PKG3D lg;
  memset(&lg, 0, sizeof lg);
  lg.comm = 0; lg.num_proc = 1; lg.myid = 0;
  lg.nktot = nktot; lg.ncoef = ncoef; lg.nkf1 = n1; lg.nkf2 = n2; lg.nkf3 = n3;
  lg.threadFlag = 2; lg.igeneric_opt = 0; lg.numThreads = 1; lg.numThreadsFFTW3 = 1;
  create_para_fft_pkg3d(&lg, ew->kastr, ew->kbstr, ew->kcstr, 0);
  para_fft_gen3d_init(&lg);
  /* 2. vext */
  CPEWALD *cpew = &cp->cpewald;
  double *ak2_keep = cpew->ak2;
  cpew->ak2 = d1(ncoef);
  CPSCR *scr = &cp->cpscr;
  scr->cpscr_loc.vextr = d1(ncoef); scr->cpscr_loc.vexti = d1(ncoef);
  scr->cpscr_loc.vextr_loc = d1(ncoef); scr->cpscr_loc.vexti_loc = d1(ncoef);
  scr->cpscr_loc.dvextr = d1(ncoef); scr->cpscr_loc.dvexti = d1(ncoef);
  scr->cpscr_rho.rhocr_up = d1(ncoef); scr->cpscr_rho.rhoci_up = d1(ncoef);
  PSEUDO *ps = &cp->pseudo;
  /* the spline tables of this call: the local channel's own knots (the KB
   * knots stop short of the density cutoff); the s and p blocks are not read */
  const int nsp = nsp_loc;
  const int nsp_keep = ps->nsplin_g;
  const double gmin_keep = ps->gmin_spl, dg_keep = ps->dg_spl;
  ps->nsplin_g = nsp; ps->gmin_spl = gmin_loc; ps->dg_spl = dg_loc;
  double *keep[8] = {ps->vps0, ps->vps1, ps->vps2, ps->vps3, ps->dvps0, ps->dvps1, ps->dvps2, ps->dvps3};
  const int nang_keep = ps->n_ang_max;
  double *nv[4];
  for (int d = 0; d < 4; d++) {
    nv[d] = d1(3 * nsp);
    memcpy(&nv[d][1 + 2 * nsp], vloc + (size_t)d * nsp, sizeof(double) * nsp);  /* local block (l = 2) */
  }
  ps->vps0 = nv[0]; ps->vps1 = nv[1]; ps->vps2 = nv[2]; ps->vps3 = nv[3];
  ps->dvps0 = d1(3 * nsp); ps->dvps1 = d1(3 * nsp); ps->dvps2 = d1(3 * nsp); ps->dvps3 = d1(3 * nsp);
  ps->n_ang_max = 2;
  ps->loc_opt = i1(2); ps->loc_opt[1] = 2;
  ps->q_pseud = d1(2);
  const double gz_keep = ps->gzvps[1];
  ps->gzvps[1] = gzvps_loc;
  r->cls.for_scr.index_atm = i1(4);
  r->gd.ewald.alp_ewd = 1.0;
  cp->cpopts.cp_ptens_calc = 0;
  double vrecip = 0.0, hess = 0.0;
  controlEwdLocPreScf(&r->cls.clatoms_info, &r->apos, cell, &r->gd.ptens, ew, cpew, scr, ps, &r->cls.ewd_scr,
                      &cp->cpopts, &r->cls.atommaps, &vrecip, &hess, &cp->communicate, &r->cls.for_scr, 0, 0);
  for (int i = 0; i < ncoef; i++) { vext_re[i] = scr->cpscr_loc.vextr[i + 1]; vext_im[i] = scr->cpscr_loc.vexti[i + 1]; }
  /* 3. rho(G) and V_KS */
  scr->cpscr_rho.rho_up = d1(N);
  memcpy(&scr->cpscr_rho.rho_up[1], rho_in, sizeof(double) * N);
  double *vks_keep = scr->cpscr_rho.v_ks_up;
  scr->cpscr_rho.v_ks_up = d1(N);
  CPCOEFFS_INFO *ci = &cp->cpcoeffs_info;
  ci->cp_elf_calc_frq = 0; ci->cp_laplacian_on = 0;
  calcRhoStoRecipFullg(cpew, scr, ci, ew, cell, scr->cpscr_rho.rhocr_up, scr->cpscr_rho.rhoci_up,
                       scr->cpscr_rho.rho_up, NULL, NULL, NULL, NULL, NULL, NULL, 0, 0, 1, &cp->communicate, &lg, &lg);
  for (int i = 0; i < ncoef; i++) { rhog_re[i] = scr->cpscr_rho.rhocr_up[i + 1]; rhog_im[i] = scr->cpscr_rho.rhoci_up[i + 1]; }
  CPOPTS *op = &cp->cpopts;
  op->cp_lda = 1; op->cp_lsda = 0; op->cp_nonint = 0; op->cp_para_opt = 0; op->cp_lyp = 0; op->cp_lypm1 = 0;
  op->fftw3dFlag = 1;
  STAT_AVG *sa = &r->gd.stat_avg;
  sa->cp_ehart = sa->cp_eext = sa->cp_exc = sa->cp_muxc = 0.0;
  CP_COMM_STATE_PKG up, dn;
  memset(&up, 0, sizeof up); memset(&dn, 0, sizeof dn);
  up.nstate = 1; up.num_proc = 1;
  double ks_offset = 0.0;
  double pvten[10] = {0};
  char typ[16];
  strcpy(typ, xc == 2 ? "pw_lda" : "pz_lda");
  cpGetVksStodft(op, scr, cpew, ew, &cp->communicate, &up, &dn, sa, &ks_offset, cell, typ, pvten, 0.0, 1.0, 1, 0, 0, 0,
                 0, 0, &lg, &lg, &lg, &lg, 0);
  memcpy(vks, &scr->cpscr_rho.v_ks_up[1], sizeof(double) * N);
  energies[0] = sa->cp_ehart; energies[1] = sa->cp_eext; energies[2] = sa->cp_exc; energies[3] = sa->cp_muxc;
  /* 4. the local-pseudopotential and Ewald reciprocal forces of the atoms
   * (calcLocExtPostScf -> control_ewd_loc, energy/cp/cp_energy_eext.c:646,
   * with the rho(G) of step 3) and the Ewald self and background energies
   * (ewald3d_selfbgr_cp, :2200) as calcEnergyForce forms them
   * (stodft/calc-nuclei-force.c:254, 581-590) */
  if (force) {
    CLATOMS_INFO *ci2 = &r->cls.clatoms_info;
    CLATOMS_POS *ap = &r->apos;
    double *q_keep = ci2->q;
    ci2->q = d1(r->natm);
    for (int a = 0; a < r->natm; a++) ci2->q[a + 1] = q[a];
    ps->q_pseud[1] = q_pseud;
    ew->alp_ewd = alp_ewd;
    ew->self_erf = 1.0;
    cpew->ewaldLocalOpt = 0;
    cpew->realSparseOpt = 0;
    ap->fxCl = d1(r->natm); ap->fyCl = d1(r->natm); ap->fzCl = d1(r->natm);
    for (int a = 1; a <= r->natm; a++) {
      ap->fx[a] = ap->fy[a] = ap->fz[a] = 0.0;
      r->cls.ewd_scr.fx2[a] = r->cls.ewd_scr.fy2[a] = r->cls.ewd_scr.fz2[a] = 0.0;
    }
    if (!r->gd.ptens.pvten_tot) r->gd.ptens.pvten_tot = d1(9);
    if (!r->gd.ptens.pvten) r->gd.ptens.pvten = d1(9);
    double vrec = 0.0, hl = 0.0, vself = 0.0, vbgr = 0.0;
    control_ewd_loc(ci2, ap, cell, &r->gd.ptens, ew, cpew, scr, ps, &r->cls.ewd_scr, &cp->cpopts, &r->cls.atommaps,
                    &vrec, &hl, &cp->communicate, &r->cls.for_scr, 0, 0);
    ewald3d_selfbgr_cp(ci2, ew, &r->gd.ptens, fabs(getdeth(cell->hmat)), &vself, &vbgr, 3);
    for (int a = 0; a < r->natm; a++) {
      force[3 * a] = ap->fx[a + 1]; force[3 * a + 1] = ap->fy[a + 1]; force[3 * a + 2] = ap->fz[a + 1];
    }
    ewald_e[0] = vrec; ewald_e[1] = vself; ewald_e[2] = vbgr;
    ci2->q = q_keep;
  }
  /* the system as it was */
  scr->cpscr_rho.v_ks_up = vks_keep;
  cpew->ak2 = ak2_keep;
  ps->vps0 = keep[0]; ps->vps1 = keep[1]; ps->vps2 = keep[2]; ps->vps3 = keep[3];
  ps->dvps0 = keep[4]; ps->dvps1 = keep[5]; ps->dvps2 = keep[6]; ps->dvps3 = keep[7];
  ps->n_ang_max = nang_keep;
  ps->gzvps[1] = gz_keep;
  ps->nsplin_g = nsp_keep; ps->gmin_spl = gmin_keep; ps->dg_spl = dg_keep;
  return 0;
}

/* The reference's real-space Ewald pair table (spline_vdv with itype 1,
 * iperd 1: vcoul_bin's fitted erfc, interface/inter_params/spline_fit.c:
 * 28-101, 415-437) on its own r grid r_i = dr (i - 3) + rmin, i = 1..n,
 * dr = (rmax - rmin)/(n - 5): r, v and dv = -(dv/dr)/r at each point, for
 * ishift 0 (plain), 1 (shifted to 0 at rmax) or 2 (switched over rheal). */
void ref_coul_table(int n, double rmin, double rmax, double alp, double qij, int ishift, double rheal, double *r,
                    double *v, double *dv) {
  double dr = 0.0, dri = 0.0;
  spline_vdv(rmin, rmax, v - 1, dv - 1, n, &dr, &dri, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, alp, qij, 1,
             1, ishift, rheal, 0, 0.0, 0.0, 1.0);
  for (int i = 1; i <= n; i++) r[i - 1] = dr * (double)(i - 3) + rmin;
}
