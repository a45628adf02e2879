/*
 * sdft_b200.h -- C ABI of the B200 stochastic-DFT filter hot path.
 *
 * Every entry point takes plain pointers and sizes and returns an int
 * status (SDFT_OK == 0).  Orbital arrays use the PINY layout: state-major,
 * coefficient-minor, half G-sphere with G=0 stored LAST, separate real and
 * imaginary arrays.  Pointers here are 0-based; a PINY caller holding the
 * 1-based cmalloc(n)-1 pointer passes &p[1].
 *
 * Reference interfaces replaced (file:line inside the reference project):
 *   sdft_gvec_count / sdft_gvec_fill  <- setkvec3d_sm        interface/cp_ewald/set_cp_ewald.c:685
 *   sdft_fft_maps                     <- setfft_indx (filter maps)  mathlib/fft_create_package.c:981,139-248
 *   sdft_hpsi                         <- calcCoefForceWrapSCF stodft/reduced-energy/energy-wrapper-scf.c:1066
 *   sdft_normh_cheby                  <- normHCheby          stodft/normh.c:182
 *   sdft_normh_newton                 <- normHNewtonHerm     stodft/normh.c:35
 *   sdft_filter_cheby                 <- filterChebyPolyHerm stodft/filter.c:318
 *   sdft_filter_newton                <- filterNewtonPolyHerm stodft/filter.c:33
 *   sdft_cheby_moments                <- calcChebyMoments    stodft/calc-chempot-chebyshev.c:596
 *   sdft_chempot_cheby                <- calcChemPotCheby (bisection part) stodft/calc-chempot-chebyshev.c:30
 *   sdft_num_elec_cheby               <- calcNumElecCheby    stodft/calc-chempot-chebyshev.c:918
 *   sdft_cheby_coeff                  <- calcChebyCoeff      stodft/coeff.c:1093
 *   sdft_round_fft                    <- roundFFT            stodft/coeff.c:1556
 *   sdft_newton_samp / sdft_newton_coeff <- genSampNewtonHermit / genCoeffNewtonHermit stodft/coeff.c:423,199
 *   sdft_density                      <- rhoCalcRealStoHybrid stodft/density.c:43 (+ sum_rho mathlib/fft_package.c:2502)
 *   sdft_noise_real                   <- genNoiseOrbitalReal stodft/gen-noise.c:162
 *   sdft_gaussran2                    <- gaussran2 / ran_essl / DURAND mathlib/mathlib.c:118,30; mathlib/blas_wrappers.f:39
 *   sdft_gaussran2_signs_dev          <- the gaussran2 call of genNoiseOrbitalReal, stodft/gen-noise.c:256 (signs only)
 *   sdft_lanczos_bounds               <- genEnergyMax/genEnergyMin stodft/calc-spectral-range.c:33,339 (Lanczos)
 *   sdft_energy_chempot_dev           <- calcEnergyChemPot stodft/calc-energy.c:32
 *   sdft_nl_force_dev                 <- calcEnergyForce stodft/calc-nuclei-force.c:33 (nonlocal part:
 *                                        calcNlPseudoPostScf stodft/reduced-energy/energy-wrapper-post-scf.c:224)
 *   sdft_xc_lda_dev                   <- excpot_pz_lda / excpot_pw_lda energy/cp/xc_functionals.c:268,378
 *   sdft_vks_from_rho                 <- calcRhoStoRecipFullg stodft/density.c:699 + cpGetVksStodft
 *                                        stodft/reduced-energy/cp-energy-ee-rho-stodft.c:644
 *   sdft_vks_set_local                <- controlEwdLocPreScf's vext(G) loop
 *                                        stodft/reduced-energy/cp-energy-eext-stodft.c:340-470
 *   sdft_vks_local_forces             <- calcLocExtPostScf / control_ewd_loc energy/cp/cp_energy_eext.c:646
 *                                        + ewald3d_selfbgr_cp :2200 (calc-nuclei-force.c:254,581)
 *   sdft_ewald_real                   <- energy_control_inter_real's Ewald pair term (calc-nuclei-force.c:605,635;
 *                                        vcoul_bin interface/inter_params/spline_fit.c:415-437)
 *   sdft_mixer_*                      <- genDensityMix stodft/diis.c:34; checkpointOutput/Input
 *                                        stodft/checkpointIO.c:32,218
 */
#ifndef SDFT_B200_H
#define SDFT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define SDFT_OK            0
#define SDFT_ERR_ARG       1   /* invalid argument / size                  */
#define SDFT_ERR_CUDA      2   /* CUDA runtime error (message via sdft_last_error) */
#define SDFT_ERR_NOMEM     3   /* device allocation failed                 */
#define SDFT_ERR_STATE     4   /* call out of order (e.g. no potential set) */
#define SDFT_ERR_UNSUPPORTED 5 /* grid size / l channel not supported       */
#define SDFT_ERR_NODEVICE  6   /* no CUDA device visible                    */
#define SDFT_ERR_TIMEOUT   7   /* a bounded device-side wait gave up        */

/* ---- precision modes ------------------------------------------------- */
#define SDFT_PREC_FP64  0      /* everything FP64 (plain form)               */
#define SDFT_PREC_MIXED 1      /* FP32 FFT + V multiply, KB GEMMs on INT8
                                  tensor cores in the Ozaki digit scheme
                                  (about 28-bit operands, exact products and
                                  sums), FP64 recurrence / accumulators /
                                  reductions */
#define SDFT_PREC_MIXED_FAST 2 /* as MIXED, but the back projection (whose
                                  result is stored in FP32) multiplies
                                  24-bit digits (3 x 8 bits, 6 products
                                  instead of 10): about 8 % faster at 512
                                  atoms, force error ~2e-7 instead of ~2e-8 */

typedef struct sdft_ctx sdft_ctx;

/* Kleinman-Bylander projector description (one radial projector per l
 * channel, n_rad = 1).  Radial form factors are PINY spline tables
 * evaluated exactly as get_vpsnow (energy/cp/cp_energy_eext.c:2139):
 *   v(g) = ((vps3*h + vps2)*h + vps1)*h + vps0,  h = g - g_i,
 *   i = clamp((int)((g-gmin)/dg) + 1, 1, nsplin) (1-based knot).        */
typedef struct {
  int natm;              /* atoms carrying nonlocal channels             */
  const double *pos;     /* natm*3 cartesian coordinates (bohr)          */
  const int *type;       /* natm, 0-based atom type                      */
  int ntype;
  int lmax;              /* highest l channel present (0..2)             */
  const int *lmax_type;  /* ntype: highest l of each type (-1 = none)    */
  int nsplin_g;
  double gmin_spl, dg_spl;
  const double *vps;     /* [ntype][lmax+1][4][nsplin_g]: vps0..vps3     */
  const double *vpsnorm; /* [ntype][lmax+1]  KB energies                 */
  const double *gzvps0;  /* [ntype]  l=0 value at G=0                    */
} sdft_kb_desc;

/* ---- errors ----------------------------------------------------------- */
const char *sdft_last_error(void);
int sdft_version(void);

/* ---- G-sphere setup (host only) --------------------------------------- */
/* hmat: 9 doubles, PINY column-major cell matrix (hmat[0]=h11, hmat[1]=h21,
 * ...).  ecut in Hartree: 0.5|G|^2 <= ecut.  kmax: scan limits (kmax_cp).
 * Returns nktot (half sphere without G=0); ncoef = nktot+1.             */
int sdft_gvec_count(const double *hmat, double ecut, const int *kmax, int *nktot);
/* Fill ka/kb/kc[ncoef] (0-based arrays, G=0 last) and ibreak1/2[nktot]
 * in the setkvec3d_sm order.                                            */
int sdft_gvec_fill(const double *hmat, double ecut, const int *kmax, int nktot,
                   int *ka, int *kb, int *kc, int *ibreak1, int *ibreak2);
/* Complex grid indices of G and -G in the filter layout (c fastest):
 * map[i] = mapFFTWFilter[i+1], mapc[i] = mapConFFTWFilter[i+1].        */
int sdft_fft_maps(int nkf1, int nkf2, int nkf3, int ncoef, const int *ka,
                  const int *kb, const int *kc, int *map, int *mapc);
/* ak2Kinetic (get_ak2_sm, energy/cp/cp_energy_eext.c:2260): |G|^2, capped
 * at gcut^2 when gcut > 0.  out[ncoef], G=0 entry 0.                    */
int sdft_ak2_kinetic(const double *hmat, int ncoef, const int *ka, const int *kb,
                     const int *kc, double gcut, double *ak2);

/* ---- context ----------------------------------------------------------- */
/* Creates a device context for one G-sphere / FFT grid.  max_states is the
 * largest orbital block later passed to the compute calls.              */
int sdft_ctx_create(int nkf1, int nkf2, int nkf3, int ncoef, const int *ka,
                    const int *kb, const int *kc, const double *hmat,
                    int precision, int max_states, int device, sdft_ctx **out);
int sdft_ctx_destroy(sdft_ctx *ctx);
/* Kinetic cutoff cap gCutoffKe (<=0: none).                             */
int sdft_ctx_set_kinetic_cap(sdft_ctx *ctx, double gcut);
/* V_KS(r): nkf1*nkf2*nkf3 doubles in the filter layout, c fastest
 * (the reference's v_ks_up after the transpose at
 * stodft/reduced-energy/cp-energy-ee-rho-stodft.c:984-1007), in host or
 * device memory (sdft_vks_from_rho can leave it on the device).         */
int sdft_ctx_set_vks(sdft_ctx *ctx, const double *v_ks);
/* KB nonlocal projectors; kb == NULL or kb->natm == 0 disables them.   */
int sdft_ctx_set_kb(sdft_ctx *ctx, const sdft_kb_desc *kb);
/* Bytes of device memory the context holds (for HBM-budget admission). */
long long sdft_ctx_device_bytes(const sdft_ctx *ctx);
/* CUDA stream the context launches on (cudaStream_t as void*).          */
void *sdft_ctx_stream(sdft_ctx *ctx);

/* ---- hot path: host buffers in/out ------------------------------------- */
/* Raw PINY coefficient force f = -(2 H c) scaled as the reference keeps it:
 * H c = -f/4 (G != 0), -f/2 (G = 0).  enl (nullable): nonlocal energy. */
int sdft_hpsi(sdft_ctx *ctx, int nstate, const double *cre, const double *cim,
              double *fcre, double *fcim, double *enl);

/* One normalized-H step.  cheby: iPoly>=1, wf1 = T_{k-1} (used if iPoly>1);
 * on return f = T_{k+1}; with cpy_flag the buffers rotate as normHCheby.  */
int sdft_normh_cheby(sdft_ctx *ctx, int nstate, int ipoly, int cpy_flag,
                     double scale, double energy_mean, double *cre, double *cim,
                     double *wf1re, double *wf1im, double *fcre, double *fcim);
int sdft_normh_newton(sdft_ctx *ctx, int nstate, double scale, double energy_mean,
                      double zn, double *cre, double *cim, double *fcre, double *fcim);

/* Chebyshev filter: stoWf[imu] = sum_k expanCoeff[k*numChemPot+imu] T_k(Hn) chi.
 * sto_re/sto_im: numChemPot host pointers to nstate*ncoef doubles.
 * moments (nullable, storeChebyMomentsFlag): L+1 doubles, overwritten:
 * moments[k] = sum_s <chi_s|T_k chi_s> (half-sphere weighted), k < L.  */
int sdft_filter_cheby(sdft_ctx *ctx, int nstate, const double *cre, const double *cim,
                      int L, int num_chem_pot, const double *expan_coeff,
                      double scale, double energy_mean,
                      double **sto_re, double **sto_im, double *moments);
/* Newton filter with interpolation points samp_point[L].               */
int sdft_filter_newton(sdft_ctx *ctx, int nstate, const double *cre, const double *cim,
                       int L, int num_chem_pot, const double *expan_coeff,
                       const double *samp_point, double scale, double energy_mean,
                       double **sto_re, double **sto_im);
/* Chebyshev moments by the doubling identities, L+1 doubles (unnormalised
 * sum over the nstate orbitals, as before the Reduce of calcChemPotCheby). */
int sdft_cheby_moments(sdft_ctx *ctx, int nstate, const double *cre, const double *cim,
                       int L, double scale, double energy_mean, double *moments);
/* rho[ia + nkf1*(ib + nkf2*ic)] = sum_s |psi_s(r)|^2 (package layout,
 * a fastest), unscaled like rhoCalcRealStoHybrid's rho_scr.            */
int sdft_density(sdft_ctx *ctx, int nstate, const double *cre, const double *cim,
                 double *rho);
/* Noise orbitals of genNoiseOrbitalReal for state-rank myid of np ranks:
 * random +-sqrt(N) real-space values (gaussran2 signs), FFT to G.     */
int sdft_noise_real(sdft_ctx *ctx, int nstate, double seed, int np_states, int myid,
                    double *cre, double *cim);

/* ---- hot path: device-resident variants -------------------------------- */
/* Orbital block kept in HBM by the context (slot 0: chi). */
int sdft_upload_orbitals(sdft_ctx *ctx, int nstate, const double *cre, const double *cim);
int sdft_noise_real_dev(sdft_ctx *ctx, int nstate, double seed, int np_states, int myid);
int sdft_filter_cheby_dev(sdft_ctx *ctx, int nstate, int L, int num_chem_pot,
                          const double *expan_coeff, double scale, double energy_mean);
int sdft_filter_newton_dev(sdft_ctx *ctx, int nstate, int L, int num_chem_pot,
                           const double *expan_coeff, const double *samp_point,
                           double scale, double energy_mean);
int sdft_cheby_moments_dev(sdft_ctx *ctx, int nstate, int L, double scale,
                           double energy_mean, double *moments);
/* Density of the filtered orbitals of chem-pot imu, result stays on device
 * unless rho != NULL (host or device memory; copied, then synchronised).
 * occ_over_nsto scales it (aveFactUp).                                   */
int sdft_density_dev(sdft_ctx *ctx, int nstate, int imu, double occ_over_nsto,
                     double *rho);
int sdft_download_filtered(sdft_ctx *ctx, int nstate, int imu, double *re, double *im);
/* The last density computed on the context (by sdft_density_dev or a batch
 * replay), copied to host or device memory without recomputing it. */
int sdft_download_density(sdft_ctx *ctx, double *rho);
/* Waits for the context's stream.  SDFT_ERR_TIMEOUT when a bounded wait in
 * a tensor-core GEMM gave up since the last sync (that work's results are
 * not valid); the error word is then cleared, so the context serves later
 * calls.  No counterpart in the reference (its calls are synchronous).  */
int sdft_sync(sdft_ctx *ctx);
/* Diagnostic without a counterpart in the reference: one kernel on the
 * context's stream waits on an mbarrier that nothing arrives at, through
 * the GEMMs' bounded-wait helper capped at `polls` polls (1..2^22), gives
 * up and sets the context's error word; the next sdft_sync reports
 * SDFT_ERR_TIMEOUT.  Shows on a device that a wait which runs out ends with
 * an error status the host reads and leaves the context usable. */
int sdft_ctx_selftest_wait(sdft_ctx *ctx, long long polls);
/* Cap on the device memory this library allocates on `device`: contexts,
 * mixers and scratch together, bytes; 0 removes the cap.  An allocation
 * that would pass it fails with SDFT_ERR_NOMEM like one the device refuses:
 * the call that needed it returns the error and its context stays usable.
 * A serving loop with a fixed HBM budget sets it so that an estimate that
 * was too small cannot take memory from other requests.  No counterpart in
 * the reference (PINY allocates host memory only). */
int sdft_set_device_memory_limit(int device, long long bytes);
/* Bytes this library holds on `device` now (-1 for a bad index).       */
long long sdft_device_memory_in_use(int device);

/* ---- events (host code that times and orders device work) ------------- */
/* No counterpart in the reference.  For callers that drive the library
 * without another CUDA binding (the serving loop, the autotuner):
 * sdft_set_device makes `device` current for the calling thread;
 * an event is created with timing on `device`, recorded on a stream (a
 * context's or batch's stream, NULL = the legacy default stream), queried
 * (*done = 1 once the work before it has finished, 0 before), waited for,
 * and two recorded events give the elapsed device time in ms.          */
int sdft_set_device(int device);
int sdft_event_create(int device, void **ev);
int sdft_event_record(void *ev, void *stream);
int sdft_event_query(void *ev, int *done);
int sdft_event_synchronize(void *ev);
int sdft_event_elapsed_ms(void *ev0, void *ev1, float *ms);
int sdft_event_destroy(void *ev);
/* Kernel launches issued by the context since creation (own kernels only). */
long long sdft_launch_count(const sdft_ctx *ctx);
/* Per-kernel device timing with CUDA events on the context stream.
 * Kinds: 0 pack+c-FFT (stage A), 1 plane FFT x V (stage B), 2 c-FFT+unpack+
 * recurrence (stage C), 3 KB projection GEMM, 4 KB back-projection GEMM,
 * 5 density planes, 6 noise planes, 7 other.  read_timing synchronises,
 * returns accumulated milliseconds / launch counts per kind and resets.   */
#define SDFT_NKIND 8
int sdft_ctx_set_timing(sdft_ctx *ctx, int enable);
int sdft_ctx_read_timing(sdft_ctx *ctx, double *ms, long long *count);

/* ---- spectral bounds and energies --------------------------------------- */
/* Spectral bounds of H from nstep Lanczos steps on one orbital, all vectors
 * device resident (the role of genEnergyMax/genEnergyMin,
 * stodft/calc-spectral-range.c:33,339, which run power iterations; 20
 * Lanczos steps replace them here).  v0re/v0im (host, ncoef each): start
 * vector, normalised on the device.  alpha/beta (nullable, nstep each) get
 * the tridiagonal coefficients, *nsteps how many steps ran (fewer when
 * beta < 1e-12).  *emin / *emax = extreme eigenvalues of the tridiagonal
 * matrix -/+ margin (0.1 Ha in calc-spectral-range.c).  Uses orbital slot
 * 0 of the context (resident orbitals are invalidated). */
int sdft_lanczos_bounds(sdft_ctx *ctx, int nstep, const double *v0re, const double *v0im, double margin,
                        double *alpha, double *beta, int *nsteps, double *emin, double *emax);
/* calcEnergyChemPot (stodft/calc-energy.c:32-207) for chemical potential
 * imu of the filtered orbitals resident on the device (first nstate):
 * energy_ke = occ/2 sum_s sum_{G != 0} 2 ak2Kinetic |c_s(G)|^2 / nsto_total,
 * energy_pnl = occ E_NL / nsto_total, E_NL the Kleinman-Bylander energy of
 * the orbitals (stat_avg->cp_enl of calcNonLocalPseudoScf).  With several
 * ranks, sum the per-rank values (each passing the global nsto_total). */
int sdft_energy_chempot_dev(sdft_ctx *ctx, int nstate, int imu, double occ, int nsto_total,
                            double *energy_ke, double *energy_pnl);
/* The nonlocal (Kleinman-Bylander) atomic forces of calcEnergyForce
 * (stodft/calc-nuclei-force.c:33-480: calcNlPseudoPostScf, then occNumber /
 * numStateStoUp) for chemical potential imu of the filtered orbitals
 * resident on the device (first nstate):
 * fatm[3 a + d] = -2 occ / nsto_total sum_{s, l, m} vnorm_l / vol
 *                 (Re Z dRe Z/dR_ad + Im Z dIm Z/dR_ad),
 * atoms in the order of sdft_kb_desc.pos.  energy_pnl (nullable) as in
 * sdft_energy_chempot_dev.  With several ranks, sum the per-rank forces. */
int sdft_nl_force_dev(sdft_ctx *ctx, int nstate, int imu, double occ, int nsto_total, double *fatm,
                      double *energy_pnl);

/* ---- exchange-correlation ----------------------------------------------- */
#define SDFT_XC_PZ_LDA 1  /* Perdew-Zunger 1981 (excpot_pz_lda)            */
#define SDFT_XC_PW_LDA 2  /* Perdew-Wang 1992 (excpot_pw_lda)              */
/* The LDA step of cpGetVksStodft (stodft/reduced-energy/
 * cp-energy-ee-rho-stodft.c:838-870; energy/cp/xc_functionals.c:268,378),
 * spin-unpolarised: over the n real-space points, vks += V_xc(rho) and
 * *exc / *muxc (nullable) = E_xc and sum V_xc rho, both times vol / n.
 * rho and vks are device pointers; runs on `stream` and synchronises it. */
int sdft_xc_lda_dev(int kind, long long n, const double *rho, double *vks, double vol, double *exc,
                    double *muxc, void *stream);

/* ---- the Kohn-Sham potential from the density (SCF caller) ------------- */
/* A density grid: the half sphere of the density cutoff (0.5|G|^2 <= 4 Ecut,
 * setkvec3d of interface/cp_ewald/set_cp_ewald.c:525, PINY order, G = 0
 * last) on an nkf1 x nkf2 x nkf3 grid (edges 2^a 3^b <= 128) that holds it.
 * hmat as for sdft_ctx_create. */
typedef struct sdft_vks sdft_vks;
int sdft_vks_create(int nkf1, int nkf2, int nkf3, const double *hmat, int ncoef, const int *ka,
                    const int *kb, const int *kc, int device, sdft_vks **out);
int sdft_vks_destroy(sdft_vks *v);
/* The local pseudopotential on the density sphere, as controlEwdLocPreScf
 * forms vext (cp-energy-eext-stodft.c:412-413, 449-455) for a periodic
 * cell whose local tables carry the whole local potential:
 *   vext(G) = (1/vol) sum_a v_t(a)(|G|) (cos, -sin)(2 pi k.s_a),
 *   vext(0) = (1/vol) sum_a gzvps[t(a)],
 * s_a = h^-1 r_a; v_t by get_vpsnow's cubic on the per-knot Taylor table
 * vloc[(t*4 + d)*nsplin + knot] (d = 0..3), knots gmin + k dg.  pos is
 * natm x 3 cartesian (bohr), type[a] in 0..ntype-1 (host arrays).        */
int sdft_vks_set_local(sdft_vks *v, int natm, const double *pos, int ntype, const int *type, int nsplin,
                       double gmin_spl, double dg_spl, const double *vloc, const double *gzvps);
/* calcRhoStoRecipFullg followed by cpGetVksStodft (cp_dual_grid_opt 0,
 * periodic, LDA or none): rho is nkf1*nkf2*nkf3 doubles in the package
 * layout (a fastest), the density times the cell volume as the reference
 * passes it (host or device memory).  rho(G) = (1/N) sum_r rho(r) e^{-iG.r}
 * on the half sphere; V(G) = vext(G) + 4 pi rho(G)/(|G|^2 vol) (G != 0),
 * V(0) = vext(0); V(r) = sum_G V(G) e^{+iG.r} over G and -G; plus V_xc of
 * rho/vol when xc_kind is SDFT_XC_PZ_LDA or SDFT_XC_PW_LDA (0: none).
 * vks_filter receives V_KS in the filter layout, c fastest (host or device
 * memory: pass it to sdft_ctx_set_vks); rho_g (nullable) receives rho(G),
 * re[ncoef] then im[ncoef]; energies (nullable) = {E_H, E_ext, E_xc,
 * mu_xc} as cp_ehart, cp_eext, cp_exc, cp_muxc.  Synchronous.           */
int sdft_vks_from_rho(sdft_vks *v, const double *rho, int xc_kind, double *vks_filter, double *rho_g,
                      double *energies);
/* vext(G) of the last sdft_vks_set_local: re[ncoef], im[ncoef] (host).  */
int sdft_vks_get_vext(sdft_vks *v, double *re, double *im);
/* The local-pseudopotential and Ewald reciprocal-space forces on the atoms
 * of sdft_vks_set_local, from rho(G) of the last sdft_vks_from_rho: the
 * part of calcEnergyForce (stodft/calc-nuclei-force.c:254) that
 * calcLocExtPostScf runs through control_ewd_loc (energy/cp/
 * cp_energy_eext.c:646, periodic, ewaldLocalOpt 0), plus the Ewald self
 * and background energies (ewald3d_selfbgr_cp, :2200, calc-nuclei-force.c:
 * 581-590).  Over the half sphere, per atom a of charge q[a] and type t:
 *   vt = v_t(|G|) - 4 pi (q[a] - q_pseud[t]) / G^2,
 *   S(G) = sum_b q_b e^{i 2 pi k.s_b}, preg = e^{-G^2/4 alp^2} 4 pi/(G^2 vol),
 *   F_a += G [(2 preg Re S q_a + 2 Re rho vt/vol) sin(2 pi k.s_a)
 *             - (2 preg Im S q_a - 2 Im rho vt/vol) cos(2 pi k.s_a)].
 * force[natm*3] (hartree/bohr); ewald = {vrecip = sum preg |S|^2,
 * vself = -alp/sqrt(pi) sum q^2, vbgr = -pi (sum q)^2 / (2 alp^2 vol)}.
 * The real-space ion-ion Ewald sum (energy_control_inter_real, PINY's
 * classical force engine) is not part of this call. */
/* The real-space ion-ion Ewald sum of the nuclear force: what
 * calc-nuclei-force.c:605/635 takes from PINY's pair engine
 * (energy_control_inter_real over the vcoul_bin table,
 * interface/inter_params/spline_fit.c:415-437, iperd > 0), summed here
 * directly over every pair and periodic image closer than rmax:
 *   E = 1/2 sum_a sum_{b, n; (b, n) != (a, 0)} v(|r_a - r_b - h n|),
 *   v(r) = q_a q_b gerfc(alp r)/r with the reference's fit of erfc,
 *   ishift 0: as is; 1: shifted to 0 at rmax; 2: times the reference's cubic
 *   switch over [rmax - rheal, rmax] (spline_fit.c:61-72, 87-92).
 * pos[natm*3] Cartesian (bohr), q[natm], hmat as elsewhere (cell vectors in
 * columns); force[natm*3] = -dE/dR, *energy = E (hartree).  The reference
 * interpolates v from a table; this evaluates it at each distance, FP64.
 * Host arrays; runs on the current device and `stream` (may be 0), returns
 * after it completes.  rmax may span at most 16 cells per direction.
 * Together with sdft_vks_local_forces' reciprocal, self and background
 * terms it is the full Ewald ion-ion energy. */
int sdft_ewald_real(int natm, const double *pos, const double *q, const double *hmat, double alp_ewd, double rmax,
                    int ishift, double rheal, double *force, double *energy, void *stream);
int sdft_vks_local_forces(sdft_vks *v, const double *q, const double *q_pseud, double alp_ewd, double *force,
                          double *ewald);

/* ---- density mixing and checkpoint files -------------------------------- */
/* genDensityMix (stodft/diis.c:34-464) with the densities on the device,
 * spin-unpolarised, one rank (with several ranks, each mixes its own slice
 * of the grid; the DIIS dot products then need a sum over ranks, which this
 * mixer does not do).  n grid values; num_diis <= 16 DIIS terms; the first
 * num_step_mix steps after step 0 mix with mix_ratio_big, later ones run
 * DIIS with the extra mixing alpha = mix_ratio_sm (steps <= 10) or
 * mix_ratio_sm2. */
typedef struct sdft_mixer sdft_mixer;
int sdft_mixer_create(int device, long long n, int num_diis, int num_step_mix, double mix_ratio_big,
                      double mix_ratio_sm, double mix_ratio_sm2, sdft_mixer **out);
/* One SCF step iscf (0, 1, 2, ...): rho_correct = the new density
 * (rhoUpCorrect), rho = the mixed density (rho_up), written for iscf >= 1
 * and left untouched at iscf 0 as the reference does.  Host or device
 * pointers (unified addressing). */
int sdft_mixer_step(sdft_mixer *m, int iscf, const double *rho_correct, double *rho);
/* Last step index, min(iscf, num_diis) and the DIIS coefficients of the
 * last DIIS step (nullable outputs). */
int sdft_mixer_state(const sdft_mixer *m, int *iscf, int *num_diis_now, double *coef);
/* checkpointOutput (stodft/checkpointIO.c:32): text file "iscf numDiisNow",
 * rho * vol, the banked densities and the errors, one "%.16lg" value per
 * line -- byte-identical to the reference's density-checkpoint. */
int sdft_mixer_write_checkpoint(sdft_mixer *m, const char *path, const double *rho, double vol);
/* checkpointInput (stodft/checkpointIO.c:218): restores the step index,
 * the banks and errors; rho and the mixer's rho_old receive the file's
 * density values as stored (rho * vol, not divided back, as the reference
 * does). */
int sdft_mixer_read_checkpoint(sdft_mixer *m, const char *path, double *rho);
int sdft_mixer_destroy(sdft_mixer *m);

/* ---- tuning and batched systems ---------------------------------------- */
/* No counterpart in the reference (it filters one system per run).
 * Split-K of the nonlocal projection GEMM: 0 = built-in cost model,
 * 1..64 = fixed (chosen by the autotuner in tuner.py).                    */
int sdft_ctx_set_gemm_split(sdft_ctx *ctx, int split);
/* Orbital columns per output tile of the mixed-precision KB GEMMs: 0 = per
 * call (64 where it pads the orbital count less than 128, e.g. 16..64 or
 * 129..192 orbitals), 64 or 128 = fixed (chosen by the autotuner in
 * tuner.py).  Results are bitwise equal for every width: each output is the
 * same exact integer sum per K range.  No counterpart in the reference. */
int sdft_ctx_set_gemm_bn(sdft_ctx *ctx, int bn);
/* Threads per CTA of the FP32 plane stage (one CTA per plane and orbital
 * pair): 256, 128 (more CTAs per SM, faster on small planes), or 0 = the
 * library's default, 128 for planes of 48 x 48 to 72 x 72 points and 256
 * otherwise.  128 is
 * accepted by mixed-precision contexts on the fast FFT path only; chosen
 * per system by the autotuner (tuner.py).  No counterpart in the reference. */
int sdft_ctx_set_plane_threads(sdft_ctx *ctx, int nt);
/* CUDA stream priority of the context's stream (lower = more urgent, 0 =
 * default; clamped to the device's range).  Call while the context is idle:
 * the stream is replaced.  A server gives cheap requests the urgent
 * priorities so they are not queued behind large ones on a shared GPU. */
int sdft_ctx_set_priority(sdft_ctx *ctx, int priority);
/* One CUDA graph running, for every context i (orbitals resident, V and KB
 * set), the Chebyshev filter of nstate[i] orbitals with the L[i]
 * coefficients coeffs[i] (one chemical potential) followed by the density
 * of the result scaled by occ_over_nsto[i].  Each context's stream is one
 * branch of the graph, so systems of different grids run concurrently.
 * Creation sizes every buffer, uploads the coefficients and captures;
 * sdft_batch_launch replays the whole batch with a single graph launch
 * (asynchronous; refilters whatever orbitals are resident).  Afterwards each
 * context's result is read with sdft_density_dev / sdft_download_filtered. */
typedef struct sdft_batch sdft_batch;
int sdft_batch_create(int n, sdft_ctx *const *ctxs, const int *nstate, const int *L,
                      const double *const *coeffs, const double *scale, const double *emean,
                      const double *occ_over_nsto, sdft_batch **out);
int sdft_batch_launch(sdft_batch *b);
int sdft_batch_sync(sdft_batch *b);
void *sdft_batch_stream(sdft_batch *b);
/* Priority of the stream the batch's graph is launched into (its kernels
 * run at that priority); as sdft_ctx_set_priority, while idle. */
int sdft_batch_set_priority(sdft_batch *b, int priority);
/* own kernels + memsets issued by one replay */
long long sdft_batch_kernel_count(const sdft_batch *b);
int sdft_batch_destroy(sdft_batch *b);

/* ---- allocation-free device helper ------------------------------------ */
/* No counterpart in the reference.  Per-orbital half-sphere inner products
 *   out[s] = 2 sum_G (a_re b_re + a_im b_im) - a_re(G0) b_re(G0)
 * (the sum over all ncoef stored coefficients, as the reference's ddot
 * forms it in stodft/filter.c:492 and calc-chempot-chebyshev.c:725)
 * of nstate orbitals of ncoef coefficients (G0 last), all five arrays in
 * device memory of the calling thread's current device; queued on `stream`
 * (a cudaStream_t, NULL = default stream) and asynchronous.  Allocates
 * nothing: for callers whose device memory is fully owned by their own pool
 * or fixed in size.  Partial sums live in a static 64 KB device array
 * compiled into the library; nstate above 1024 is rejected
 * (SDFT_ERR_ARG).  The first call on a device loads the kernels there
 * and should come before any stream capture; every call looks the array's
 * address up in the current context.  Calls that may overlap on one
 * device race on the array: order them on one stream.                    */
int sdft_half_dots_noalloc(const double *a_re, const double *a_im,
                           const double *b_re, const double *b_im,
                           int ncoef, int nstate, double *out, void *stream);

/* ---- host FP64 helpers (no device) ------------------------------------ */
int sdft_round_fft(int n);
/* fun_flag 1: F, 2: sqrt(F) (Fermi-Dirac 1/(1+exp(beta(x-mu)))).        */
int sdft_cheby_coeff(int L, int num_cheby_grid, double energy_diff, double energy_mean,
                     double beta, double chem_pot, int fun_flag, double *coeffs);
double sdft_num_elec_cheby(int L, int num_cheby_grid, double energy_diff,
                           double energy_mean, double beta, double chem_pot,
                           double occ, const double *moments);
/* Bisection of calcChemPotCheby on normalised moments (moments / N_sto). */
int sdft_chempot_cheby(int L, double energy_diff, double energy_mean, double beta,
                       double occ, const double *moments, double num_elec_true,
                       double chem_pot_init, double gap_init, double *chem_pot,
                       double *num_elec);
int sdft_newton_samp(int L, double smin, double smax, double scale, double energy_min,
                     double *samp_point, double *samp_point_unscale);
int sdft_newton_coeff(int L, int num_chem_pot, const double *chem_pot, double beta,
                      const double *samp_point, const double *samp_point_unscale,
                      double *expan_coeff);
/* gaussran2 with the DURAND uniform generator; qseed updated in place. */
int sdft_gaussran2(int nran, double *qseed, double *gauss);
/* Signs of gaussran2(nran, *qseed) generated on the device: neg (device
 * memory, nran bytes) gets 1 where the value is negative, 0 elsewhere --
 * the sign pattern genNoiseOrbitalReal (stodft/gen-noise.c:256) turns into
 * noise.  Byte-identical to the host generator; *qseed is left where
 * gaussran2 leaves it.  Runs on `stream` (cudaStream_t, 0 = default) and
 * synchronises it. */
int sdft_gaussran2_signs_dev(long long nran, double *qseed, unsigned char *neg, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SDFT_B200_H */
