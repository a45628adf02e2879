// sdft_lanczos.h -- vector kernels of the device Lanczos bounds and the
// filtered-orbital energies (sdft_lanczos.cu).
#pragma once
#include <cuda_runtime.h>

namespace sdft {

constexpr int kRedBlocks = 128, kRedThreads = 256;  // partials of a deterministic reduction

// *out = <a|b> over the half sphere (2 sum(re re + im im) - re(G0) re(G0));
// part: kRedBlocks doubles of scratch
void launch_half_dot(const double *a, const double *b, int ncoef, int ngp, double *part, double *out,
                     cudaStream_t st);
// raw force -> H c in place (-f/4, -f/2 and Im = 0 at G0)
void launch_lz_hc(double *f, int ncoef, int ngp, cudaStream_t st);
// h <- h - (*alpha) c - beta p  (p null: no p term)
void launch_lz_w(double *h, const double *c, const double *p, const double *alpha, double beta, int ncoef, int ngp,
                 cudaStream_t st);
// p <- c, c <- w / beta
void launch_lz_next(const double *w, double *c, double *p, double beta, int ncoef, int ngp, cudaStream_t st);
// c <- c / sqrt(*nrm2)
void launch_lz_div(double *c, const double *nrm2, int ncoef, int ngp, cudaStream_t st);
// *out = sum over nstate rows, G != G0 of 2 ak2 (re^2 + im^2)
void launch_ekin(const double *v, int nstate, int ncoef, int ngp, const double *ak2, double *part, double *out,
                 cudaStream_t st);
// out = i G_d v per row (Re out = -G_d Im v, Im out = G_d Re v; G = 0 and
// the row padding [ncoef, ngp) zero); gk: G_d per coefficient
void launch_dcoef(const double *v, int nstate, int ncoef, int ngp, const double *gk, double *out, cudaStream_t st);
// f[3 a + d] = -2 scale sum_{state, u in rows of atom a} w[u] Z0[s][u] Zd[s][u]
void launch_nl_force_atoms(const double *Z0, const double *Zd, int ldz, const double *w, const int *row_start,
                           const int *row_count, int natm, int nstate, double scale, int d, double *f,
                           cudaStream_t st);
// smallest and largest eigenvalue of the symmetric tridiagonal matrix
// (diagonal a[0..n), off-diagonal b[0..n-1)), by Sturm bisection (host)
void tridiag_extremes(const double *a, const double *b, int n, double *lo, double *hi);

}  // namespace sdft
