// sdft_lanczos.cu -- vector kernels of the device Lanczos bounds and of the
// filtered-orbital energies and KB atomic forces.
//
// Vectors are one orbital row of the context layout: re[0, ncoef) then
// im[0, ncoef) at offset ngp; G0 is entry ncoef - 1.  Reductions are
// deterministic: kRedBlocks fixed block partials, each a fixed-order tree,
// summed in block order by one thread.
#include <cuda_runtime.h>
#include <algorithm>
#include "sdft_lanczos.h"

namespace sdft {

namespace {

__device__ __forceinline__ void block_sum_to(double a, double *out) {
  __shared__ double sh[kRedThreads];
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int s = kRedThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// half-sphere inner product <a|b> = 2 sum (re re + im im) - re(G0) re(G0)
__global__ void __launch_bounds__(kRedThreads) k_hdot_part(const double *__restrict__ a, const double *__restrict__ b,
                                                           int ncoef, int ngp, double *__restrict__ part) {
  double s = 0.0;
  for (int g = blockIdx.x * kRedThreads + threadIdx.x; g < ncoef; g += kRedBlocks * kRedThreads) {
    const double rr = a[g] * b[g], ii = a[ngp + g] * b[ngp + g];
    s += (g == ncoef - 1) ? rr + 2.0 * ii : 2.0 * (rr + ii);
  }
  block_sum_to(s, part + blockIdx.x);
}

__global__ void k_sum_fixed(const double *__restrict__ part, int n, double *__restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += part[i];
    *out = s;
  }
}

// H c from the raw PINY force f (-4 H c at G != 0, -2 H c at G0), in place;
// Im H c (G0) = 0
__global__ void k_lz_hc(double *__restrict__ f, int ncoef, int ngp) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ncoef; g += gridDim.x * blockDim.x) {
    const bool g0 = g == ncoef - 1;
    f[g] = (g0 ? -0.5 : -0.25) * f[g];
    f[ngp + g] = g0 ? 0.0 : -0.25 * f[ngp + g];
  }
}

// w = h - alpha c - beta p (in place in h); p may be null when beta == 0
__global__ void k_lz_w(double *__restrict__ h, const double *__restrict__ c, const double *__restrict__ p,
                       const double *__restrict__ alpha, double beta, int ncoef, int ngp) {
  const double a = *alpha;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ncoef; g += gridDim.x * blockDim.x) {
    for (int part = 0; part < 2; part++) {
      const int i = part * ngp + g;
      double w = h[i] - a * c[i];
      if (p) w -= beta * p[i];
      h[i] = w;
    }
  }
}

// p = c, c = w / beta
__global__ void k_lz_next(const double *__restrict__ w, double *__restrict__ c, double *__restrict__ p, double beta,
                          int ncoef, int ngp) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ncoef; g += gridDim.x * blockDim.x) {
    for (int part = 0; part < 2; part++) {
      const int i = part * ngp + g;
      p[i] = c[i];
      c[i] = w[i] / beta;
    }
  }
}

// c /= d (normalisation of the start vector)
__global__ void k_lz_div(double *__restrict__ c, const double *__restrict__ nrm2, int ncoef, int ngp) {
  const double d = sqrt(*nrm2);
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ncoef; g += gridDim.x * blockDim.x) {
    c[g] = c[g] / d;
    c[ngp + g] = c[ngp + g] / d;
  }
}

// sum over nstate rows and G != G0 of 2 ak2(G) (re^2 + im^2); block b takes
// the rows [nstate b / kRedBlocks, nstate (b+1) / kRedBlocks), threads the G
// vectors of each row (a fixed order, no index division)
__global__ void __launch_bounds__(kRedThreads) k_ekin_part(const double *__restrict__ v, int nstate, int ncoef,
                                                           int ngp, const double *__restrict__ ak2,
                                                           double *__restrict__ part) {
  double s = 0.0;
  const int ng = ncoef - 1;
  const int r0 = (int)((long long)nstate * blockIdx.x / kRedBlocks);
  const int r1 = (int)((long long)nstate * (blockIdx.x + 1) / kRedBlocks);
  for (int st = r0; st < r1; st++) {
    const double *row = v + (size_t)st * 2 * ngp;
    for (int g = threadIdx.x; g < ng; g += kRedThreads) {
      const double re = row[g], im = row[ngp + g];
      s += 2.0 * ak2[g] * (re * re + im * im);
    }
  }
  block_sum_to(s, part + blockIdx.x);
}

// i G_d c: the orbital whose KB projection is dZ/dR_d (get_nlmat,
// energy/cp/cp_energy_eext_nonloc.c:648-748, accumulates the same sums with
// the factor G_d and the Re/Im roles swapped)
// grid (x: coefficient blocks, y: orbital rows); no index division
__global__ void k_dcoef(const double *__restrict__ v, int ncoef, int ngp, const double *__restrict__ gk,
                        double *__restrict__ out) {
  const double *row = v + (size_t)blockIdx.y * 2 * ngp;
  double *o = out + (size_t)blockIdx.y * 2 * ngp;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngp; g += gridDim.x * blockDim.x) {
    const bool in = g < ncoef - 1;
    const double k = in ? gk[g] : 0.0;
    const double re = in ? row[g] : 0.0, im = in ? row[ngp + g] : 0.0;
    o[g] = -k * im;
    o[ngp + g] = k * re;
  }
}

// one block per atom: the force component d of getnl_pot_pv_fatm ->
// sumnl_pot_pv_fatm_hess (cp_energy_eext_nonloc.c:1473-1500) over the merged
// projector rows (w carries vnorm / vol and the doubled weight of a merged
// conjugate pair, whose dZ obeys the same pairing as Z)
__global__ void __launch_bounds__(kRedThreads) k_nl_force_atoms(const double *__restrict__ Z0,
                                                                const double *__restrict__ Zd, int ldz,
                                                                const double *__restrict__ w,
                                                                const int *__restrict__ rs,
                                                                const int *__restrict__ rc, int nstate, double scale,
                                                                int d, double *__restrict__ f) {
  const int a = blockIdx.x, u0 = rs[a], nu = rc[a];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nu * nstate; i += kRedThreads) {
    const int s = i / nu, u = u0 + (i - s * nu);
    acc += w[u] * Z0[(size_t)s * ldz + u] * Zd[(size_t)s * ldz + u];
  }
  __shared__ double sh[kRedThreads];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int h = kRedThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) f[3 * a + d] = -2.0 * scale * sh[0];
}

inline int grid_for(int n) {
  int b = (n + 255) / 256;
  return b < 1 ? 1 : (b > 1024 ? 1024 : b);
}

}  // namespace

void launch_half_dot(const double *a, const double *b, int ncoef, int ngp, double *part, double *out,
                     cudaStream_t st) {
  k_hdot_part<<<kRedBlocks, kRedThreads, 0, st>>>(a, b, ncoef, ngp, part);
  k_sum_fixed<<<1, 32, 0, st>>>(part, kRedBlocks, out);
}

void launch_lz_hc(double *f, int ncoef, int ngp, cudaStream_t st) {
  k_lz_hc<<<grid_for(ncoef), 256, 0, st>>>(f, ncoef, ngp);
}

void launch_lz_w(double *h, const double *c, const double *p, const double *alpha, double beta, int ncoef, int ngp,
                 cudaStream_t st) {
  k_lz_w<<<grid_for(ncoef), 256, 0, st>>>(h, c, p, alpha, beta, ncoef, ngp);
}

void launch_lz_next(const double *w, double *c, double *p, double beta, int ncoef, int ngp, cudaStream_t st) {
  k_lz_next<<<grid_for(ncoef), 256, 0, st>>>(w, c, p, beta, ncoef, ngp);
}

void launch_lz_div(double *c, const double *nrm2, int ncoef, int ngp, cudaStream_t st) {
  k_lz_div<<<grid_for(ncoef), 256, 0, st>>>(c, nrm2, ncoef, ngp);
}

void launch_ekin(const double *v, int nstate, int ncoef, int ngp, const double *ak2, double *part, double *out,
                 cudaStream_t st) {
  k_ekin_part<<<kRedBlocks, kRedThreads, 0, st>>>(v, nstate, ncoef, ngp, ak2, part);
  k_sum_fixed<<<1, 32, 0, st>>>(part, kRedBlocks, out);
}

void launch_dcoef(const double *v, int nstate, int ncoef, int ngp, const double *gk, double *out, cudaStream_t st) {
  const int bx = std::min(8, (ngp + 255) / 256);
  for (int s0 = 0; s0 < nstate; s0 += 65535) {  // grid.y limit
    const int n = std::min(65535, nstate - s0);
    const size_t off = (size_t)s0 * 2 * ngp;
    k_dcoef<<<dim3(bx < 1 ? 1 : bx, n), 256, 0, st>>>(v + off, ncoef, ngp, gk, out + off);
  }
}

void launch_nl_force_atoms(const double *Z0, const double *Zd, int ldz, const double *w, const int *row_start,
                           const int *row_count, int natm, int nstate, double scale, int d, double *f,
                           cudaStream_t st) {
  k_nl_force_atoms<<<natm, kRedThreads, 0, st>>>(Z0, Zd, ldz, w, row_start, row_count, nstate, scale, d, f);
}

// Extreme eigenvalues of the symmetric tridiagonal matrix (diagonal a[0..n),
// off-diagonal b[0..n-1)) by Sturm-sequence bisection: count(x) = number of
// eigenvalues below x from the signs of the LDL^T pivots.
static int count_below(const double *a, const double *b, int n, double x) {
  int c = 0;
  double d = 1.0;
  for (int i = 0; i < n; i++) {
    const double off = i > 0 ? b[i - 1] * b[i - 1] : 0.0;
    d = (a[i] - x) - (i > 0 ? off / d : 0.0);
    if (d == 0.0) d = -1e-300;
    if (d < 0.0) c++;
  }
  return c;
}

void tridiag_extremes(const double *a, const double *b, int n, double *lo, double *hi) {
  double gl = a[0], gu = a[0];
  for (int i = 0; i < n; i++) {
    const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i < n - 1 ? fabs(b[i]) : 0.0);
    gl = fmin(gl, a[i] - r);
    gu = fmax(gu, a[i] + r);
  }
  const double pad = 1e-12 * fmax(1.0, fmax(fabs(gl), fabs(gu)));
  gl -= pad;
  gu += pad;
  for (int which = 0; which < 2; which++) {
    // smallest: largest x with count(x) == 0; largest: smallest x with count(x) == n
    double l = gl, u = gu;
    for (int it = 0; it < 200 && u - l > 0.0; it++) {
      const double m = 0.5 * (l + u);
      if (m <= l || m >= u) break;
      const int c = count_below(a, b, n, m);
      if (which == 0 ? c >= 1 : c >= n) u = m;
      else l = m;
    }
    (which == 0 ? *lo : *hi) = 0.5 * (l + u);
  }
}

}  // namespace sdft
