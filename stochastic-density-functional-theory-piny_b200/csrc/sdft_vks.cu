// sdft_vks.cu -- the Kohn-Sham potential from the stochastic density on the
// device: the density in G space (calcRhoStoRecipFullg, stodft/density.c:699),
// the Hartree and local-pseudopotential terms of cpGetVksStodft
// (stodft/reduced-energy/cp-energy-ee-rho-stodft.c:644-830), the LDA
// exchange-correlation step (sdft_xc.cu) and the transpose into the filter
// layout (:984-1007); and the local pseudopotential on the density sphere
// (controlEwdLocPreScf's vext loop, cp-energy-eext-stodft.c:340-470, for
// periodic cells and a splined short-range local potential).
//
// One handle (sdft_vks) holds a density grid: the half sphere of the density
// cutoff in PINY order with G = 0 last (setkvec3d), its grid positions, |G|^2,
// vext(G), and a complex FP64 work grid.  The steps of one call:
//   1. z(r) = rho_in(r) + 0 i, rho_in in the package layout (a fastest), the
//      density times the cell volume as calcRhoStoRecipFullg receives it;
//   2. three-axis FFT with exp(-i G.r) and 1/N (para_fft_gen3d_bck_to_g with
//      scale_opt 1; the sign is the one its code applies): rho(G) on the
//      half sphere;
//   3. E_H = 2 sum_{G!=0} 1/2 (4 pi / (|G|^2 vol)) |rho(G)|^2,
//      E_ext = 2 sum_{G!=0} Re(vext(G) conj-free dot rho(G)) + vext(0) rho(0),
//      V(G) = vext(G) + 4 pi rho(G) / (|G|^2 vol) (G != 0), V(0) = vext(0);
//   4. V(G) and its conjugate at -G on a zeroed grid, three-axis FFT with
//      exp(+i G.r), no scale (para_fft_gen3d_fwd_to_r), real part;
//   5. + V_xc(rho_in / vol) by PZ81 or PW92 (sdft_xc_lda_dev) when asked;
//   6. transpose to the filter layout, c fastest.
// Every reduction is a fixed-order sum over fixed blocks.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <vector>
#include "sdft_internal.h"
#include "sdft_fft.cuh"

struct sdft_vks {
  int device = 0;
  cudaStream_t st = nullptr;
  int n1 = 0, n2 = 0, n3 = 0;
  long long N = 0;
  int ncoef = 0;  // half sphere + G0 (last)
  double hmat[9] = {}, hmati[9] = {}, vol = 0.0;
  std::vector<int> ka, kb, kc;
  int *d_map = nullptr, *d_mapc = nullptr;  // package-layout grid index of G and -G
  double *d_ak2 = nullptr;                  // |G|^2 (G0: 0)
  double2 *d_vext = nullptr;                // vext(G), 0 until set_local
  double2 *d_vg = nullptr;                  // V(G) of the last call
  double2 *d_z = nullptr;                   // complex work grid [N]
  double *d_vpkg = nullptr, *d_nr = nullptr;  // V(r) package layout, rho_in / vol
  double2 *d_tw = nullptr;                  // exp(-2 pi i t / n_axis), n1 + n2 + n3
  double *d_part = nullptr;                 // reduction partials + results
  double *d_rhog = nullptr;                 // rho(G) re/im of the last call [2][ncoef]
  bool have_local = false, have_rho = false;
  // kept from sdft_vks_set_local for the atomic forces
  int natm = 0, ntype = 0;
  int *d_kabc = nullptr, *d_type = nullptr;  // [3 ncoef], [natm]
  double *d_frac = nullptr, *d_vgt = nullptr;  // [3 natm], [ntype][ncoef - 1]
};

namespace sdft {
namespace {

constexpr int kLines = 16, kFftThreads = 256, kGBlocks = 128, kGThreads = 256;

// One axis of the three-axis FFT: every CTA transforms kLines lines of
// length n held in shared memory (line pitch n + 1), in place, natural order
// in and out.  axis 0: lines along a (contiguous), line index b + n2 c;
// axis 1: lines along b, line (a, c), the CTA's lines are kLines consecutive
// a at one c; axis 2: lines along c, line (a, b) likewise.  Consecutive
// threads touch consecutive a, so global accesses are coalesced.
template <int DIR>
__global__ void __launch_bounds__(kFftThreads)
k_fft3_axis(double2 *__restrict__ z, int n1, int n2, int n3, int axis, const double2 *__restrict__ tw_g,
            double scale) {
  extern __shared__ __align__(16) double2 sm[];
  const int n = axis == 0 ? n1 : (axis == 1 ? n2 : n3);
  double2 *tw = sm;
  double2 *buf = sm + n;
  const int P = n + 1, tid = threadIdx.x;
  for (int t = tid; t < n; t += kFftThreads) tw[t] = tw_g[t];
  // line geometry
  long long base0 = 0, lstride = 0, estride = 0;
  int nl = kLines;
  if (axis == 0) {
    const long long l0 = (long long)blockIdx.x * kLines;
    const long long nlines = (long long)n2 * n3;
    nl = (int)min((long long)kLines, nlines - l0);
    base0 = l0 * n1; lstride = n1; estride = 1;
  } else {
    const int na = (n1 + kLines - 1) / kLines;
    const int a0 = (blockIdx.x % na) * kLines, o = blockIdx.x / na;
    nl = min(kLines, n1 - a0);
    lstride = 1;
    if (axis == 1) { base0 = a0 + (long long)n1 * n2 * o; estride = n1; }
    else { base0 = a0 + (long long)n1 * o; estride = (long long)n1 * n2; }
  }
  if (axis == 0) {
    for (int i = tid; i < nl * n; i += kFftThreads) {
      const int l = i / n, e = i - l * n;
      buf[l * P + e] = z[base0 + l * lstride + e];
    }
  } else {
    for (int i = tid; i < kLines * n; i += kFftThreads) {
      const int l = i % kLines, e = i / kLines;
      if (l < nl) buf[l * P + e] = z[base0 + l + e * estride];
    }
  }
  __syncthreads();
  const LineMap lm{nl, nl, P, 0, 1};
  fft_lines<DIR, (kLines * 128 + kFftThreads - 1) / kFftThreads>(buf, n, lm, tw, kFftThreads, tid);
  if (axis == 0) {
    for (int i = tid; i < nl * n; i += kFftThreads) {
      const int l = i / n, e = i - l * n;
      double2 v = buf[l * P + e];
      v.x *= scale; v.y *= scale;
      z[base0 + l * lstride + e] = v;
    }
  } else {
    for (int i = tid; i < kLines * n; i += kFftThreads) {
      const int l = i % kLines, e = i / kLines;
      if (l < nl) {
        double2 v = buf[l * P + e];
        v.x *= scale; v.y *= scale;
        z[base0 + l + e * estride] = v;
      }
    }
  }
}

__global__ void k_pack_real(const double *__restrict__ r, double2 *__restrict__ z, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = make_double2(r[i], 0.0);
}

// rho(G) from the transformed grid, the energies' block partials and V(G):
// part[b] = E_H half-sphere partial of block b, part[kGBlocks + b] = E_ext's.
__global__ void __launch_bounds__(kGThreads)
k_vks_gspace(const double2 *__restrict__ z, const int *__restrict__ map, const double *__restrict__ ak2,
             const double2 *__restrict__ vext, int ncoef, double vol, double2 *__restrict__ vg,
             double *__restrict__ rhog, double *__restrict__ part) {
  const double fpi = 4.0 * M_PI;
  const int nk = ncoef - 1;
  double eh = 0.0, ee = 0.0;
  for (int i = blockIdx.x * kGThreads + threadIdx.x; i < nk; i += kGBlocks * kGThreads) {
    const double2 r = z[map[i]];
    const double2 v = vext[i];
    const double gh = fpi / (ak2[i] * vol);
    eh += 0.5 * gh * (r.x * r.x + r.y * r.y);
    ee += v.x * r.x + v.y * r.y;
    vg[i] = make_double2(v.x + gh * r.x, v.y + gh * r.y);
    rhog[i] = r.x;
    rhog[ncoef + i] = r.y;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double r0 = z[map[nk]].x;
    vg[nk] = make_double2(vext[nk].x, 0.0);
    rhog[nk] = r0;
    rhog[ncoef + nk] = 0.0;
  }
  __shared__ double s0[kGThreads / 32], s1[kGThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    eh += __shfl_down_sync(0xffffffffu, eh, o);
    ee += __shfl_down_sync(0xffffffffu, ee, o);
  }
  if ((threadIdx.x & 31) == 0) { s0[threadIdx.x >> 5] = eh; s1[threadIdx.x >> 5] = ee; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < kGThreads / 32; w++) { a += s0[w]; b += s1[w]; }
    part[blockIdx.x] = a;
    part[kGBlocks + blockIdx.x] = b;
  }
}

// E_H = 2 sum, E_ext = 2 sum + vext(0) rho(0), in block order (one thread)
__global__ void k_vks_energies(const double *__restrict__ part, const double2 *__restrict__ vext,
                               const double *__restrict__ rhog, int ncoef, double *__restrict__ out) {
  double eh = 0.0, ee = 0.0;
  for (int b = 0; b < kGBlocks; b++) { eh += part[b]; ee += part[kGBlocks + b]; }
  out[0] = 2.0 * eh;
  out[1] = 2.0 * ee + vext[ncoef - 1].x * rhog[ncoef - 1];
}

__global__ void k_vks_scatter(const double2 *__restrict__ vg, const int *__restrict__ map,
                              const int *__restrict__ mapc, int ncoef, double2 *__restrict__ z) {
  const int nk = ncoef - 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncoef; i += gridDim.x * blockDim.x) {
    const double2 v = vg[i];
    z[map[i]] = v;
    if (i < nk) z[mapc[i]] = make_double2(v.x, -v.y);
  }
}

// V(r) = Re z (package layout) and rho_in / vol for the xc step
__global__ void k_vks_real(const double2 *__restrict__ z, const double *__restrict__ rho_in, double rvol,
                           double *__restrict__ v, double *__restrict__ nr, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    v[i] = z[i].x;
    nr[i] = rho_in[i] * rvol;
  }
}

// package layout (a fastest) -> filter layout (c fastest)
__global__ void k_pkg_to_filter(const double *__restrict__ v, double *__restrict__ out, int n1, int n2, int n3) {
  const long long N = (long long)n1 * n2 * n3;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int ic = (int)(i % n3);
    const long long ab = i / n3;
    const int ib = (int)(ab % n2), ia = (int)(ab / n2);
    out[i] = v[ia + (long long)n1 * (ib + (long long)n2 * ic)];
  }
}

// vext(G) = (1/vol) sum_a v_t(a)(|G|) (cos, -sin)(2 pi k . s_a) for G != 0 and
// (1/vol) sum_a gzvps_t(a) at G0 (cp-energy-eext-stodft.c:412-413, 449-455);
// vg_tab[t * (ncoef - 1) + i] = v_t(|G_i|) evaluated on the host.
__global__ void k_vext(const int *__restrict__ kabc, const double *__restrict__ frac, const int *__restrict__ type,
                       int natm, const double *__restrict__ vg_tab, const double *__restrict__ gzv, int ncoef,
                       double rvol, double2 *__restrict__ vext) {
  const int nk = ncoef - 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncoef; i += gridDim.x * blockDim.x) {
    if (i == nk) {
      double s = 0.0;
      for (int a = 0; a < natm; a++) s += gzv[type[a]];
      vext[i] = make_double2(s * rvol, 0.0);
      continue;
    }
    const double ka = kabc[3 * i], kb = kabc[3 * i + 1], kc = kabc[3 * i + 2];
    double sr = 0.0, si = 0.0;
    for (int a = 0; a < natm; a++) {
      const double arg = (ka * frac[3 * a] + kb * frac[3 * a + 1] + kc * frac[3 * a + 2]) * (2.0 * M_PI);
      double sn, cs;
      sincos(arg, &sn, &cs);
      const double v = vg_tab[(size_t)type[a] * nk + i];
      sr += cs * v;
      si += sn * v;
    }
    vext[i] = make_double2(sr * rvol, -si * rvol);
  }
}

struct Mat3 { double m[9]; };
constexpr int kFChunks = 8;

// Ewald structure factor of the charges per G != 0:
// ab[i] = 2 preg (Re S, Im S), S = sum_b q_b e^{i 2 pi k.s_b},
// preg = exp(-G^2 / 4 alp^2) 4 pi / (G^2 vol); part[b] = block b's sum of preg |S|^2
__global__ void __launch_bounds__(kGThreads)
k_ewald_sfac(const int *__restrict__ kabc, const double *__restrict__ frac, const double *__restrict__ q, int natm,
             int ncoef, Mat3 hi, double vol, double alp, double2 *__restrict__ ab, double *__restrict__ part) {
  const int nk = ncoef - 1;
  double vr = 0.0;
  for (int i = blockIdx.x * kGThreads + threadIdx.x; i < nk; i += kGBlocks * kGThreads) {
    const double ka = kabc[3 * i], kb = kabc[3 * i + 1], kc = kabc[3 * i + 2];
    const double xk = (ka * hi.m[0] + kb * hi.m[1] + kc * hi.m[2]) * (2.0 * M_PI);
    const double yk = (ka * hi.m[3] + kb * hi.m[4] + kc * hi.m[5]) * (2.0 * M_PI);
    const double zk = (ka * hi.m[6] + kb * hi.m[7] + kc * hi.m[8]) * (2.0 * M_PI);
    const double g2 = xk * xk + yk * yk + zk * zk;
    double sr = 0.0, si = 0.0;
    for (int b = 0; b < natm; b++) {
      double sn, cs;
      sincos((ka * frac[3 * b] + kb * frac[3 * b + 1] + kc * frac[3 * b + 2]) * (2.0 * M_PI), &sn, &cs);
      sr += q[b] * cs;
      si += q[b] * sn;
    }
    const double preg = exp(-g2 / (4.0 * alp * alp)) * 4.0 * M_PI / (g2 * vol);
    vr += preg * (sr * sr + si * si);
    ab[i] = make_double2(2.0 * preg * sr, 2.0 * preg * si);
  }
  __shared__ double s0[kGThreads / 32];
  for (int o = 16; o > 0; o >>= 1) vr += __shfl_down_sync(0xffffffffu, vr, o);
  if ((threadIdx.x & 31) == 0) s0[threadIdx.x >> 5] = vr;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < kGThreads / 32; w++) a += s0[w];
    part[blockIdx.x] = a;
  }
}

// Force partials: block (a, j) sums atom a's terms over G chunk j
// (control_ewd_loc's loop, energy/cp/cp_energy_eext.c:1120-1175):
//   vt = v_t(|G|) - 4 pi (q_a - q_pseud_t) / G^2,
//   F_a += G [(AB.x q_a + 2 rho_r vt / vol) sin(arg) - (AB.y q_a - 2 rho_i vt / vol) cos(arg)]
__global__ void __launch_bounds__(kGThreads)
k_loc_force(const int *__restrict__ kabc, const double *__restrict__ frac, const int *__restrict__ type,
            const double *__restrict__ q, const double *__restrict__ qps, int ncoef, Mat3 hi, double vol,
            const double *__restrict__ vgt, const double2 *__restrict__ ab, const double *__restrict__ rhog,
            double *__restrict__ fpart) {
  const int a = blockIdx.x, j = blockIdx.y, nk = ncoef - 1;
  const int t = type[a];
  const double qa = q[a], dq = q[a] - qps[t];
  const double sa = frac[3 * a], sb = frac[3 * a + 1], sc = frac[3 * a + 2];
  const int per = (nk + kFChunks - 1) / kFChunks;
  const int i0 = j * per, i1 = min(nk, i0 + per);
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int i = i0 + threadIdx.x; i < i1; i += kGThreads) {
    const double ka = kabc[3 * i], kb = kabc[3 * i + 1], kc = kabc[3 * i + 2];
    const double xk = (ka * hi.m[0] + kb * hi.m[1] + kc * hi.m[2]) * (2.0 * M_PI);
    const double yk = (ka * hi.m[3] + kb * hi.m[4] + kc * hi.m[5]) * (2.0 * M_PI);
    const double zk = (ka * hi.m[6] + kb * hi.m[7] + kc * hi.m[8]) * (2.0 * M_PI);
    const double g2 = xk * xk + yk * yk + zk * zk;
    const double vt = vgt[(size_t)t * nk + i] - 4.0 * M_PI * dq / g2;
    double sn, cs;
    sincos((ka * sa + kb * sb + kc * sc) * (2.0 * M_PI), &sn, &cs);
    const double2 s = ab[i];
    const double pr = s.x * qa + 2.0 * rhog[i] * vt / vol;
    const double pi = s.y * qa - 2.0 * rhog[ncoef + i] * vt / vol;
    const double w = pr * sn - pi * cs;
    fx += w * xk;
    fy += w * yk;
    fz += w * zk;
  }
  __shared__ double r[3][kGThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_down_sync(0xffffffffu, fx, o);
    fy += __shfl_down_sync(0xffffffffu, fy, o);
    fz += __shfl_down_sync(0xffffffffu, fz, o);
  }
  if ((threadIdx.x & 31) == 0) { r[0][threadIdx.x >> 5] = fx; r[1][threadIdx.x >> 5] = fy; r[2][threadIdx.x >> 5] = fz; }
  __syncthreads();
  if (threadIdx.x < 3) {
    double acc = 0.0;
    for (int w = 0; w < kGThreads / 32; w++) acc += r[threadIdx.x][w];
    fpart[((size_t)a * kFChunks + j) * 3 + threadIdx.x] = acc;
  }
}

// chunks of every atom summed in order; out[natm*3] then vrecip from part
__global__ void k_loc_force_sum(const double *__restrict__ fpart, int natm, const double *__restrict__ part,
                                double *__restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 3 * natm; e += gridDim.x * blockDim.x) {
    const int a = e / 3, d = e - 3 * a;
    double acc = 0.0;
    for (int j = 0; j < kFChunks; j++) acc += fpart[((size_t)a * kFChunks + j) * 3 + d];
    out[e] = acc;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double v = 0.0;
    for (int b = 0; b < kGBlocks; b++) v += part[b];
    out[3 * natm] = v;
  }
}

void inv3(const double *h, double *hi, double *det) {
  const double d = h[0] * (h[4] * h[8] - h[7] * h[5]) - h[3] * (h[1] * h[8] - h[7] * h[2]) +
                   h[6] * (h[1] * h[5] - h[4] * h[2]);
  hi[0] = (h[4] * h[8] - h[5] * h[7]) / d; hi[3] = (h[5] * h[6] - h[3] * h[8]) / d; hi[6] = (h[3] * h[7] - h[4] * h[6]) / d;
  hi[1] = (h[7] * h[2] - h[1] * h[8]) / d; hi[4] = (h[0] * h[8] - h[2] * h[6]) / d; hi[7] = (h[1] * h[6] - h[0] * h[7]) / d;
  hi[2] = (h[1] * h[5] - h[2] * h[4]) / d; hi[5] = (h[2] * h[3] - h[0] * h[5]) / d; hi[8] = (h[0] * h[4] - h[1] * h[3]) / d;
  *det = d;
}

bool edge_ok(int n) {
  if (n < 2 || n > 128) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

int fft3(sdft_vks *v, int dir, double scale) {
  const int ns[3] = {v->n1, v->n2, v->n3};
  const double2 *tw[3] = {v->d_tw, v->d_tw + v->n1, v->d_tw + v->n1 + v->n2};
  for (int axis = 0; axis < 3; axis++) {
    const int n = ns[axis];
    const long long nblk = axis == 0 ? ((long long)v->n2 * v->n3 + kLines - 1) / kLines
                                     : (long long)((v->n1 + kLines - 1) / kLines) * (axis == 1 ? v->n3 : v->n2);
    const size_t smem = sizeof(double2) * (size_t)(n + kLines * (n + 1));
    const double sc = axis == 2 ? scale : 1.0;
    if (dir > 0) k_fft3_axis<+1><<<(unsigned)nblk, kFftThreads, smem, v->st>>>(v->d_z, v->n1, v->n2, v->n3, axis, tw[axis], sc);
    else k_fft3_axis<-1><<<(unsigned)nblk, kFftThreads, smem, v->st>>>(v->d_z, v->n1, v->n2, v->n3, axis, tw[axis], sc);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SDFT_OK : set_error(SDFT_ERR_CUDA, cudaGetErrorString(e));
}

}  // namespace
}  // namespace sdft

using namespace sdft;

#define CKV(call)                                                                       \
  do {                                                                                  \
    cudaError_t e__ = (call);                                                           \
    if (e__ != cudaSuccess) return set_error(SDFT_ERR_CUDA, cudaGetErrorString(e__));   \
  } while (0)

extern "C" int sdft_vks_destroy(sdft_vks *v) {
  if (!v) return SDFT_OK;
  cudaSetDevice(v->device);
  void *ptrs[] = {v->d_map, v->d_mapc, v->d_ak2, v->d_vext, v->d_vg, v->d_z, v->d_vpkg, v->d_nr, v->d_tw, v->d_part,
                  v->d_rhog, v->d_kabc, v->d_type, v->d_frac, v->d_vgt};
  for (void *p : ptrs) dev_free(p, v->st);
  if (v->st) {
    cudaStreamSynchronize(v->st);
    cudaStreamDestroy(v->st);
  }
  delete v;
  return SDFT_OK;
}

extern "C" int sdft_vks_create(int n1, int n2, int n3, const double *hmat, int ncoef, const int *ka, const int *kb,
                               const int *kc, int device, sdft_vks **out) {
  if (!out || !hmat || !ka || !kb || !kc) return set_error(SDFT_ERR_ARG, "vks_create: null argument");
  *out = nullptr;
  if (!edge_ok(n1) || !edge_ok(n2) || !edge_ok(n3))
    return set_error(SDFT_ERR_UNSUPPORTED, "vks_create: grid edges must be 2^a 3^b in [2,128]");
  if (ncoef < 2) return set_error(SDFT_ERR_ARG, "vks_create: ncoef");
  if (ka[ncoef - 1] != 0 || kb[ncoef - 1] != 0 || kc[ncoef - 1] != 0)
    return set_error(SDFT_ERR_ARG, "vks_create: G=0 must be stored last");
  for (int i = 0; i < ncoef - 1; i++) {
    if (2 * std::abs(ka[i]) + 1 > n1 || 2 * std::abs(kb[i]) + 1 > n2 || 2 * std::abs(kc[i]) + 1 > n3)
      return set_error(SDFT_ERR_UNSUPPORTED, "vks_create: the density sphere does not fit the grid (|k| >= n/2)");
    const bool half = ka[i] > 0 || (ka[i] == 0 && kb[i] > 0) || (ka[i] == 0 && kb[i] == 0 && kc[i] > 0);
    if (!half) return set_error(SDFT_ERR_ARG, "vks_create: G list is not a half sphere");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(SDFT_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return set_error(SDFT_ERR_ARG, "vks_create: device index");
  sdft_vks *v = new sdft_vks();
  auto fail = [&](int code) { sdft_vks_destroy(v); return code; };
  v->device = device;
  v->n1 = n1; v->n2 = n2; v->n3 = n3;
  v->N = (long long)n1 * n2 * n3;
  v->ncoef = ncoef;
  for (int i = 0; i < 9; i++) v->hmat[i] = hmat[i];
  inv3(v->hmat, v->hmati, &v->vol);
  v->vol = std::fabs(v->vol);
  v->ka.assign(ka, ka + ncoef); v->kb.assign(kb, kb + ncoef); v->kc.assign(kc, kc + ncoef);
  if (cudaSetDevice(device) != cudaSuccess) return fail(set_error(SDFT_ERR_CUDA, "cudaSetDevice failed"));
  if (cudaStreamCreateWithFlags(&v->st, cudaStreamNonBlocking) != cudaSuccess)
    return fail(set_error(SDFT_ERR_CUDA, "stream create failed"));
  // grid positions (package layout, a fastest) of G and -G; |G|^2 (hmat
  // columns are the cell vectors, column-major: G = 2 pi k h^-1)
  std::vector<int> map(ncoef), mapc(ncoef);
  std::vector<double> ak2(ncoef);
  auto w = [](int k, int n) { return k < 0 ? k + n : k; };
  const double tpi = 2.0 * M_PI;
  const double *hi = v->hmati;
  for (int i = 0; i < ncoef; i++) {
    map[i] = w(ka[i], n1) + n1 * (w(kb[i], n2) + n2 * w(kc[i], n3));
    mapc[i] = w(-ka[i], n1) + n1 * (w(-kb[i], n2) + n2 * w(-kc[i], n3));
    const double a = ka[i], b = kb[i], c = kc[i];
    const double xk = (a * hi[0] + b * hi[1] + c * hi[2]) * tpi, yk = (a * hi[3] + b * hi[4] + c * hi[5]) * tpi,
                 zk = (a * hi[6] + b * hi[7] + c * hi[8]) * tpi;
    ak2[i] = xk * xk + yk * yk + zk * zk;
  }
  ak2[ncoef - 1] = 0.0;
  std::vector<double2> tw(n1 + n2 + n3);
  {
    int off = 0;
    for (int n : {n1, n2, n3}) {
      for (int t = 0; t < n; t++) tw[off + t] = make_double2(std::cos(tpi * t / n), -std::sin(tpi * t / n));
      off += n;
    }
  }
  int r;
#define DMV(p, bytes)                                                              \
  do {                                                                             \
    if ((r = dev_alloc(device, v->st, (void **)&(p), (bytes)))) return fail(r);    \
  } while (0)
  DMV(v->d_map, ncoef * sizeof(int));
  DMV(v->d_mapc, ncoef * sizeof(int));
  DMV(v->d_ak2, ncoef * sizeof(double));
  DMV(v->d_vext, ncoef * sizeof(double2));
  DMV(v->d_vg, ncoef * sizeof(double2));
  DMV(v->d_z, v->N * sizeof(double2));
  DMV(v->d_vpkg, v->N * sizeof(double));
  DMV(v->d_nr, v->N * sizeof(double));
  DMV(v->d_tw, tw.size() * sizeof(double2));
  DMV(v->d_part, (2 * kGBlocks + 8) * sizeof(double));
  DMV(v->d_rhog, 2 * (size_t)ncoef * sizeof(double));
#undef DMV
  auto ck = [&](cudaError_t e) { return e == cudaSuccess ? SDFT_OK : set_error(SDFT_ERR_CUDA, cudaGetErrorString(e)); };
  if ((r = ck(cudaMemcpyAsync(v->d_map, map.data(), ncoef * sizeof(int), cudaMemcpyHostToDevice, v->st))) ||
      (r = ck(cudaMemcpyAsync(v->d_mapc, mapc.data(), ncoef * sizeof(int), cudaMemcpyHostToDevice, v->st))) ||
      (r = ck(cudaMemcpyAsync(v->d_ak2, ak2.data(), ncoef * sizeof(double), cudaMemcpyHostToDevice, v->st))) ||
      (r = ck(cudaMemcpyAsync(v->d_tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, v->st))) ||
      (r = ck(cudaMemsetAsync(v->d_vext, 0, ncoef * sizeof(double2), v->st))) ||
      (r = ck(cudaStreamSynchronize(v->st))))
    return fail(r);
  {
    const size_t smax = sizeof(double2) * (size_t)(128 + kLines * 129);
    if ((r = ck(cudaFuncSetAttribute(k_fft3_axis<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax))) ||
        (r = ck(cudaFuncSetAttribute(k_fft3_axis<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax))))
      return fail(r);
  }
  *out = v;
  return SDFT_OK;
}

extern "C" int sdft_vks_set_local(sdft_vks *v, int natm, const double *pos, int ntype, const int *type, int nsplin,
                                  double gmin_spl, double dg_spl, const double *vloc, const double *gzvps) {
  if (!v || natm < 1 || !pos || ntype < 1 || !type || nsplin < 1 || dg_spl <= 0.0 || !vloc || !gzvps)
    return set_error(SDFT_ERR_ARG, "vks_set_local: bad argument");
  for (int a = 0; a < natm; a++)
    if (type[a] < 0 || type[a] >= ntype) return set_error(SDFT_ERR_ARG, "vks_set_local: atom type out of range");
  cudaSetDevice(v->device);
  const int nk = v->ncoef - 1;
  // v_t(|G|) by get_vpsnow's cubic form on the per-knot Taylor table
  // (energy/cp/cp_energy_eext.c:2139-2185): vloc[(t*4 + d)*nsplin + knot]
  std::vector<double> vg((size_t)ntype * std::max(nk, 1));
  const double tpi = 2.0 * M_PI;
  const double *hi = v->hmati;
  for (int i = 0; i < nk; i++) {
    const double a = v->ka[i], b = v->kb[i], c = v->kc[i];
    const double xk = (a * hi[0] + b * hi[1] + c * hi[2]) * tpi, yk = (a * hi[3] + b * hi[4] + c * hi[5]) * tpi,
                 zk = (a * hi[6] + b * hi[7] + c * hi[8]) * tpi;
    const double g = std::sqrt(xk * xk + yk * yk + zk * zk);
    int iii = (int)((g - gmin_spl) / dg_spl) + 1;
    if (iii > nsplin) iii = nsplin;
    if (iii < 1) iii = 1;
    const double h = g - ((double)(iii - 1) * dg_spl + gmin_spl);
    for (int t = 0; t < ntype; t++) {
      const double *tab = vloc + (size_t)t * 4 * nsplin;
      const int k = iii - 1;
      vg[(size_t)t * nk + i] = ((tab[3 * nsplin + k] * h + tab[2 * nsplin + k]) * h + tab[nsplin + k]) * h + tab[k];
    }
  }
  // fractional coordinates s = h^-1 r (ewd_scr_x/y/z of the reference)
  std::vector<double> frac(3 * (size_t)natm);
  for (int a = 0; a < natm; a++) {
    const double x = pos[3 * a], y = pos[3 * a + 1], z = pos[3 * a + 2];
    const double s[3] = {x * hi[0] + y * hi[3] + z * hi[6], x * hi[1] + y * hi[4] + z * hi[7],
                         x * hi[2] + y * hi[5] + z * hi[8]};
    for (int d = 0; d < 3; d++) frac[3 * a + d] = s[d];
  }
  std::vector<int> kabc(3 * (size_t)v->ncoef);
  for (int i = 0; i < v->ncoef; i++) { kabc[3 * i] = v->ka[i]; kabc[3 * i + 1] = v->kb[i]; kabc[3 * i + 2] = v->kc[i]; }
  int *d_k = nullptr, *d_t = nullptr;
  double *d_f = nullptr, *d_vg = nullptr, *d_gz = nullptr;
  int r = SDFT_OK;
  auto ck = [&](cudaError_t e) { return e == cudaSuccess ? SDFT_OK : set_error(SDFT_ERR_CUDA, cudaGetErrorString(e)); };
  if (!(r = dev_alloc(v->device, v->st, (void **)&d_k, kabc.size() * sizeof(int))) &&
      !(r = dev_alloc(v->device, v->st, (void **)&d_t, natm * sizeof(int))) &&
      !(r = dev_alloc(v->device, v->st, (void **)&d_f, frac.size() * sizeof(double))) &&
      !(r = dev_alloc(v->device, v->st, (void **)&d_vg, vg.size() * sizeof(double))) &&
      !(r = dev_alloc(v->device, v->st, (void **)&d_gz, ntype * sizeof(double))) &&
      !(r = ck(cudaMemcpyAsync(d_k, kabc.data(), kabc.size() * sizeof(int), cudaMemcpyHostToDevice, v->st))) &&
      !(r = ck(cudaMemcpyAsync(d_t, type, natm * sizeof(int), cudaMemcpyHostToDevice, v->st))) &&
      !(r = ck(cudaMemcpyAsync(d_f, frac.data(), frac.size() * sizeof(double), cudaMemcpyHostToDevice, v->st))) &&
      !(r = ck(cudaMemcpyAsync(d_vg, vg.data(), vg.size() * sizeof(double), cudaMemcpyHostToDevice, v->st))) &&
      !(r = ck(cudaMemcpyAsync(d_gz, gzvps, ntype * sizeof(double), cudaMemcpyHostToDevice, v->st)))) {
    const int blocks = (int)std::min<long long>((v->ncoef + 255) / 256, 148 * 8);
    k_vext<<<blocks, 256, 0, v->st>>>(d_k, d_f, d_t, natm, d_vg, d_gz, v->ncoef, 1.0 / v->vol, v->d_vext);
    r = ck(cudaGetLastError());
    if (!r) r = ck(cudaStreamSynchronize(v->st));
  }
  dev_free(d_gz, v->st);
  if (r) {
    for (void *p : {(void *)d_k, (void *)d_t, (void *)d_f, (void *)d_vg}) dev_free(p, v->st);
    cudaStreamSynchronize(v->st);
    return r;
  }
  // the atoms and the radial values stay for sdft_vks_local_forces
  for (void *p : {(void *)v->d_kabc, (void *)v->d_type, (void *)v->d_frac, (void *)v->d_vgt}) dev_free(p, v->st);
  v->d_kabc = d_k; v->d_type = d_t; v->d_frac = d_f; v->d_vgt = d_vg;
  v->natm = natm; v->ntype = ntype;
  cudaStreamSynchronize(v->st);
  v->have_local = true;
  return SDFT_OK;
}

extern "C" int sdft_vks_local_forces(sdft_vks *v, const double *q, const double *q_pseud, double alp_ewd,
                                     double *force, double *ewald) {
  if (!v || !q || !q_pseud || !force || !ewald || !(alp_ewd > 0.0))
    return set_error(SDFT_ERR_ARG, "vks_local_forces: bad argument");
  if (!v->have_local || !v->have_rho)
    return set_error(SDFT_ERR_STATE, "vks_local_forces: needs sdft_vks_set_local and sdft_vks_from_rho first");
  cudaSetDevice(v->device);
  const int natm = v->natm;
  const int nk = v->ncoef - 1;
  double *d_q = nullptr, *d_qp = nullptr, *d_fp = nullptr, *d_out = nullptr;
  double2 *d_ab = nullptr;
  int r = SDFT_OK;
  auto ck = [&](cudaError_t e) { return e == cudaSuccess ? SDFT_OK : set_error(SDFT_ERR_CUDA, cudaGetErrorString(e)); };
  std::vector<double> out(3 * (size_t)natm + 1);
  Mat3 hi;
  for (int i = 0; i < 9; i++) hi.m[i] = v->hmati[i];
  if (!(r = dev_alloc(v->device, v->st, (void **)&d_q, natm * sizeof(double))) &&
      !(r = dev_alloc(v->device, v->st, (void **)&d_qp, v->ntype * sizeof(double))) &&
      !(r = dev_alloc(v->device, v->st, (void **)&d_ab, std::max(nk, 1) * sizeof(double2))) &&
      !(r = dev_alloc(v->device, v->st, (void **)&d_fp, (size_t)natm * kFChunks * 3 * sizeof(double))) &&
      !(r = dev_alloc(v->device, v->st, (void **)&d_out, out.size() * sizeof(double))) &&
      !(r = ck(cudaMemcpyAsync(d_q, q, natm * sizeof(double), cudaMemcpyHostToDevice, v->st))) &&
      !(r = ck(cudaMemcpyAsync(d_qp, q_pseud, v->ntype * sizeof(double), cudaMemcpyHostToDevice, v->st)))) {
    k_ewald_sfac<<<kGBlocks, kGThreads, 0, v->st>>>(v->d_kabc, v->d_frac, d_q, natm, v->ncoef, hi, v->vol, alp_ewd,
                                                   d_ab, v->d_part);
    k_loc_force<<<dim3(natm, kFChunks), kGThreads, 0, v->st>>>(v->d_kabc, v->d_frac, v->d_type, d_q, d_qp, v->ncoef,
                                                               hi, v->vol, v->d_vgt, d_ab, v->d_rhog, d_fp);
    k_loc_force_sum<<<(3 * natm + 255) / 256, 256, 0, v->st>>>(d_fp, natm, v->d_part, d_out);
    r = ck(cudaGetLastError());
    if (!r) r = ck(cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, v->st));
    if (!r) r = ck(cudaStreamSynchronize(v->st));
  }
  for (void *p : {(void *)d_q, (void *)d_qp, (void *)d_ab, (void *)d_fp, (void *)d_out}) dev_free(p, v->st);
  cudaStreamSynchronize(v->st);
  if (r) return r;
  for (int i = 0; i < 3 * natm; i++) force[i] = out[i];
  // ewald3d_selfbgr_cp (energy/cp/cp_energy_eext.c:2200), self_erf = 1
  double sq = 0.0, sq2 = 0.0;
  for (int a = 0; a < natm; a++) { sq += q[a]; sq2 += q[a] * q[a]; }
  ewald[0] = out[3 * (size_t)natm];
  ewald[1] = -sq2 * alp_ewd / std::sqrt(M_PI);
  ewald[2] = -0.5 * sq * sq * M_PI / (alp_ewd * alp_ewd * v->vol);
  return SDFT_OK;
}

extern "C" int sdft_vks_from_rho(sdft_vks *v, const double *rho, int xc_kind, double *vks_filter, double *rho_g,
                                 double *energies) {
  if (!v || !rho || !vks_filter) return set_error(SDFT_ERR_ARG, "vks_from_rho: null argument");
  if (xc_kind != 0 && xc_kind != SDFT_XC_PZ_LDA && xc_kind != SDFT_XC_PW_LDA)
    return set_error(SDFT_ERR_ARG, "vks_from_rho: xc_kind 0, SDFT_XC_PZ_LDA or SDFT_XC_PW_LDA");
  if (!v->have_local) return set_error(SDFT_ERR_STATE, "vks_from_rho: local potential not set (sdft_vks_set_local)");
  cudaSetDevice(v->device);
  const long long N = v->N;
  const int blocks = (int)std::min<long long>((N + 255) / 256, 148 * 8);
  // rho may be host or device memory: stage it in the real-space buffer
  CKV(cudaMemcpyAsync(v->d_nr, rho, N * sizeof(double), cudaMemcpyDefault, v->st));
  k_pack_real<<<blocks, 256, 0, v->st>>>(v->d_nr, v->d_z, N);
  int r;
  if ((r = fft3(v, -1, 1.0 / (double)N))) return r;
  k_vks_gspace<<<kGBlocks, kGThreads, 0, v->st>>>(v->d_z, v->d_map, v->d_ak2, v->d_vext, v->ncoef, v->vol, v->d_vg,
                                                 v->d_rhog, v->d_part);
  k_vks_energies<<<1, 1, 0, v->st>>>(v->d_part, v->d_vext, v->d_rhog, v->ncoef, v->d_part + 2 * kGBlocks);
  CKV(cudaMemsetAsync(v->d_z, 0, N * sizeof(double2), v->st));
  k_vks_scatter<<<(int)std::min(((long long)v->ncoef + 255) / 256, 148LL * 8), 256, 0, v->st>>>(
      v->d_vg, v->d_map, v->d_mapc, v->ncoef, v->d_z);
  if ((r = fft3(v, +1, 1.0))) return r;
  // d_nr held rho_in; V(r) into d_vpkg, rho_in / vol back into d_nr
  k_vks_real<<<blocks, 256, 0, v->st>>>(v->d_z, v->d_nr, 1.0 / v->vol, v->d_vpkg, v->d_nr, N);
  CKV(cudaGetLastError());
  double e[4] = {0.0, 0.0, 0.0, 0.0};
  if (xc_kind) {
    if ((r = sdft_xc_lda_dev(xc_kind, N, v->d_nr, v->d_vpkg, v->vol, &e[2], &e[3], v->st))) return r;
  }
  // into the filter layout: the caller's buffer directly when it is device
  // memory, else through the work grid (free again at this point)
  cudaPointerAttributes at{};
  const bool dev_out = cudaPointerGetAttributes(&at, vks_filter) == cudaSuccess &&
                       (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  double *dst = dev_out ? vks_filter : reinterpret_cast<double *>(v->d_z);
  k_pkg_to_filter<<<blocks, 256, 0, v->st>>>(v->d_vpkg, dst, v->n1, v->n2, v->n3);
  CKV(cudaGetLastError());
  if (!dev_out) CKV(cudaMemcpyAsync(vks_filter, dst, N * sizeof(double), cudaMemcpyDeviceToHost, v->st));
  if (rho_g) CKV(cudaMemcpyAsync(rho_g, v->d_rhog, 2 * (size_t)v->ncoef * sizeof(double), cudaMemcpyDefault, v->st));
  CKV(cudaMemcpyAsync(e, v->d_part + 2 * kGBlocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, v->st));
  CKV(cudaStreamSynchronize(v->st));
  v->have_rho = true;
  if (energies) for (int i = 0; i < 4; i++) energies[i] = e[i];
  return SDFT_OK;
}

extern "C" int sdft_vks_get_vext(sdft_vks *v, double *re, double *im) {
  if (!v || !re || !im) return set_error(SDFT_ERR_ARG, "vks_get_vext: null argument");
  cudaSetDevice(v->device);
  std::vector<double2> h(v->ncoef);
  CKV(cudaMemcpyAsync(h.data(), v->d_vext, v->ncoef * sizeof(double2), cudaMemcpyDeviceToHost, v->st));
  CKV(cudaStreamSynchronize(v->st));
  for (int i = 0; i < v->ncoef; i++) { re[i] = h[i].x; im[i] = h[i].y; }
  return SDFT_OK;
}

// ---------------------------------------------------------------------------
// Real-space ion-ion Ewald sum (the part of calcEnergyForce's nuclear force
// that calc-nuclei-force.c:605/635 gets from PINY's pair engine,
// energy_control_inter_real, over the vcoul_bin table).  The pair term is
// vcoul_bin's (interface/inter_params/spline_fit.c:415-437, iperd > 0) with
// spline_vdv's shift or switch (:61-72, :87-92), evaluated at each distance
// in FP64 instead of interpolated from a table:
//   v = qq gerfc(alp r)/r,  dv = -(dv/dr)/r = (gerfc/r^2 + dgerfc/r) qq/r,
//   gerfc(x) = sum_i e_i t^i exp(-x^2), t = 1/(1 + p x)  (the reference's fit
//   of erfc, within 2.3e-9 of it).
// One CTA per atom a sums its pairs (b, image n) over a fixed thread split and
// reduces them in a fixed order, so results are reproducible.
// ---------------------------------------------------------------------------
namespace sdft {
namespace {
constexpr int kEwThreads = 256;
// the fit's constants, spline_fit.c:373-376
__device__ __forceinline__ void gerfc_fit(double x, double alp, double r, double &g, double &dg) {
  constexpr double p = 0.3614;
  constexpr double e[9] = {0.2041422096422003, 0.1997535956961481, 0.2213176596405576, 0.03360430734640255,
                           0.4732592578721755, -0.509078520069735,  0.6772631491947646, -0.369912979092217,
                           0.06965131976970335};
  const double ex = exp(-x * x);
  const double t = 1.0 / (1.0 + p * x);
  double poly = 0.0, dpoly = 0.0;
#pragma unroll
  for (int i = 9; i >= 1; i--) {
    poly = poly * t + e[i - 1];
    dpoly = dpoly * t + i * e[i - 1];
  }
  g = poly * t * ex;
  dg = dpoly * t * t * ex * p * alp + 2.0 * alp * alp * g * r;
}

__global__ void __launch_bounds__(kEwThreads)
k_ewald_real(const double *__restrict__ x, const double *__restrict__ q, int natm, const double *__restrict__ img,
             int nimg, double alp, double rmax, int ishift, double rheal, double vshift, double *__restrict__ force,
             double *__restrict__ epart) {
  const int a = blockIdx.x;
  const double xa = x[3 * a], ya = x[3 * a + 1], za = x[3 * a + 2], qa = q[a];
  const double rmax2 = rmax * rmax;
  double fx = 0.0, fy = 0.0, fz = 0.0, en = 0.0;
  const long long tot = (long long)natm * nimg;
  for (long long t = threadIdx.x; t < tot; t += kEwThreads) {
    const int b = (int)(t / nimg), m = (int)(t - (long long)b * nimg);
    if (b == a && m == 0) continue;  // image 0 is n = 0
    const double dx = xa - x[3 * b] - img[3 * m], dy = ya - x[3 * b + 1] - img[3 * m + 1],
                 dz = za - x[3 * b + 2] - img[3 * m + 2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= rmax2) continue;
    const double r = sqrt(r2), qq = qa * q[b];
    double g, dg;
    gerfc_fit(r * alp, alp, r, g, dg);
    double v = qq * g / r;
    double dv = (g / r2 + dg / r) * qq / r;
    if (ishift == 2) {
      double rp = (r - rmax + rheal) / rheal;
      rp = fmin(fmax(rp, 0.0), 1.0);
      const double sw = 1.0 + rp * rp * (2.0 * rp - 3.0);
      const double dsw = -6.0 * (rp / rheal) * (rp - 1.0) / r;
      dv = dv * sw + v * dsw;
      v = v * sw;
    } else if (ishift == 1) {
      v -= qq * vshift;
    }
    en += 0.5 * v;
    fx += dv * dx;
    fy += dv * dy;
    fz += dv * dz;
  }
  __shared__ double red[kEwThreads / 32][4];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_down_sync(0xffffffffu, fx, o);
    fy += __shfl_down_sync(0xffffffffu, fy, o);
    fz += __shfl_down_sync(0xffffffffu, fz, o);
    en += __shfl_down_sync(0xffffffffu, en, o);
  }
  if ((threadIdx.x & 31) == 0) {
    const int w = threadIdx.x >> 5;
    red[w][0] = fx; red[w][1] = fy; red[w][2] = fz; red[w][3] = en;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < kEwThreads / 32; w++)
      for (int c = 0; c < 4; c++) s[c] += red[w][c];
    force[3 * a] = s[0]; force[3 * a + 1] = s[1]; force[3 * a + 2] = s[2];
    epart[a] = s[3];
  }
}

double gerfc_host(double x) {  // the same fit on the host (the ishift 1 shift)
  const double p = 0.3614;
  const double e[9] = {0.2041422096422003, 0.1997535956961481, 0.2213176596405576, 0.03360430734640255,
                       0.4732592578721755, -0.509078520069735,  0.6772631491947646, -0.369912979092217,
                       0.06965131976970335};
  const double t = 1.0 / (1.0 + p * x);
  double poly = 0.0;
  for (int i = 9; i >= 1; i--) poly = poly * t + e[i - 1];
  return poly * t * std::exp(-x * x);
}
}  // namespace
}  // namespace sdft

extern "C" int sdft_ewald_real(int natm, const double *pos, const double *q, const double *hmat, double alp_ewd,
                               double rmax, int ishift, double rheal, double *force, double *energy, void *stream) {
  if (natm < 1 || !pos || !q || !hmat || !force || !energy || !(alp_ewd > 0.0) || !(rmax > 0.0) || ishift < 0 ||
      ishift > 2 || (ishift == 2 && !(rheal > 0.0 && rheal <= rmax)))
    return set_error(SDFT_ERR_ARG, "ewald_real: bad argument");
  double hi[9], vol;
  inv3(hmat, hi, &vol);
  vol = std::fabs(vol);
  if (!(vol > 0.0)) return set_error(SDFT_ERR_ARG, "ewald_real: singular cell");
  // positions wrapped into the cell; lattice translations h n with |n_i| <=
  // ceil(rmax / w_i) + 1 (w_i the width across face i), n = 0 first
  std::vector<double> x(3 * (size_t)natm);
  for (int a = 0; a < natm; a++) {
    double s[3];
    for (int i = 0; i < 3; i++) {
      s[i] = pos[3 * a] * hi[i] + pos[3 * a + 1] * hi[i + 3] + pos[3 * a + 2] * hi[i + 6];
      s[i] -= std::floor(s[i]);
    }
    for (int i = 0; i < 3; i++) x[3 * a + i] = hmat[i] * s[0] + hmat[i + 3] * s[1] + hmat[i + 6] * s[2];
  }
  int nmax[3];
  for (int j = 0; j < 3; j++) {
    const double *u = hmat + 3 * ((j + 1) % 3), *w = hmat + 3 * ((j + 2) % 3);
    const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
    const double width = vol / std::sqrt(cx * cx + cy * cy + cz * cz);
    const double n = std::ceil(rmax / width) + 1.0;
    if (n > 16.0) return set_error(SDFT_ERR_ARG, "ewald_real: cutoff spans more than 16 cells");
    nmax[j] = (int)n;
  }
  std::vector<double> img(3, 0.0);
  for (int i = -nmax[0]; i <= nmax[0]; i++)
    for (int j = -nmax[1]; j <= nmax[1]; j++)
      for (int k = -nmax[2]; k <= nmax[2]; k++) {
        if (!i && !j && !k) continue;
        for (int c = 0; c < 3; c++) img.push_back(hmat[c] * i + hmat[c + 3] * j + hmat[c + 6] * k);
      }
  const int nimg = (int)(img.size() / 3);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(SDFT_ERR_NODEVICE, "ewald_real: no device");
  const size_t bytes = (x.size() + natm + img.size() + 4 * (size_t)natm) * sizeof(double);
  void *buf = nullptr;
  int r = dev_alloc(dev, stream, &buf, bytes);
  if (r) return r;
  double *d_x = static_cast<double *>(buf), *d_q = d_x + x.size(), *d_img = d_q + natm, *d_f = d_img + img.size(),
         *d_e = d_f + 3 * (size_t)natm;
  std::vector<double> ep(natm);
  cudaError_t e = cudaMemcpyAsync(d_x, x.data(), x.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_q, q, natm * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_img, img.data(), img.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_ewald_real<<<natm, kEwThreads, 0, st>>>(d_x, d_q, natm, d_img, nimg, alp_ewd, rmax, ishift, rheal,
                                              gerfc_host(alp_ewd * rmax) / rmax, d_f, d_e);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(force, d_f, 3 * (size_t)natm * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ep.data(), d_e, natm * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  dev_free(buf, stream);
  if (e != cudaSuccess) return set_error(SDFT_ERR_CUDA, cudaGetErrorString(e));
  double s = 0.0;
  for (int a = 0; a < natm; a++) s += ep[a];
  *energy = s;
  return SDFT_OK;
}
