// sdft_kernels.cu -- sm_100a kernels of the stochastic-DFT filter hot path.
//
// One application of H to a block of orbitals is split into
//   stage A  (per orbital pair x column batch): sphere -> columns pack of
//            dble_pack_coef_fftw3d_filter (mathlib/fft_package.c:3195-3259),
//            backward FFT along c over the occupied (ka,kb) columns only;
//   stage B  (per pair x c-plane): backward FFT along b (occupied ka rows)
//            and a, multiply by V_KS (cp_vpsi, energy/cp/cp_energy_ee_rho.c:2790),
//            forward FFT along a and b;
//   stage C  (per pair x column batch): forward FFT along c, unpack of
//            dble_upack_coef_sum_fftw3d_filter (mathlib/fft_package.c:3513-3600)
//            fused with the kinetic term (stodft/reduced-energy/
//            cp-energy-ee-rho-stodft.c:308-320), the KB force, the normalised-H
//            scaling / Chebyshev or Newton recurrence (stodft/normh.c:35-344),
//            the filter accumulation (stodft/filter.c:596-612) and the moment
//            dots (stodft/calc-chempot-chebyshev.c:722-842).
// The KB projection / back projection run as DMMA FP64 GEMMs.
#include <cuda_runtime.h>
#include <cstdio>
#include "sdft_fft.cuh"
#include "sdft_internal.h"
#include "sdft_kernels.cuh"

namespace sdft {

template <typename T> __device__ __forceinline__ const typename CT<T>::type *tw_ptr(const DevGeom &g, int dim);
template <> __device__ __forceinline__ const double2 *tw_ptr<double>(const DevGeom &g, int dim) {
  return dim == 1 ? g.tw1 : (dim == 2 ? g.tw2 : g.tw3);
}
template <> __device__ __forceinline__ const float2 *tw_ptr<float>(const DevGeom &g, int dim) {
  return dim == 1 ? g.tw1f : (dim == 2 ? g.tw2f : g.tw3f);
}

// ============================================================================
// Stage A: pack + backward c-FFT over the columns of kCPB mirror pairs.
// ============================================================================
template <typename T>
__global__ void __launch_bounds__(kColThreads)
k_stage_a(DevGeom g, const double *__restrict__ C, int nstate, int pair0,
          typename CT<T>::type *__restrict__ X) {
  using C2 = typename CT<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tw = reinterpret_cast<C2 *>(smem_raw);
  C2 *buf = tw + g.n3;
  const int P3 = g.n3 + 1;
  const int tid = threadIdx.x;
  const int cp0 = blockIdx.x * kCPB;
  const int cp1 = min(cp0 + kCPB, g.ncp);
  const int col0 = 2 * cp0;
  const int ncl = min(2 * cp1, g.ncols) - col0;
  const int p = pair0 + blockIdx.y;
  const int s1 = 2 * p, s2 = 2 * p + 1;
  const bool has2 = s2 < nstate;
  const C2 *twg = tw_ptr<T>(g, 3);
  for (int t = tid; t < g.n3; t += blockDim.x) tw[t] = twg[t];
  for (int i = tid; i < ncl * P3; i += blockDim.x) buf[i] = cmk<C2>(0.0, 0.0);
  __syncthreads();
  const size_t o1 = (size_t)s1 * 2 * g.ngp, o2 = (size_t)s2 * 2 * g.ngp;
  const int warp = tid >> 5, lane = tid & 31;
  for (int cp = cp0 + warp; cp < cp1; cp += kColThreads / 32) {
    const int lc = 2 * (cp - cp0);
    const bool zc = (cp == g.ncp - 1);
    const int lm = zc ? lc : lc + 1;
    const int gs = g.cp_gstart[cp], gc = g.cp_gcount[cp];
    for (int e = lane; e < gc; e += 32) {
      const int gi = gs + e;
      const int kc = g.gkc[gi];
      const double a = C[o1 + gi], b = C[o1 + g.ngp + gi];
      const double c = has2 ? C[o2 + gi] : 0.0, d = has2 ? C[o2 + g.ngp + gi] : 0.0;
      const int kd = kc < 0 ? kc + g.n3 : kc;
      const int km = kc > 0 ? g.n3 - kc : -kc;
      buf[lc * P3 + kd] = cmk<C2>(a - d, b + c);
      buf[lm * P3 + km] = cmk<C2>(a + d, -b + c);
    }
    if (zc && lane == 0) {
      const int g0 = g.ncoef - 1;
      buf[lc * P3] = cmk<C2>(C[o1 + g0], has2 ? C[o2 + g0] : 0.0);
    }
  }
  __syncthreads();
  LineMap lmap{ncl, ncl, P3, 0, 1};
  fft_lines<+1, (2 * kCPB * kMaxEdge + kColThreads - 1) / kColThreads>(buf, g.n3, lmap, tw, blockDim.x, tid);
  C2 *Xp = X + (size_t)blockIdx.y * g.n3 * g.ncols_pad;
  for (int i = tid; i < g.n3 * ncl; i += blockDim.x) {
    const int ic = i / ncl, cl = i - ic * ncl;
    Xp[(size_t)ic * g.ncols_pad + col0 + cl] = buf[cl * P3 + ic];
  }
}

// ============================================================================
// Stage B: one c-plane of one pair: b/a backward FFT, x V, a/b forward FFT.
// ============================================================================
template <typename T, int NT, int MAXE>
__global__ void __launch_bounds__(NT, 1)
k_stage_b(DevGeom g, typename CT<T>::type *__restrict__ X, const T *__restrict__ Vp) {
  using C2 = typename CT<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tw1 = reinterpret_cast<C2 *>(smem_raw);
  C2 *tw2 = tw1 + g.n1;
  C2 *pl = tw2 + g.n2;
  const int P2 = g.n2 + 1;
  const int tid = threadIdx.x;
  const int ic = blockIdx.x;
  {
    const C2 *t1 = tw_ptr<T>(g, 1), *t2 = tw_ptr<T>(g, 2);
    for (int t = tid; t < g.n1; t += NT) tw1[t] = t1[t];
    for (int t = tid; t < g.n2; t += NT) tw2[t] = t2[t];
  }
  for (int i = tid; i < g.n1 * P2; i += NT) pl[i] = cmk<C2>(0.0, 0.0);
  __syncthreads();
  C2 *Xrow = X + ((size_t)blockIdx.y * g.n3 + ic) * g.ncols_pad;
  for (int col = tid; col < g.ncols; col += NT) {
    const int ab = g.col_ab[col];
    pl[(ab >> 16) * P2 + (ab & 0xffff)] = Xrow[col];
  }
  __syncthreads();
  const LineMap rows{2 * g.kamax + 1, g.kamax + 1, P2, (g.n1 - g.kamax) * P2, 1};
  const LineMap cols{g.n2, g.n2, 1, 0, P2};
  fft_lines<+1, MAXE>(pl, g.n2, rows, tw2, NT, tid);
  fft_lines<+1, MAXE>(pl, g.n1, cols, tw1, NT, tid);
  const T *Vpl = Vp + (size_t)ic * g.n1 * g.n2;
  for (int e = tid; e < g.n1 * g.n2; e += NT) {
    const int ia = e / g.n2, ib = e - ia * g.n2;
    C2 v = pl[ia * P2 + ib];
    const T w = Vpl[e];
    v.x *= w; v.y *= w;
    pl[ia * P2 + ib] = v;
  }
  __syncthreads();
  fft_lines<-1, MAXE>(pl, g.n1, cols, tw1, NT, tid);
  fft_lines<-1, MAXE>(pl, g.n2, rows, tw2, NT, tid);
  for (int col = tid; col < g.ncols; col += NT) {
    const int ab = g.col_ab[col];
    Xrow[col] = pl[(ab >> 16) * P2 + (ab & 0xffff)];
  }
}

// Density planes: one CTA per (c-plane, pair); |psi1|^2 + |psi2|^2 of the
// plane goes to rho_pair[pair][plane] (package layout, a fastest) and a
// second kernel sums the pairs in a fixed order.
template <typename T, int NT, int MAXE>
__global__ void __launch_bounds__(NT, 1)
k_stage_b_density(DevGeom g, const typename CT<T>::type *__restrict__ X, double *__restrict__ rho_pair) {
  using C2 = typename CT<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tw1 = reinterpret_cast<C2 *>(smem_raw);
  C2 *tw2 = tw1 + g.n1;
  C2 *pl = tw2 + g.n2;
  const int P2 = g.n2 + 1;
  const int tid = threadIdx.x;
  const int ic = blockIdx.x;
  {
    const C2 *t1 = tw_ptr<T>(g, 1), *t2 = tw_ptr<T>(g, 2);
    for (int t = tid; t < g.n1; t += NT) tw1[t] = t1[t];
    for (int t = tid; t < g.n2; t += NT) tw2[t] = t2[t];
  }
  for (int i = tid; i < g.n1 * P2; i += NT) pl[i] = cmk<C2>(0.0, 0.0);
  __syncthreads();
  const C2 *Xrow = X + ((size_t)blockIdx.y * g.n3 + ic) * g.ncols_pad;
  for (int col = tid; col < g.ncols; col += NT) {
    const int ab = g.col_ab[col];
    pl[(ab >> 16) * P2 + (ab & 0xffff)] = Xrow[col];
  }
  __syncthreads();
  const LineMap rows{2 * g.kamax + 1, g.kamax + 1, P2, (g.n1 - g.kamax) * P2, 1};
  const LineMap cols{g.n2, g.n2, 1, 0, P2};
  fft_lines<+1, MAXE>(pl, g.n2, rows, tw2, NT, tid);
  fft_lines<+1, MAXE>(pl, g.n1, cols, tw1, NT, tid);
  const int E = g.n1 * g.n2;
  double *out = rho_pair + (size_t)blockIdx.y * g.N + (size_t)ic * E;
  for (int e = tid; e < E; e += NT) {
    const int ib = e / g.n1, ia = e - ib * g.n1;
    const C2 v = pl[ia * P2 + ib];
    out[e] = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
  }
}

// Noise planes: +-sqrt(N) real fields of two orbitals -> forward a/b FFT.
template <typename T, int NT, int MAXE>
__global__ void __launch_bounds__(NT, 1)
k_stage_b_noise(DevGeom g, const unsigned char *__restrict__ neg, int nstate, int pair0,
                typename CT<T>::type *__restrict__ X) {
  using C2 = typename CT<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tw1 = reinterpret_cast<C2 *>(smem_raw);
  C2 *tw2 = tw1 + g.n1;
  C2 *pl = tw2 + g.n2;
  const int P2 = g.n2 + 1;
  const int tid = threadIdx.x;
  const int ic = blockIdx.x;
  const int p = pair0 + blockIdx.y;
  const int s1 = 2 * p, s2 = 2 * p + 1;
  const bool has2 = s2 < nstate;
  {
    const C2 *t1 = tw_ptr<T>(g, 1), *t2 = tw_ptr<T>(g, 2);
    for (int t = tid; t < g.n1; t += NT) tw1[t] = t1[t];
    for (int t = tid; t < g.n2; t += NT) tw2[t] = t2[t];
  }
  const double rv = sqrt((double)g.N);
  const int E = g.n1 * g.n2;
  const unsigned char *n1p = neg + (size_t)s1 * g.N + (size_t)ic * E;
  const unsigned char *n2p = neg + (size_t)s2 * g.N + (size_t)ic * E;
  for (int e = tid; e < E; e += NT) {
    const int ib = e / g.n1, ia = e - ib * g.n1;
    const double v1 = n1p[e] ? -rv : rv;
    const double v2 = has2 ? (n2p[e] ? -rv : rv) : 0.0;
    pl[ia * P2 + ib] = cmk<C2>(v1, v2);
  }
  __syncthreads();
  const LineMap rows{2 * g.kamax + 1, g.kamax + 1, P2, (g.n1 - g.kamax) * P2, 1};
  const LineMap cols{g.n2, g.n2, 1, 0, P2};
  fft_lines<-1, MAXE>(pl, g.n1, cols, tw1, NT, tid);
  fft_lines<-1, MAXE>(pl, g.n2, rows, tw2, NT, tid);
  C2 *Xrow = X + ((size_t)blockIdx.y * g.n3 + ic) * g.ncols_pad;
  for (int col = tid; col < g.ncols; col += NT) {
    const int ab = g.col_ab[col];
    Xrow[col] = pl[(ab >> 16) * P2 + (ab & 0xffff)];
  }
}

// ============================================================================
// Stage C: forward c-FFT + unpack + fused epilogue.
// ============================================================================
struct Dots { double d0, d1, d2; };

__device__ __forceinline__ void epilogue(const DevGeom &g, const EpiArgs &e, int s, int gi, bool g0,
                                         double fr, double fi, Dots &dt, double &mx) {
  const size_t o = (size_t)s * 2 * g.ngp + gi;
  if (e.mode == EPI_NOISE) {
    e.OUT[o] = fr;
    e.OUT[o + g.ngp] = fi;
    mx = fmax(mx, fmax(absmax_key_d(fr), absmax_key_d(fi)));
    return;
  }
  const double cr = e.C[o], ci = e.C[o + g.ngp];
  if (e.FNL) {
    fr += e.FNL[o];
    fi += e.FNL[o + g.ngp];
  } else if (e.FNLf) {
    fr += (double)e.FNLf[o];
    fi += (double)e.FNLf[o + g.ngp];
  }
  if (!g0) {
    const double k2 = 2.0 * g.ak2[gi];
    fr -= k2 * cr;
    fi -= k2 * ci;
  } else {
    fi = 0.0;
  }
  if (e.mode == EPI_HPSI) {
    e.OUT[o] = fr;
    e.OUT[o + g.ngp] = fi;
    mx = fmax(mx, fmax(absmax_key_d(fr), absmax_key_d(fi)));
    return;
  }
  const double sc = g0 ? e.s2 : e.s1;
  double nr = sc * fr + e.pre * cr;
  double ni = g0 ? 0.0 : (e.s1 * fi + e.pre * ci);
  if (e.mode == EPI_CHEBK || e.mode == EPI_MOMK) {
    nr -= e.PREV[o];
    if (!g0) ni -= e.PREV[o + g.ngp];
  }
  e.OUT[o] = nr;
  e.OUT[o + g.ngp] = ni;
  mx = fmax(mx, fmax(absmax_key_d(nr), absmax_key_d(ni)));
  if (e.ACC) {
    for (int imu = 0; imu < e.nmu; imu++) {
      double *A = e.ACC + imu * e.acc_stride;
      const double a = e.acoef[imu];
      if (e.acoef0) {
        const double a0 = e.acoef0[imu];
        A[o] = a0 * cr + a * nr;
        A[o + g.ngp] = a0 * ci + a * ni;
      } else if (e.acoefp) {
        const double ap = e.acoefp[imu];
        A[o] += ap * cr + a * nr;
        A[o + g.ngp] += ap * ci + a * ni;
      } else {
        A[o] += a * nr;
        A[o + g.ngp] += a * ni;
      }
    }
  }
  if (e.dots) {
    const double wr = g0 ? 1.0 : 2.0;
    const double xr = e.CHI[o], xi = e.CHI[o + g.ngp];
    dt.d0 += wr * xr * nr + 2.0 * xi * ni;
    if (e.mode == EPI_MOMK) {
      dt.d1 += wr * nr * cr + 2.0 * ni * ci;
      dt.d2 += wr * nr * nr + 2.0 * ni * ni;
    } else if (e.ndots > 1) {  // first step: <chi,chi>
      dt.d1 += wr * xr * xr + 2.0 * xi * xi;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kColThreads)
k_stage_c(DevGeom g, const typename CT<T>::type *__restrict__ X, EpiArgs e) {
  using C2 = typename CT<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tw = reinterpret_cast<C2 *>(smem_raw);
  C2 *buf = tw + g.n3;
  __shared__ double red[kColThreads / 32][3];
  const int P3 = g.n3 + 1;
  const int tid = threadIdx.x;
  const int cp0 = blockIdx.x * kCPB;
  const int cp1 = min(cp0 + kCPB, g.ncp);
  const int col0 = 2 * cp0;
  const int ncl = min(2 * cp1, g.ncols) - col0;
  const int p = e.pair0 + blockIdx.y;
  const int s1 = 2 * p, s2 = 2 * p + 1;
  const bool has2 = s2 < e.nstate;
  const C2 *twg = tw_ptr<T>(g, 3);
  for (int t = tid; t < g.n3; t += blockDim.x) tw[t] = twg[t];
  const C2 *Xp = X + (size_t)blockIdx.y * g.n3 * g.ncols_pad;
  for (int i = tid; i < g.n3 * ncl; i += blockDim.x) {
    const int ic = i / ncl, cl = i - ic * ncl;
    buf[cl * P3 + ic] = Xp[(size_t)ic * g.ncols_pad + col0 + cl];
  }
  __syncthreads();
  LineMap lmap{ncl, ncl, P3, 0, 1};
  fft_lines<-1, (2 * kCPB * kMaxEdge + kColThreads - 1) / kColThreads>(buf, g.n3, lmap, tw, blockDim.x, tid);
  Dots dt{0.0, 0.0, 0.0};
  double mx1 = 0.0, mx2 = 0.0;
  const int warp = tid >> 5, lane = tid & 31;
  const double invN = e.invN;
  const bool noise = (e.mode == EPI_NOISE);
  for (int cp = cp0 + warp; cp < cp1; cp += kColThreads / 32) {
    const int lc = 2 * (cp - cp0);
    const bool zc = (cp == g.ncp - 1);
    const int lm = zc ? lc : lc + 1;
    const int gs = g.cp_gstart[cp], gc = g.cp_gcount[cp];
    const int ntot = gc + (zc ? 1 : 0);
    for (int en = lane; en < ntot; en += 32) {
      if (en < gc) {
        const int gi = gs + en;
        const int kc = g.gkc[gi];
        const int kd = kc < 0 ? kc + g.n3 : kc;
        const int km = kc > 0 ? g.n3 - kc : -kc;
        const C2 F = buf[lc * P3 + kd], Fm = buf[lm * P3 + km];
        const double tr = (double)F.x * invN, ti = (double)F.y * invN;
        const double trc = (double)Fm.x * invN, tic = (double)Fm.y * invN;
        double f1r, f1i, f2r, f2i;
        if (!noise) {
          f1r = -(2.0 * (tr + trc));
          f1i = -(2.0 * (ti - tic));
          f2r = -(2.0 * (ti + tic));
          f2i = -(2.0 * (-tr + trc));
        } else {
          f1r = -0.5 * (tr + trc);
          f1i = -0.5 * (ti - tic);
          f2r = -0.5 * (ti + tic);
          f2i = -0.5 * (trc - tr);
        }
        epilogue(g, e, s1, gi, false, f1r, f1i, dt, mx1);
        if (has2) epilogue(g, e, s2, gi, false, f2r, f2i, dt, mx2);
      } else {
        const int g0 = g.ncoef - 1;
        const C2 F = buf[lc * P3];
        const double tr = (double)F.x * invN, ti = (double)F.y * invN;
        const double m = noise ? -1.0 : -2.0;
        epilogue(g, e, s1, g0, true, m * tr, 0.0, dt, mx1);
        if (has2) epilogue(g, e, s2, g0, true, m * ti, 0.0, dt, mx2);
      }
    }
  }
  if (e.omax) {
    __shared__ double mred[kColThreads / 32][2];
    omax_flush(e.omax, s1, s2, has2, mx1, mx2, mred);
  }
  if (e.dots) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      dt.d0 += __shfl_down_sync(0xffffffffu, dt.d0, off);
      dt.d1 += __shfl_down_sync(0xffffffffu, dt.d1, off);
      dt.d2 += __shfl_down_sync(0xffffffffu, dt.d2, off);
    }
    if (lane == 0) { red[warp][0] = dt.d0; red[warp][1] = dt.d1; red[warp][2] = dt.d2; }
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, b = 0.0, c = 0.0;
      for (int w = 0; w < kColThreads / 32; w++) { a += red[w][0]; b += red[w][1]; c += red[w][2]; }
      double *dst = e.dots + ((size_t)p * g.nbatch + blockIdx.x) * 3;
      dst[0] = a; dst[1] = b; dst[2] = c;
    }
  }
}

// ============================================================================
// DMMA FP64 NT GEMM: out[n*ldo+m] = sum_p A[m*lda+p] B[n*ldb+p]
// Block tile 128(m) x 64(n) x 16(k), 8 warps as 4(m) x 2(n), warp tile
// 32 x 32 = 4 x 4 mma.m8n8k4 tiles; cp.async double-buffered smem.
// ============================================================================
constexpr int GBM = 128, GBN = 64, GBK = 16, GPITCH = GBK + 4;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256)
k_gemm_nt_f64(const double *__restrict__ A, int lda, const double *__restrict__ B, int ldb,
              double *__restrict__ out, int ldo, int K, int Mst, int Nst, int kchunk,
              size_t split_stride) {
  extern __shared__ __align__(16) unsigned char gsm[];
  double (*As)[GBM][GPITCH] = reinterpret_cast<double (*)[GBM][GPITCH]>(gsm);
  double (*Bs)[GBN][GPITCH] = reinterpret_cast<double (*)[GBN][GPITCH]>(gsm + sizeof(double) * 2 * GBM * GPITCH);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int m0 = blockIdx.x * GBM, n0 = blockIdx.y * GBN;
  const int kbeg = blockIdx.z * kchunk;
  const int kend = min(K, kbeg + kchunk);
  const int nk = (kend - kbeg) / GBK;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

  auto load_tile = [&](int buf, int k0) {
    // A: 128 rows x 8 chunks(16B); B: 64 rows x 8 chunks
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int c = tid + i * 256;
      const int r = c >> 3, q = c & 7;
      cp_async16(&As[buf][r][q * 2], A + (size_t)(m0 + r) * lda + k0 + q * 2);
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int c = tid + i * 256;
      const int r = c >> 3, q = c & 7;
      cp_async16(&Bs[buf][r][q * 2], B + (size_t)(n0 + r) * ldb + k0 + q * 2);
    }
    cp_async_commit();
  };
  if (nk > 0) load_tile(0, kbeg);
  for (int kt = 0; kt < nk; kt++) {
    const int cur = kt & 1;
    if (kt + 1 < nk) {
      load_tile(cur ^ 1, kbeg + (kt + 1) * GBK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GBK / 4; kk++) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; i++) af[i] = As[cur][wm * 32 + i * 8 + (lane >> 2)][kk * 4 + (lane & 3)];
#pragma unroll
      for (int j = 0; j < 4; j++) bf[j] = Bs[cur][wn * 32 + j * 8 + (lane >> 2)][kk * 4 + (lane & 3)];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    __syncthreads();
  }
  double *o = out + (size_t)blockIdx.z * split_stride;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int m = m0 + wm * 32 + i * 8 + (lane >> 2);
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int v = 0; v < 2; v++) {
        const int n = n0 + wn * 32 + j * 8 + (lane & 3) * 2 + v;
        if (m < Mst && n < Nst) o[(size_t)n * ldo + m] = acc[i][j][v];
      }
    }
  }
}

__global__ void k_split_reduce(const double *__restrict__ work, int split, size_t stride, int ldo,
                               int Mst, int Nst, double *__restrict__ out) {
  const size_t total = (size_t)Mst * Nst;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int n = (int)(i / Mst), m = (int)(i - (size_t)n * Mst);
    const size_t idx = (size_t)n * ldo + m;
    double s = 0.0;
    for (int z = 0; z < split; z++) s += work[z * stride + idx];
    out[idx] = s;
  }
}

// ============================================================================
// small kernels
// ============================================================================
// Moment-dot partials (3 per stage-C CTA): block b sums the CTAs
// [nparts b / kDotBlocks, nparts (b+1) / kDotBlocks) in a fixed order, then one
// thread adds the kDotBlocks block sums in order (k_dots_sum).
__global__ void __launch_bounds__(256) k_dots_reduce(const double *__restrict__ part, int nparts,
                                                     double *__restrict__ blk) {
  __shared__ double sh[256][3];
  const int i0 = (int)((long long)nparts * blockIdx.x / kDotBlocks);
  const int i1 = (int)((long long)nparts * (blockIdx.x + 1) / kDotBlocks);
  double a[3] = {0.0, 0.0, 0.0};
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    for (int d = 0; d < 3; d++) a[d] += part[(size_t)i * 3 + d];
  for (int d = 0; d < 3; d++) sh[threadIdx.x][d] = a[d];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int d = 0; d < 3; d++) sh[threadIdx.x][d] += sh[threadIdx.x + s][d];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; d++) blk[blockIdx.x * 3 + d] = sh[0][d];
}

__global__ void k_dots_sum(const double *__restrict__ blk, int ndots, double *__restrict__ out) {
  if (threadIdx.x < ndots) {
    double a = 0.0;
    for (int b = 0; b < kDotBlocks; b++) a += blk[b * 3 + threadIdx.x];
    out[threadIdx.x] = a;
  }
}

// E_NL partials: block b sums the rows [nstate b / kEnlBlocks, nstate (b+1) /
// kEnlBlocks) in a fixed order (row by row, threads over the projector
// channels, then a fixed tree), so the total does not depend on scheduling.
__global__ void __launch_bounds__(256) k_enl_part(const double *__restrict__ Z, int ldz,
                                                  const double *__restrict__ w, int P, int nstate,
                                                  double *__restrict__ part) {
  __shared__ double sh[256];
  const int r0 = (int)((long long)nstate * blockIdx.x / kEnlBlocks);
  const int r1 = (int)((long long)nstate * (blockIdx.x + 1) / kEnlBlocks);
  double a = 0.0;
  for (int s = r0; s < r1; s++) {
    const double *zr = Z + (size_t)s * ldz;
    for (int u = threadIdx.x; u < P; u += blockDim.x) {
      const double z = zr[u];
      a += w[u] * z * z;
    }
  }
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_enl_sum(const double *__restrict__ part, double *__restrict__ out) {
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int b = 0; b < kEnlBlocks; b++) a += part[b];
    *out = a;
  }
}

__global__ void k_scale_copy(const double *__restrict__ src, double *__restrict__ dst, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = a * src[i];
}

__global__ void k_density_reduce(const double *__restrict__ part, int nsplit, int N, double scale,
                                 double *__restrict__ rho) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int z = 0; z < nsplit; z++) s += part[(size_t)z * N + i];
    rho[i] = s * scale;
  }
}

template <typename T>
__global__ void k_vks_transpose(const double *__restrict__ v, T *__restrict__ Vp, int n1, int n2, int n3) {
  const size_t N = (size_t)n1 * n2 * n3;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    const int ib = (int)(i % n2);
    const int ia = (int)((i / n2) % n1);
    const int ic = (int)(i / ((size_t)n1 * n2));
    Vp[i] = (T)v[((size_t)ia * n2 + ib) * n3 + ic];
  }
}

// ============================================================================
// launch wrappers
// ============================================================================
static inline int grid1d(size_t n, int bs) {
  size_t b = (n + bs - 1) / bs;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

template <typename T> static size_t col_smem(const DevGeom &g) {
  return sizeof(typename CT<T>::type) * (size_t)(g.n3 + 2 * kCPB * (g.n3 + 1));
}
template <typename T> size_t plane_smem(const DevGeom &g) {
  return sizeof(typename CT<T>::type) * (size_t)(g.n1 + g.n2 + g.n1 * (g.n2 + 1));
}

template <typename T>
void launch_stage_a(const DevGeom &g, const double *C, int nstate, int pair0, int npairs, void *X,
                    cudaStream_t st) {
  const size_t sm = col_smem<T>(g);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_stage_a<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  dim3 grid(g.nbatch, npairs);
  k_stage_a<T><<<grid, kColThreads, sm, st>>>(g, C, nstate, pair0, (typename CT<T>::type *)X);
}

template <typename T>
void launch_stage_c(const DevGeom &g, const void *X, const EpiArgs &e, int npairs, cudaStream_t st) {
  const size_t sm = col_smem<T>(g);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_stage_c<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  dim3 grid(g.nbatch, npairs);
  k_stage_c<T><<<grid, kColThreads, sm, st>>>(g, (const typename CT<T>::type *)X, e);
}

// Plane kernels: 512 threads, MAXE bucket chosen from n1*n2.
#define SDFT_PLANE_DISPATCH(KERNEL, T, ...)                                              \
  do {                                                                                   \
    const int E = g.n1 * g.n2;                                                           \
    const size_t sm = plane_smem<T>(g);                                                  \
    if (E <= 512 * 2) {                                                                  \
      auto k = KERNEL<T, 512, 2>;                                                        \
      static const bool attr_once = (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), true); (void)attr_once;  \
      k<<<grid, 512, sm, st>>>(__VA_ARGS__);                                             \
    } else if (E <= 512 * 5) {                                                           \
      auto k = KERNEL<T, 512, 5>;                                                        \
      static const bool attr_once = (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), true); (void)attr_once;  \
      k<<<grid, 512, sm, st>>>(__VA_ARGS__);                                             \
    } else if (E <= 512 * 11) {                                                          \
      auto k = KERNEL<T, 512, 11>;                                                       \
      static const bool attr_once = (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), true); (void)attr_once;  \
      k<<<grid, 512, sm, st>>>(__VA_ARGS__);                                             \
    } else if (E <= 512 * 18) {                                                          \
      auto k = KERNEL<T, 512, 18>;                                                       \
      static const bool attr_once = (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), true); (void)attr_once;  \
      k<<<grid, 512, sm, st>>>(__VA_ARGS__);                                             \
    } else {                                                                             \
      auto k = KERNEL<T, 512, 24>;                                                       \
      static const bool attr_once = (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), true); (void)attr_once;  \
      k<<<grid, 512, sm, st>>>(__VA_ARGS__);                                             \
    }                                                                                    \
  } while (0)

template <typename T>
void launch_stage_b(const DevGeom &g, void *X, const T *Vp, int npairs, cudaStream_t st) {
  dim3 grid(g.n3, npairs);
  SDFT_PLANE_DISPATCH(k_stage_b, T, g, (typename CT<T>::type *)X, Vp);
}

template <typename T>
void launch_stage_b_density(const DevGeom &g, const void *X, int npairs, int nsplit, double *rho_part,
                            cudaStream_t st) {
  (void)nsplit;
  dim3 grid(g.n3, npairs);
  SDFT_PLANE_DISPATCH(k_stage_b_density, T, g, (const typename CT<T>::type *)X, rho_part);
}

template <typename T>
void launch_stage_b_noise(const DevGeom &g, const unsigned char *neg, int nstate, int pair0, int npairs,
                          void *X, cudaStream_t st) {
  dim3 grid(g.n3, npairs);
  SDFT_PLANE_DISPATCH(k_stage_b_noise, T, g, neg, nstate, pair0, (typename CT<T>::type *)X);
}

void launch_density_reduce(const double *rho_part, int nsplit, int N, double scale, double *rho,
                           cudaStream_t st) {
  k_density_reduce<<<grid1d(N, 256), 256, 0, st>>>(rho_part, nsplit, N, scale, rho);
}

void launch_gemm_nt_f64(const double *A, int lda, const double *B, int ldb, double *out, int ldo, int M,
                        int N, int K, int Mst, int Nst, int split, double *work, cudaStream_t st) {
  if (split < 1) split = 1;
  int kchunk = (K / GBK + split - 1) / split * GBK;
  split = (K + kchunk - 1) / kchunk;
  dim3 grid(M / GBM, N / GBN, split);
  const size_t sm = sizeof(double) * 2 * (GBM + GBN) * GPITCH;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_gemm_nt_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  if (split == 1) {
    k_gemm_nt_f64<<<grid, 256, sm, st>>>(A, lda, B, ldb, out, ldo, K, Mst, Nst, kchunk, 0);
  } else {
    const size_t stride = (size_t)N * ldo;
    k_gemm_nt_f64<<<grid, 256, sm, st>>>(A, lda, B, ldb, work, ldo, K, Mst, Nst, kchunk, stride);
    k_split_reduce<<<grid1d((size_t)Mst * Nst, 256), 256, 0, st>>>(work, split, stride, ldo, Mst, Nst, out);
  }
}

void launch_dots_reduce(const double *part, int nparts, int ndots, double *blk, double *out, cudaStream_t st) {
  k_dots_reduce<<<kDotBlocks, 256, 0, st>>>(part, nparts, blk);
  k_dots_sum<<<1, 32, 0, st>>>(blk, ndots, out);
}

void launch_enl(const double *Z, int ldz, const double *w, int P, int nstate, double *out, cudaStream_t st) {
  k_enl_part<<<kEnlBlocks, 256, 0, st>>>(Z, ldz, w, P, nstate, out + 1);
  k_enl_sum<<<1, 32, 0, st>>>(out + 1, out);
}

void launch_scale_copy(const double *src, double *dst, double a, size_t n, cudaStream_t st) {
  k_scale_copy<<<grid1d(n, 256), 256, 0, st>>>(src, dst, a, n);
}

template <typename T>
void launch_vks_transpose(const double *v, T *Vp, int n1, int n2, int n3, cudaStream_t st) {
  k_vks_transpose<T><<<grid1d((size_t)n1 * n2 * n3, 256), 256, 0, st>>>(v, Vp, n1, n2, n3);
}

template void launch_stage_a<double>(const DevGeom &, const double *, int, int, int, void *, cudaStream_t);
template void launch_stage_a<float>(const DevGeom &, const double *, int, int, int, void *, cudaStream_t);
template void launch_stage_b<double>(const DevGeom &, void *, const double *, int, cudaStream_t);
template void launch_stage_b<float>(const DevGeom &, void *, const float *, int, cudaStream_t);
template void launch_stage_c<double>(const DevGeom &, const void *, const EpiArgs &, int, cudaStream_t);
template void launch_stage_c<float>(const DevGeom &, const void *, const EpiArgs &, int, cudaStream_t);
template void launch_stage_b_density<double>(const DevGeom &, const void *, int, int, double *, cudaStream_t);
template void launch_stage_b_density<float>(const DevGeom &, const void *, int, int, double *, cudaStream_t);
template void launch_stage_b_noise<double>(const DevGeom &, const unsigned char *, int, int, int, void *, cudaStream_t);
template void launch_stage_b_noise<float>(const DevGeom &, const unsigned char *, int, int, int, void *, cudaStream_t);
template void launch_vks_transpose<double>(const double *, double *, int, int, int, cudaStream_t);
template void launch_vks_transpose<float>(const double *, float *, int, int, int, cudaStream_t);
template size_t plane_smem<double>(const DevGeom &);
template size_t plane_smem<float>(const DevGeom &);

}  // namespace sdft
