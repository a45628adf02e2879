// sdft_kernels2.cu -- fast-path FFT stages with compile-time grid edges.
//
// Same stage split as sdft_kernels.cu (A: pack + c-FFT, B: plane FFTs x V,
// C: c-FFT + unpack/epilogue) but every 1-D transform is the two-pass
// factorised FFT of sdft_fft2.cuh:
//   stage A writes the c-transformed columns in the permuted real-space
//   order r = pos_N3(ic) (X row r);
//   stage B forward-transforms b then a (natural -> permuted), multiplies by
//   V stored in the same permuted order, and transforms back a then b
//   (permuted -> natural);
//   stage C transforms X rows r back to natural kc (permuted -> natural).
// So no data movement is ever spent on undoing an FFT permutation.
#include <cuda_runtime.h>
#include <cmath>
#include <type_traits>
#include "sdft_fft2.cuh"
#include "sdft_internal.h"
#include "sdft_kernels.cuh"
#include "sdft_kernels2.cuh"

namespace sdft {

// exp(-2 pi i t/N) of every compile-time FFT edge in constant memory (the
// warps of the plane passes read one twiddle index at a time, which the
// constant cache broadcasts without a shared-memory wavefront); offsets of
// the edges 12, 16, 24, 32, 36, 48, 64, 72, 96, 128
constexpr int kTwEdges[] = {12, 16, 24, 32, 36, 48, 64, 72, 96, 128};
constexpr int kTwTotal = 528;
constexpr int tw_off(int n) {
  int o = 0;
  for (int e : kTwEdges) {
    if (e == n) return o;
    o += e;
  }
  return -1;
}
template <int N> struct TwOff {
  static constexpr int value = tw_off(N);
  static_assert(value >= 0, "edge without a constant twiddle table");
};
__constant__ float2 c_twf[kTwTotal];
__constant__ double2 c_twd[kTwTotal];

template <int N, typename C> struct TwC;
template <int N> struct TwC<N, float2> {
  __device__ __forceinline__ float2 operator()(int t) const { return c_twf[TwOff<N>::value + t]; }
};
template <int N> struct TwC<N, double2> {
  __device__ __forceinline__ double2 operator()(int t) const { return c_twd[TwOff<N>::value + t]; }
};

int init_const_twiddles() {
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
  if (done[dev]) return 0;
  float2 hf[kTwTotal];
  double2 hd[kTwTotal];
  for (int e : kTwEdges)
    for (int t = 0; t < e; t++) {  // the same values as the context's twiddle tables
      const double a = 2.0 * M_PI * (double)t / (double)e;
      hd[tw_off(e) + t] = make_double2(std::cos(a), -std::sin(a));
      hf[tw_off(e) + t] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
  if (cudaMemcpyToSymbol(c_twf, hf, sizeof hf) != cudaSuccess) return 1;
  if (cudaMemcpyToSymbol(c_twd, hd, sizeof hd) != cudaSuccess) return 1;
  done[dev] = true;
  return 0;
}

template <typename T> __device__ __forceinline__ const typename CT<T>::type *twp(const DevGeom &g, int d);
template <> __device__ __forceinline__ const double2 *twp<double>(const DevGeom &g, int d) {
  return d == 1 ? g.tw1 : (d == 2 ? g.tw2 : g.tw3);
}
template <> __device__ __forceinline__ const float2 *twp<float>(const DevGeom &g, int d) {
  return d == 1 ? g.tw1f : (d == 2 ? g.tw2f : g.tw3f);
}

// ---------------------------------------------------------------------------
// stage A
// ---------------------------------------------------------------------------
template <typename T, int N3>
__global__ void __launch_bounds__(kColThreads)
kf_stage_a(DevGeom g, const double *__restrict__ C, int nstate, int pair0, typename CT<T>::type *__restrict__ X) {
  using C2 = typename CT<T>::type;
  constexpr int P3 = N3 + 1;
  __shared__ __align__(16) C2 buf[2 * kCPB * P3];
  const int tid = threadIdx.x;
  const int cp0 = blockIdx.x * kCPB;
  const int cp1 = min(cp0 + kCPB, g.ncp);
  const int col0 = 2 * cp0;
  const int ncl = min(2 * cp1, g.ncols) - col0;
  const int p = pair0 + blockIdx.y;
  const int s1 = 2 * p, s2 = 2 * p + 1;
  const bool has2 = s2 < nstate;
  for (int i = tid; i < ncl * P3; i += kColThreads) buf[i] = cmk<C2>(0.0, 0.0);
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
      const int kd = kc < 0 ? kc + N3 : kc;
      const int km = kc > 0 ? N3 - kc : -kc;
      buf[lc * P3 + kd] = cmk<C2>(a - d, b + c);
      buf[lm * P3 + km] = cmk<C2>(a + d, -b + c);
    }
    if (zc && lane == 0) {
      const int g0 = g.ncoef - 1;
      buf[lc * P3] = cmk<C2>(C[o1 + g0], has2 ? C[o2 + g0] : 0.0);
    }
  }
  __syncthreads();
  dif<N3, 1, +1>(buf, Lines1{P3}, ncl, TwC<N3, C2>{}, tid, kColThreads);
  C2 *Xp = X + (size_t)blockIdx.y * N3 * g.ncols_pad;
  for (int i = tid; i < N3 * ncl; i += kColThreads) {
    const int r = i / ncl, cl = i - r * ncl;
    Xp[(size_t)r * g.ncols_pad + col0 + cl] = buf[cl * P3 + r];
  }
}

// ---------------------------------------------------------------------------
// stage C
// ---------------------------------------------------------------------------
struct Dots2 { double d0, d1, d2; };

// Writes OUT for orbital s at G index gi and returns the written pair in
// (wr, wi).
// HOT: a filter step (Chebyshev or Newton, no moment dots): the noise,
// H-psi and dot branches are compiled out, which keeps the hot instance
// within 64 registers without spills.
template <bool HOT>
__device__ __forceinline__ void epilogue2(const DevGeom &g, const EpiArgs &e, int s, int gi, bool g0, double fr,
                                          double fi, Dots2 &dt, double &mx, double &wr, double &wi) {
  const size_t o = (size_t)s * 2 * g.ngp + gi;
  if (!HOT && e.mode == EPI_NOISE) {
    e.OUT[o] = fr;
    e.OUT[o + g.ngp] = fi;
    mx = fmax(mx, fmax(absmax_key_d(fr), absmax_key_d(fi)));
    wr = fr; wi = fi;
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
  if (!HOT && e.mode == EPI_HPSI) {
    e.OUT[o] = fr;
    e.OUT[o + g.ngp] = fi;
    mx = fmax(mx, fmax(absmax_key_d(fr), absmax_key_d(fi)));
    wr = fr; wi = fi;
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
  wr = nr; wi = ni;
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
  if (!HOT && e.dots) {
    const double wr = g0 ? 1.0 : 2.0;
    const double xr = e.CHI[o], xi = e.CHI[o + g.ngp];
    dt.d0 += wr * xr * nr + 2.0 * xi * ni;
    if (e.mode == EPI_MOMK) {
      dt.d1 += wr * nr * cr + 2.0 * ni * ci;
      dt.d2 += wr * nr * nr + 2.0 * ni * ni;
    } else if (e.ndots > 1) {
      dt.d1 += wr * xr * xr + 2.0 * xi * xi;
    }
  }
}

// X is not __restrict__: with e.Xnext the CTA overwrites its own columns of
// the same scratch (read into shared memory at the start) for the next step.
// Filter-step epilogue for both orbitals of a pair at G index gi: every load
// of both orbitals is issued before any store (OUT may alias PREV, so a load
// placed after a store could not be moved above it), which doubles the loads
// in flight per thread.  Same arithmetic as epilogue2 for CHEB1 / CHEBK /
// NEWTON without dots; returns the written values (a: s1, b: s2).
__device__ __forceinline__ void epilogue_pair_hot(const DevGeom &g, const EpiArgs &e, int s1, bool has2, int gi,
                                                  bool g0, double f1r, double f1i, double f2r, double f2i,
                                                  double &mx1, double &mx2, double &ar, double &ai, double &br,
                                                  double &bi) {
  const size_t n = g.ngp;
  const size_t o1 = (size_t)s1 * 2 * n + gi, o2 = o1 + 2 * n;
  const bool rec = e.mode == EPI_CHEBK;
  const bool acc1 = e.ACC && e.nmu == 1 && !e.acoef0;
  double c1r = e.C[o1], c1i = e.C[o1 + n], c2r = 0.0, c2i = 0.0;
  double x1r = 0.0, x1i = 0.0, x2r = 0.0, x2i = 0.0;
  double p1r = 0.0, p1i = 0.0, p2r = 0.0, p2i = 0.0;
  double q1r = 0.0, q1i = 0.0, q2r = 0.0, q2i = 0.0;
  if (has2) { c2r = e.C[o2]; c2i = e.C[o2 + n]; }
  if (e.FNLf) {
    x1r = e.FNLf[o1]; x1i = e.FNLf[o1 + n];
    if (has2) { x2r = e.FNLf[o2]; x2i = e.FNLf[o2 + n]; }
  } else if (e.FNL) {
    x1r = e.FNL[o1]; x1i = e.FNL[o1 + n];
    if (has2) { x2r = e.FNL[o2]; x2i = e.FNL[o2 + n]; }
  }
  if (rec) {
    p1r = e.PREV[o1]; p1i = e.PREV[o1 + n];
    if (has2) { p2r = e.PREV[o2]; p2i = e.PREV[o2 + n]; }
  }
  if (acc1) {
    q1r = e.ACC[o1]; q1i = e.ACC[o1 + n];
    if (has2) { q2r = e.ACC[o2]; q2i = e.ACC[o2 + n]; }
  }
  const double k2 = g0 ? 0.0 : 2.0 * g.ak2[gi];
  f1r += x1r - k2 * c1r;
  f2r += x2r - k2 * c2r;
  f1i += x1i - k2 * c1i;
  f2i += x2i - k2 * c2i;
  const double sc = g0 ? e.s2 : e.s1;
  ar = sc * f1r + e.pre * c1r;
  br = sc * f2r + e.pre * c2r;
  ai = g0 ? 0.0 : (e.s1 * f1i + e.pre * c1i);
  bi = g0 ? 0.0 : (e.s1 * f2i + e.pre * c2i);
  if (rec) {
    ar -= p1r;
    br -= p2r;
    if (!g0) { ai -= p1i; bi -= p2i; }
  }
  e.OUT[o1] = ar;
  e.OUT[o1 + n] = ai;
  mx1 = fmax(mx1, fmax(absmax_key_d(ar), absmax_key_d(ai)));
  if (has2) {
    e.OUT[o2] = br;
    e.OUT[o2 + n] = bi;
    mx2 = fmax(mx2, fmax(absmax_key_d(br), absmax_key_d(bi)));
  }
  if (!e.ACC) return;
  if (acc1) {
    const double a = e.acoef[0];
    const double ap = e.acoefp ? e.acoefp[0] : 0.0;
    e.ACC[o1] = q1r + ap * c1r + a * ar;
    e.ACC[o1 + n] = q1i + ap * c1i + a * ai;
    if (has2) {
      e.ACC[o2] = q2r + ap * c2r + a * br;
      e.ACC[o2 + n] = q2i + ap * c2i + a * bi;
    }
    return;
  }
  for (int k = 0; k < (has2 ? 2 : 1); k++) {
    const size_t o = k ? o2 : o1;
    const double cr = k ? c2r : c1r, ci = k ? c2i : c1i, nr = k ? br : ar, ni = k ? bi : ai;
    for (int imu = 0; imu < e.nmu; imu++) {
      double *A = e.ACC + imu * e.acc_stride;
      const double a = e.acoef[imu];
      if (e.acoef0) {
        const double a0 = e.acoef0[imu];
        A[o] = a0 * cr + a * nr;
        A[o + n] = a0 * ci + a * ni;
      } else if (e.acoefp) {
        const double ap = e.acoefp[imu];
        A[o] += ap * cr + a * nr;
        A[o + n] += ap * ci + a * ni;
      } else {
        A[o] += a * nr;
        A[o + n] += a * ni;
      }
    }
  }
}

// 6 CTAs/SM (40 registers, some spilled): latency-bound, the extra resident
// CTAs measured 4 % faster than 4 CTAs/SM at equal clocks
// (256 threads x 6 measured ahead of 384 x 4 and 320 x 5: 0.98 against 1.10 and 1.08 ms)
constexpr int kCThreads = 256, kCMinB = 6;
template <typename T, int N3, bool HOT>
__global__ void __launch_bounds__(kCThreads, kCMinB)
kf_stage_c(DevGeom g, const typename CT<T>::type *X, EpiArgs e) {
  using C2 = typename CT<T>::type;
  constexpr int P3 = N3 + 1;
  __shared__ __align__(16) C2 buf[2 * kCPB * P3];
  // packed OUT columns for the next step (e.Xnext; FP32 columns only: the
  // FP64 instance has no room for a second buffer in static shared memory)
  constexpr bool kCanPack = sizeof(T) == 4;
  __shared__ __align__(16) C2 nbuf[kCanPack ? 2 * kCPB * P3 : 1];
  __shared__ double red[kCThreads / 32][3];
  const int tid = threadIdx.x;
  const int cp0 = blockIdx.x * kCPB;
  const int cp1 = min(cp0 + kCPB, g.ncp);
  const int col0 = 2 * cp0;
  const int ncl = min(2 * cp1, g.ncols) - col0;
  const int p = e.pair0 + blockIdx.y;
  const int s1 = 2 * p, s2 = 2 * p + 1;
  const bool has2 = s2 < e.nstate;
  const C2 *Xp = X + (size_t)blockIdx.y * N3 * g.ncols_pad;
  for (int i = tid; i < N3 * ncl; i += kCThreads) {
    const int r = i / ncl, cl = i - r * ncl;
    buf[cl * P3 + r] = Xp[(size_t)r * g.ncols_pad + col0 + cl];
  }
  const bool pack = kCanPack && e.Xnext != nullptr;
  if (pack)
    for (int i = tid; i < ncl * P3; i += kCThreads) nbuf[i] = cmk<C2>(0.0, 0.0);
  // first item (point) of each column pair in the CTA's item list
  __shared__ int pref[kCPB + 1];
  if (tid == 0) {
    int s = 0;
    for (int k = 0; k < cp1 - cp0; k++) {
      pref[k] = s;
      s += g.cp_gcount[cp0 + k] + (cp0 + k == g.ncp - 1 ? 1 : 0);
    }
    pref[cp1 - cp0] = s;
  }
  __syncthreads();
  dit<N3, 1, -1>(buf, Lines1{P3}, ncl, TwC<N3, C2>{}, tid, kCThreads);
  Dots2 dt{0.0, 0.0, 0.0};
  double mx1 = 0.0, mx2 = 0.0;
  const int warp = tid >> 5, lane = tid & 31;
  const double invN = e.invN;
  const bool noise = !HOT && (e.mode == EPI_NOISE);
  // one point en of column pair cp
  auto item = [&](int cp, int en) {
    const int lc = 2 * (cp - cp0);
    const bool zc = (cp == g.ncp - 1);
    const int lm = zc ? lc : lc + 1;
    const int gs = g.cp_gstart[cp], gc = g.cp_gcount[cp];
    {
      if (en < gc) {
        const int gi = gs + en;
        const int kc = g.gkc[gi];
        const int kd = kc < 0 ? kc + N3 : kc;
        const int km = kc > 0 ? N3 - kc : -kc;
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
        double ar, ai, cr2 = 0.0, ci2 = 0.0;
        if constexpr (HOT) {
          epilogue_pair_hot(g, e, s1, has2, gi, false, f1r, f1i, f2r, f2i, mx1, mx2, ar, ai, cr2, ci2);
        } else {
          epilogue2<HOT>(g, e, s1, gi, false, f1r, f1i, dt, mx1, ar, ai);
          if (has2) epilogue2<HOT>(g, e, s2, gi, false, f2r, f2i, dt, mx2, cr2, ci2);
        }
        if (pack) {  // stage A's packing of the pair (c1 + i c2) at +kc and -kc
          nbuf[lc * P3 + kd] = cmk<C2>(ar - ci2, ai + cr2);
          nbuf[lm * P3 + km] = cmk<C2>(ar + ci2, -ai + cr2);
        }
      } else {
        const int g0 = g.ncoef - 1;
        const C2 F = buf[lc * P3];
        const double tr = (double)F.x * invN, ti = (double)F.y * invN;
        const double m = noise ? -1.0 : -2.0;
        double ar, ai, cr2 = 0.0, ci2 = 0.0;
        if constexpr (HOT) {
          epilogue_pair_hot(g, e, s1, has2, g0, true, m * tr, 0.0, m * ti, 0.0, mx1, mx2, ar, ai, cr2, ci2);
        } else {
          epilogue2<HOT>(g, e, s1, g0, true, m * tr, 0.0, dt, mx1, ar, ai);
          if (has2) epilogue2<HOT>(g, e, s2, g0, true, m * ti, 0.0, dt, mx2, cr2, ci2);
        }
        if (pack) nbuf[lc * P3] = cmk<C2>(ar, cr2);
      }
    }
  };
  {  // the CTA's points dealt out over all threads
    const int tot = pref[cp1 - cp0];
    for (int it = tid; it < tot; it += kCThreads) {
      int k = 0;
      while (k + 1 < cp1 - cp0 && it >= pref[k + 1]) k++;
      item(cp0 + k, it - pref[k]);
    }
  }
  if (e.omax) {
    __shared__ double mred[kCThreads / 32][2];
    omax_flush(e.omax, s1, s2, has2, mx1, mx2, mred);
  }
  if (!HOT && e.dots) {
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
      for (int w = 0; w < kCThreads / 32; w++) { a += red[w][0]; b += red[w][1]; c += red[w][2]; }
      double *dst = e.dots + ((size_t)p * g.nbatch + blockIdx.x) * 3;
      dst[0] = a; dst[1] = b; dst[2] = c;
    }
  }
  if (pack) {  // the next application's stage A: forward c-transform, store columns
    __syncthreads();
    dif<N3, 1, +1>(nbuf, Lines1{P3}, ncl, TwC<N3, C2>{}, tid, kCThreads);
    C2 *Xn = reinterpret_cast<C2 *>(e.Xnext) + (size_t)blockIdx.y * N3 * g.ncols_pad;
    for (int i = tid; i < N3 * ncl; i += kCThreads) {
      const int r = i / ncl, cl = i - r * ncl;
      Xn[(size_t)r * g.ncols_pad + col0 + cl] = nbuf[cl * P3 + r];
    }
  }
}

// ---------------------------------------------------------------------------
// plane stages
// ---------------------------------------------------------------------------
template <typename T> struct PlaneCfg;
template <> struct PlaneCfg<double> { static constexpr int NT = 512, MINB = 1; };
template <> struct PlaneCfg<float> { static constexpr int NT = 256, MINB = 3; };

// natural row ka -> line index helper for the rows touched by the sphere
template <int N1> struct RowsPerm {  // rows given in permuted-a order
  int kamax, ls;
  __device__ __forceinline__ int base(int l) const {
    const int ka = (l <= kamax) ? l : N1 - (2 * kamax + 1) + l;
    return pos<N1>(ka) * ls;
  }
  __device__ __forceinline__ bool valid(int) const { return true; }
};

// a-direction transform pair of one plane with the V multiply fused in:
// forward a-FFT (natural -> permuted) of the N2 columns, times V (stored in
// the permuted order, Vpl[pa*N2 + pb]), inverse a-FFT (permuted -> natural).
// The second forward pass and the first inverse pass work on the same
// R2-blocks of a column, so one register-resident unit does
// DFT -> x V -> inverse DFT without a round trip through shared memory.
// Rows with kamax < ka < N1 - kamax are zero on input (outside the sphere)
// and not needed on output: they are neither read nor written.
// PM >= 1: rows ka in the j1 = 3, 4 band (|ka| >= 3 N1/8, outside a sphere
// narrower than that) are skipped at compile time, with no activity test.
// PM == 2: the sphere is also at least N1/4 wide, so the rows with j1 = 0,
// 1, 6, 7 are always inside it and only j1 = 2, 5 are tested.
template <int N1, int PM = 0, typename C2, typename T, typename TW>
__device__ __forceinline__ void plane_a_vmul(C2 *pl, int P2, int nl, int N2, const T *__restrict__ Vpl, int kamax,
                                             const TW &tw1, int tid, int nthr) {
  constexpr int R1 = Plan<N1>::R1, R2 = Plan<N1>::R2;
  constexpr bool P34 = PM >= 1;
  static_assert(!P34 || R1 == 8, "the j1 = 3, 4 band needs R1 = 8");
  auto active_ka = [&](int ka) { return ka <= kamax || ka >= N1 - kamax; };
  // row ka = j2 + R2 j1 holds data (j1 a compile-time constant after unrolling)
  auto active_j = [&](int j1, int ka) {
    if (band34<R1>(P34, j1)) return false;
    if (PM == 2 && (j1 == 0 || j1 == 1 || j1 == 6 || j1 == 7)) return true;
    return active_ka(ka);
  };
#pragma unroll 1
  for (UnitIter it(tid, nthr, nl); it.j < R2; it.next()) {  // forward pass 1
    const int l = it.l, j2 = it.j;
    C2 *p = pl + l;
    C2 v[R1];
#pragma unroll
    for (int j1 = 0; j1 < R1; j1++) {
      const int ka = j2 + R2 * j1;
      v[j1] = active_j(j1, ka) ? p[ka * P2] : cmk<C2>(0.0, 0.0);
    }
    dftr<R1, +1>(v);
    p[j2 * P2] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R1; k1++) {
      C2 w = tw_at<C2>(tw1, j2 * k1);
      w.y = -w.y;
      p[(j2 + R2 * k1) * P2] = cmul(v[k1], w);
    }
  }
  __syncthreads();
#pragma unroll 1
  for (UnitIter it(tid, nthr, nl); it.j < R1; it.next()) {  // forward pass 2, x V, inverse pass 1
    const int l = it.l, k1 = it.j;
    C2 *p = pl + R2 * k1 * P2 + l;
    const T *vp = Vpl + (size_t)R2 * k1 * N2 + l;
    C2 v[R2];
#pragma unroll
    for (int j = 0; j < R2; j++) v[j] = p[j * P2];
    dftr<R2, +1>(v);
#pragma unroll
    for (int j = 0; j < R2; j++) v[j] = cscale(v[j], vp[(size_t)j * N2]);
    dftr<R2, -1>(v);
    p[0] = v[0];
#pragma unroll
    for (int j2 = 1; j2 < R2; j2++) p[j2 * P2] = cmul(v[j2], tw_at<C2>(tw1, j2 * k1));
  }
  __syncthreads();
#pragma unroll 1
  for (UnitIter it(tid, nthr, nl); it.j < R2; it.next()) {  // inverse pass 2
    const int l = it.l, j2 = it.j;
    C2 *p = pl + l;
    C2 v[R1];
#pragma unroll
    for (int k1 = 0; k1 < R1; k1++) v[k1] = p[(R2 * k1 + j2) * P2];
    dftr<R1, -1>(v);
#pragma unroll
    for (int j1 = 0; j1 < R1; j1++) {
      const int ka = j2 + R2 * j1;
      if (active_j(j1, ka)) p[ka * P2] = v[j1];
    }
  }
  __syncthreads();
}

// Sphere rows of a plane as b-lines (Lines2P order): line l < g1 is row l,
// line l >= g1 is row base2 + l - g1; element k of a line holds data when
// its signed kb lies in the row's column range.
template <int N2> struct RowKb {
  const int2 *rng;
  int g1, base2;
  struct In {
    int lo, hi;
    __device__ __forceinline__ bool operator()(int k) const {
      const int kb = k <= N2 / 2 ? k : k - N2;
      return kb >= lo && kb <= hi;
    }
  };
  __device__ __forceinline__ In line(int l) const {
    const int2 r = rng[l < g1 ? l : base2 + (l - g1)];
    return In{r.x, r.y};
  }
};

// NT threads per plane CTA: PlaneCfg's default, or (FP32) the 128-thread
// instance that the autotuner may pick for small planes (more resident CTAs).
// PM (DevGeom::prune34): 1 = the sphere is narrower than 3/8 of both plane
// edges (R1 = 8 plans): the j1 = 3, 4 band of the first forward and last
// inverse passes is skipped; 2 = also at least a quarter of N1 wide, so the
// a-pass tests only the rows with j1 = 2, 5.
template <typename T, int N1, int N2, int NT = PlaneCfg<T>::NT, int MINB = PlaneCfg<T>::MINB, int PM = 0>
__global__ void __launch_bounds__(NT, MINB)
kf_stage_b(DevGeom g, typename CT<T>::type *__restrict__ X, const T *__restrict__ Vp) {
  using C2 = typename CT<T>::type;
  constexpr int P2 = N2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // (the first N1 + N2 complex slots held twiddles before they moved to
  // constant memory; the row kb ranges use the first N1 of them)
  int2 *rng = reinterpret_cast<int2 *>(smem_raw);
  C2 *pl = reinterpret_cast<C2 *>(smem_raw) + N1 + N2;
  const int tid = threadIdx.x;
  const int r = blockIdx.x;
  const int ka = g.kamax;
  const bool contig = g.kb_contig != 0;
  if (contig) {
    for (int t = tid; t < N1; t += NT) rng[t] = g.kb_rng[t];
  } else {
    // zero the 2 kamax + 1 rows inside the sphere's a-range
    const Lines2 rows{ka + 1, P2, (N1 - ka) * P2};
    for (int i = tid; i < (2 * ka + 1) * N2; i += NT) {
      const int l = i / N2, b = i - l * N2;
      pl[rows.base(l) + b] = cmk<C2>(0.0, 0.0);
    }
  }
  __syncthreads();
  C2 *Xrow = X + ((size_t)blockIdx.y * g.n3 + r) * g.ncols_pad;
  for (int col = tid; col < g.ncols; col += NT) {
    const int ab = g.col_ab[col];
    pl[(ab >> 16) * P2 + (ab & 0xffff)] = Xrow[col];
  }
  __syncthreads();
  // b-transforms over the sphere rows, each row group padded to 16 lanes
  const int g1 = (ka + 1 + 15) & ~15, g2 = (ka + 15) & ~15;
  const Lines2P rowsp{ka + 1, g1, ka, P2, (N1 - ka) * P2};
  if (contig) {  // only the sphere's elements are read before and written after the b-transforms
    const RowKb<N2> m{rng, g1, N1 - ka};
    dif<N2, 1, +1, (PM >= 1)>(pl, rowsp, g1 + g2, TwC<N2, C2>{}, tid, NT, m);
    plane_a_vmul<N1, PM>(pl, P2, N2, N2, Vp + (size_t)r * N1 * N2, ka, TwC<N1, C2>{}, tid, NT);
    dit<N2, 1, -1, (PM >= 1)>(pl, rowsp, g1 + g2, TwC<N2, C2>{}, tid, NT, m);
  } else {
    dif<N2, 1, +1, (PM >= 1)>(pl, rowsp, g1 + g2, TwC<N2, C2>{}, tid, NT);
    plane_a_vmul<N1, PM>(pl, P2, N2, N2, Vp + (size_t)r * N1 * N2, ka, TwC<N1, C2>{}, tid, NT);
    dit<N2, 1, -1, (PM >= 1)>(pl, rowsp, g1 + g2, TwC<N2, C2>{}, tid, NT);
  }
  for (int col = tid; col < g.ncols; col += NT) {
    const int ab = g.col_ab[col];
    Xrow[col] = pl[(ab >> 16) * P2 + (ab & 0xffff)];
  }
}

template <typename T, int N1, int N2>
__global__ void __launch_bounds__(PlaneCfg<T>::NT, PlaneCfg<T>::MINB)
kf_stage_b_density(DevGeom g, const typename CT<T>::type *__restrict__ X, double *__restrict__ rho_pair,
                   int r3_1, int r3_2) {
  using C2 = typename CT<T>::type;
  constexpr int NT = PlaneCfg<T>::NT, P2 = N2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tw1 = reinterpret_cast<C2 *>(smem_raw);
  C2 *tw2 = tw1 + N1;
  C2 *pl = tw2 + N2;
  const int tid = threadIdx.x;
  const int r = blockIdx.x;
  const int ic = (r % r3_2) * r3_1 + r / r3_2;
  {
    const C2 *t1 = twp<T>(g, 1), *t2 = twp<T>(g, 2);
    for (int t = tid; t < N1; t += NT) tw1[t] = t1[t];
    for (int t = tid; t < N2; t += NT) tw2[t] = t2[t];
  }
  for (int i = tid; i < N1 * P2; i += NT) pl[i] = cmk<C2>(0.0, 0.0);
  __syncthreads();
  const C2 *Xrow = X + ((size_t)blockIdx.y * g.n3 + r) * g.ncols_pad;
  for (int col = tid; col < g.ncols; col += NT) {
    const int ab = g.col_ab[col];
    pl[(ab >> 16) * P2 + (ab & 0xffff)] = Xrow[col];
  }
  __syncthreads();
  const int ka = g.kamax;
  dif<N2, 1, +1>(pl, Lines2{ka + 1, P2, (N1 - ka) * P2}, 2 * ka + 1, tw2, tid, NT);
  dif<N1, P2, +1>(pl, Lines1{1}, N2, tw1, tid, NT);
  double *out = rho_pair + (size_t)blockIdx.y * g.N + (size_t)ic * N1 * N2;
  for (int e = tid; e < N1 * N2; e += NT) {
    const int ib = e / N1, ia = e - ib * N1;
    const C2 v = pl[pos<N1>(ia) * P2 + pos<N2>(ib)];
    out[e] = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
  }
}

template <typename T, int N1, int N2>
__global__ void __launch_bounds__(PlaneCfg<T>::NT, PlaneCfg<T>::MINB)
kf_stage_b_noise(DevGeom g, const unsigned char *__restrict__ neg, int nstate, int pair0,
                 typename CT<T>::type *__restrict__ X, int r3_1, int r3_2) {
  using C2 = typename CT<T>::type;
  constexpr int NT = PlaneCfg<T>::NT, P2 = N2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tw1 = reinterpret_cast<C2 *>(smem_raw);
  C2 *tw2 = tw1 + N1;
  C2 *pl = tw2 + N2;
  const int tid = threadIdx.x;
  const int r = blockIdx.x;
  const int ic = (r % r3_2) * r3_1 + r / r3_2;
  const int p = pair0 + blockIdx.y;
  const int s1 = 2 * p, s2 = 2 * p + 1;
  const bool has2 = s2 < nstate;
  {
    const C2 *t1 = twp<T>(g, 1), *t2 = twp<T>(g, 2);
    for (int t = tid; t < N1; t += NT) tw1[t] = t1[t];
    for (int t = tid; t < N2; t += NT) tw2[t] = t2[t];
  }
  const double rv = sqrt((double)g.N);
  constexpr int E = N1 * N2;
  const unsigned char *n1p = neg + (size_t)s1 * g.N + (size_t)ic * E;
  const unsigned char *n2p = neg + (size_t)s2 * g.N + (size_t)ic * E;
  for (int e = tid; e < E; e += NT) {
    const int ib = e / N1, ia = e - ib * N1;
    const double v1 = n1p[e] ? -rv : rv;
    const double v2 = has2 ? (n2p[e] ? -rv : rv) : 0.0;
    pl[ia * P2 + ib] = cmk<C2>(v1, v2);
  }
  __syncthreads();
  const int ka = g.kamax;
  dif<N1, P2, -1>(pl, Lines1{1}, N2, tw1, tid, NT);
  dif<N2, 1, -1>(pl, RowsPerm<N1>{ka, P2}, 2 * ka + 1, tw2, tid, NT);
  C2 *Xrow = X + ((size_t)blockIdx.y * g.n3 + r) * g.ncols_pad;
  for (int col = tid; col < g.ncols; col += NT) {
    const int ab = g.col_ab[col];
    Xrow[col] = pl[pos<N1>(ab >> 16) * P2 + pos<N2>(ab & 0xffff)];
  }
}

// V_KS in the permuted plane order: Vp[r][pa][pb] = v[(ia*n2+ib)*n3+ic]
// with ia = ipos_N1(pa), ib = ipos_N2(pb), ic = ipos_N3(r).
template <typename T, int N1, int N2, int N3>
__global__ void kf_vks_perm(const double *__restrict__ v, T *__restrict__ Vp) {
  const size_t N = (size_t)N1 * N2 * N3;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    const int pb = (int)(i % N2);
    const int pa = (int)((i / N2) % N1);
    const int r = (int)(i / ((size_t)N1 * N2));
    const int ia = ipos<N1>(pa), ib = ipos<N2>(pb), ic = ipos<N3>(r);
    Vp[i] = (T)v[((size_t)ia * N2 + ib) * N3 + ic];
  }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
template <int N> static constexpr int r1_of() { return Plan<N>::R1; }

template <typename T> static size_t pl_smem(int n1, int n2) {
  return sizeof(typename CT<T>::type) * (size_t)(n1 + n2 + n1 * (n2 + 1));
}

#define SDFT_FOR_N3(X)                \
  switch (g.n3) {                     \
    case 24: X(24); break;            \
    case 48: X(48); break;            \
    case 72: X(72); break;            \
    case 96: X(96); break;            \
    default: return false;            \
  }

#define SDFT_FOR_PLANE(X)                                             \
  do {                                                                \
    const int key = g.n1 * 1000 + g.n2;                               \
    switch (key) {                                                    \
      case 24024: X(24, 24); break;                                   \
      case 24048: X(24, 48); break;                                   \
      case 24072: X(24, 72); break;                                   \
      case 48024: X(48, 24); break;                                   \
      case 48048: X(48, 48); break;                                   \
      case 48072: X(48, 72); break;                                   \
      case 72024: X(72, 24); break;                                   \
      case 72048: X(72, 48); break;                                   \
      case 72072: X(72, 72); break;                                   \
      case 96096: X(96, 96); break;                                   \
      default: return false;                                          \
    }                                                                 \
  } while (0)

bool fast_supported(int n1, int n2, int n3) {
  auto ok = [](int n) { return n == 24 || n == 48 || n == 72 || n == 96; };
  if (!ok(n1) || !ok(n2) || !ok(n3)) return false;
  const int key = n1 * 1000 + n2;
  switch (key) {
    case 24024: case 24048: case 24072: case 48024: case 48048: case 48072:
    case 72024: case 72048: case 72072: case 96096: return true;
    default: return false;
  }
}

static void plan3(int n3, int &r1, int &r2) {
  switch (n3) {
    case 24: r1 = Plan<24>::R1; r2 = Plan<24>::R2; break;
    case 48: r1 = Plan<48>::R1; r2 = Plan<48>::R2; break;
    case 72: r1 = Plan<72>::R1; r2 = Plan<72>::R2; break;
    default: r1 = Plan<96>::R1; r2 = Plan<96>::R2; break;
  }
}

template <typename T>
bool fast_stage_a(const DevGeom &g, const double *C, int nstate, int pair0, int npairs, void *X, cudaStream_t st) {
  dim3 grid(g.nbatch, npairs);
#define LA(N) kf_stage_a<T, N><<<grid, kColThreads, 0, st>>>(g, C, nstate, pair0, (typename CT<T>::type *)X)
  SDFT_FOR_N3(LA);
#undef LA
  return true;
}

template <typename T>
bool fast_stage_c(const DevGeom &g, const void *X, const EpiArgs &e, int npairs, cudaStream_t st) {
  dim3 grid(g.nbatch, npairs);
  const bool hot = e.dots == nullptr && (e.mode == EPI_CHEB1 || e.mode == EPI_CHEBK || e.mode == EPI_NEWTON);
#define LC(N)                                                                                \
  do {                                                                                       \
    if (hot) kf_stage_c<T, N, true><<<grid, kCThreads, 0, st>>>(g, (const typename CT<T>::type *)X, e);  \
    else kf_stage_c<T, N, false><<<grid, kCThreads, 0, st>>>(g, (const typename CT<T>::type *)X, e);     \
  } while (0)
  SDFT_FOR_N3(LC);
#undef LC
  return true;
}

template <typename T, int A, int B, int NT, int MINB, int PM>
static void launch_plane_b(const DevGeom &g, dim3 grid, size_t sm, void *X, const T *Vp, cudaStream_t st) {
  auto k = kf_stage_b<T, A, B, NT, MINB, PM>;
  static const bool attr_once = (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), true);
  (void)attr_once;
  k<<<grid, NT, sm, st>>>(g, (typename CT<T>::type *)X, Vp);
}

template <typename T>
bool fast_stage_b(const DevGeom &g, void *X, const T *Vp, int npairs, cudaStream_t st) {
  dim3 grid(g.n3, npairs);
  const size_t sm = pl_smem<T>(g.n1, g.n2);
  const bool small = std::is_same<T, float>::value && g.plane_nt == 128;
  // the j1 = 3, 4 band skipped where both edges factor with R1 = 8 and the
  // sphere is narrower than 3/8 of them (DevGeom::prune34)
#define LBP(NT_, MB_)                                                                                     \
  do {                                                                                                    \
    if (pm == 2) launch_plane_b<T, A, B, NT_, MB_, (ok34 ? 2 : 0)>(g, grid, sm, X, Vp, st);               \
    else if (pm == 1) launch_plane_b<T, A, B, NT_, MB_, (ok34 ? 1 : 0)>(g, grid, sm, X, Vp, st);          \
    else launch_plane_b<T, A, B, NT_, MB_, 0>(g, grid, sm, X, Vp, st);                                    \
  } while (0)
#define LB(A_, B_)                                                                                        \
  do {                                                                                                    \
    constexpr int A = A_, B = B_;                                                                         \
    constexpr bool ok34 = Plan<A>::R1 == 8 && Plan<B>::R1 == 8;                                           \
    const int pm = ok34 ? g.prune34 : 0;                                                                  \
    if (small) LBP(128, 6);                                                                               \
    else LBP(PlaneCfg<T>::NT, PlaneCfg<T>::MINB);                                                         \
  } while (0)
  SDFT_FOR_PLANE(LB);
#undef LB
#undef LBP
  return true;
}

template <typename T>
bool fast_stage_b_density(const DevGeom &g, const void *X, int npairs, double *rho_pair, cudaStream_t st) {
  dim3 grid(g.n3, npairs);
  const size_t sm = pl_smem<T>(g.n1, g.n2);
  int r1, r2;
  plan3(g.n3, r1, r2);
#define LD(A, B)                                                                               \
  do {                                                                                         \
    auto k = kf_stage_b_density<T, A, B>;                                                      \
    static const bool attr_once = (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), true); (void)attr_once;             \
    k<<<grid, PlaneCfg<T>::NT, sm, st>>>(g, (const typename CT<T>::type *)X, rho_pair, r1, r2); \
  } while (0)
  SDFT_FOR_PLANE(LD);
#undef LD
  return true;
}

template <typename T>
bool fast_stage_b_noise(const DevGeom &g, const unsigned char *neg, int nstate, int pair0, int npairs, void *X,
                        cudaStream_t st) {
  dim3 grid(g.n3, npairs);
  const size_t sm = pl_smem<T>(g.n1, g.n2);
  int r1, r2;
  plan3(g.n3, r1, r2);
#define LN(A, B)                                                                                        \
  do {                                                                                                  \
    auto k = kf_stage_b_noise<T, A, B>;                                                                 \
    static const bool attr_once = (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), true); (void)attr_once;                      \
    k<<<grid, PlaneCfg<T>::NT, sm, st>>>(g, neg, nstate, pair0, (typename CT<T>::type *)X, r1, r2);   \
  } while (0)
  SDFT_FOR_PLANE(LN);
#undef LN
  return true;
}

template <typename T>
bool fast_vks_perm(const DevGeom &g, const double *v, T *Vp, cudaStream_t st) {
  const size_t N = (size_t)g.n1 * g.n2 * g.n3;
  int blocks = (int)std::min<size_t>((N + 255) / 256, 148 * 16);
#define LV3(A, B, Cc) kf_vks_perm<T, A, B, Cc><<<blocks, 256, 0, st>>>(v, Vp)
#define LV(A, B)                                            \
  do {                                                      \
    switch (g.n3) {                                         \
      case 24: LV3(A, B, 24); break;                        \
      case 48: LV3(A, B, 48); break;                        \
      case 72: LV3(A, B, 72); break;                        \
      case 96: LV3(A, B, 96); break;                        \
      default: return false;                                \
    }                                                       \
  } while (0)
  SDFT_FOR_PLANE(LV);
#undef LV
#undef LV3
  return true;
}

template bool fast_stage_a<double>(const DevGeom &, const double *, int, int, int, void *, cudaStream_t);
template bool fast_stage_a<float>(const DevGeom &, const double *, int, int, int, void *, cudaStream_t);
template bool fast_stage_c<double>(const DevGeom &, const void *, const EpiArgs &, int, cudaStream_t);
template bool fast_stage_c<float>(const DevGeom &, const void *, const EpiArgs &, int, cudaStream_t);
template bool fast_stage_b<double>(const DevGeom &, void *, const double *, int, cudaStream_t);
template bool fast_stage_b<float>(const DevGeom &, void *, const float *, int, cudaStream_t);
template bool fast_stage_b_density<double>(const DevGeom &, const void *, int, double *, cudaStream_t);
template bool fast_stage_b_density<float>(const DevGeom &, const void *, int, double *, cudaStream_t);
template bool fast_stage_b_noise<double>(const DevGeom &, const unsigned char *, int, int, int, void *, cudaStream_t);
template bool fast_stage_b_noise<float>(const DevGeom &, const unsigned char *, int, int, int, void *, cudaStream_t);
template bool fast_vks_perm<double>(const DevGeom &, const double *, double *, cudaStream_t);
template bool fast_vks_perm<float>(const DevGeom &, const double *, float *, cudaStream_t);

}  // namespace sdft
