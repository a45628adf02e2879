// sdft_fft2.cuh -- compile-time-size line FFTs for the fast path.
//
// A line of N = R1*R2 points is transformed in two passes over shared
// memory (the "four-step" factorisation N = R1 x R2 without the explicit
// transpose):
//
//   forward, natural -> permuted ("DIF" order, dif()):
//     pass 1, per (line, j2):  R1-point DFT of x[j2 + R2*j1] over j1, times
//                              w_N^(j2*k1), stored back at j2 + R2*k1
//     pass 2, per (line, k1):  R2-point DFT of the block R2*k1 + [0,R2),
//                              stored back in place
//     -> frequency k1 + R1*k2 ends up at position R2*k1 + k2.
//   reverse, permuted -> natural ("DIT" order, dit()): the two passes in
//     the opposite order with the same twiddles; either sign.
//
// Every unit reads and writes only its own positions, so a pass needs no
// barrier between its loads and stores (no butterflies held across a
// barrier, low register pressure); one __syncthreads separates the passes.
// Consumers index the permuted order directly (pos()/ipos()), so no data is
// ever moved just to undo the permutation.  The R-point DFTs run in
// registers with compile-time twiddles (sdft_twiddles.cuh).
#pragma once
#include "sdft_fft.cuh"
#include "sdft_twiddles.cuh"

namespace sdft {

template <int N> struct Plan;
template <> struct Plan<12> { static constexpr int R1 = 4, R2 = 3; };
template <> struct Plan<16> { static constexpr int R1 = 4, R2 = 4; };
template <> struct Plan<24> { static constexpr int R1 = 4, R2 = 6; };
template <> struct Plan<32> { static constexpr int R1 = 4, R2 = 8; };
template <> struct Plan<36> { static constexpr int R1 = 6, R2 = 6; };
template <> struct Plan<48> { static constexpr int R1 = 8, R2 = 6; };
template <> struct Plan<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct Plan<72> { static constexpr int R1 = 8, R2 = 9; };
template <> struct Plan<96> { static constexpr int R1 = 8, R2 = 12; };
template <> struct Plan<128> { static constexpr int R1 = 8, R2 = 16; };

// position of (frequency or real-space) index k after a dif() pass pair
template <int N> __device__ __forceinline__ int pos(int k) {
  return Plan<N>::R2 * (k % Plan<N>::R1) + k / Plan<N>::R1;
}
// index stored at position p
template <int N> __device__ __forceinline__ int ipos(int p) {
  return (p % Plan<N>::R2) * Plan<N>::R1 + p / Plan<N>::R2;
}

template <int R> __device__ __forceinline__ double twc_re(int t);
template <int R> __device__ __forceinline__ double twc_im(int t);
#define SDFT_TW(R)                                                                         \
  template <> __device__ __forceinline__ double twc_re<R>(int t) { return kTw##R##re[t]; } \
  template <> __device__ __forceinline__ double twc_im<R>(int t) { return kTw##R##im[t]; }
SDFT_TW(6)
SDFT_TW(8)
SDFT_TW(9)
SDFT_TW(12)
SDFT_TW(16)
SDFT_TW(24)
SDFT_TW(32)
#undef SDFT_TW

template <int R> struct F1 { static constexpr int A = (R % 4 == 0 && R > 4) ? 4 : ((R % 3 == 0) ? 3 : 2); };

// In-register R-point DFT, natural order in and out, sign DIR.
template <int R, int DIR, typename C> __device__ __forceinline__ void dftr(C *v) {
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2 || R == 3 || R == 4) {
    dft_small<R, DIR>(v);
  } else {
    constexpr int A = F1<R>::A, B = R / A;
    using T = decltype(v[0].x);
    C y[R];
#pragma unroll
    for (int j2 = 0; j2 < B; j2++) {
      C t[A];
#pragma unroll
      for (int j1 = 0; j1 < A; j1++) t[j1] = v[j2 + B * j1];
      dftr<A, DIR>(t);
#pragma unroll
      for (int k1 = 0; k1 < A; k1++) {
        const int e = j2 * k1;  // < R
        if (e == 0) {
          y[j2 + B * k1] = t[k1];
        } else {
          C w;
          w.x = (T)twc_re<R>(e);
          w.y = (T)(DIR < 0 ? twc_im<R>(e) : -twc_im<R>(e));
          y[j2 + B * k1] = cmul(t[k1], w);
        }
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < A; k1++) {
      C t[B];
#pragma unroll
      for (int j2 = 0; j2 < B; j2++) t[j2] = y[j2 + B * k1];
      dftr<B, DIR>(t);
#pragma unroll
      for (int k2 = 0; k2 < B; k2++) v[k1 + A * k2] = t[k2];
    }
  }
}

// Line addressing for the two-pass FFTs.  base(l) is the offset of line l,
// ES the element stride (compile time).
struct Lines1 {  // lines at l*ls
  int ls;
  __device__ __forceinline__ int base(int l) const { return l * ls; }
  __device__ __forceinline__ bool valid(int) const { return true; }
};
struct Lines2 {  // two contiguous groups of lines (rows 0..n1-1 and the top ones)
  int nl1, ls, off2;
  __device__ __forceinline__ int base(int l) const { return (l < nl1) ? l * ls : off2 + (l - nl1) * ls; }
  __device__ __forceinline__ bool valid(int) const { return true; }
};
// Two groups of rows (n1r rows from row 0, n2r rows from offset off2), each
// enumerated over a multiple of 16 lanes (g1, g2): every half-warp then
// touches 16 consecutive rows of one group, which with an odd row pitch
// (in complex elements) hit disjoint banks.  Padding lanes are not valid.
struct Lines2P {
  int n1r, g1, n2r, ls, off2;
  __device__ __forceinline__ int base(int l) const { return (l < g1) ? l * ls : off2 + (l - g1) * ls; }
  __device__ __forceinline__ bool valid(int l) const { return (l < g1) ? (l < n1r) : (l - g1 < n2r); }
};

// Unit (line l, index j) enumeration for the passes below: lines vary
// fastest across threads, so a warp touches 32 consecutive lines at the same
// j.  With line pitches of N+1 complex (odd) or unit pitch, consecutive lines
// fall in distinct banks (no shared-memory bank conflicts) and the twiddle
// index j is uniform across most of a warp (broadcast loads).  The stepping
// avoids a runtime division per unit.
struct UnitIter {
  int l, j, dl, dj, nl;
  __device__ __forceinline__ UnitIter(int tid, int nthr, int nlines) : nl(nlines) {
    dj = nthr / nl;
    dl = nthr - dj * nl;
    j = tid / nl;
    l = tid - j * nl;
  }
  __device__ __forceinline__ void next() {
    l += dl;
    j += dj;
    if (l >= nl) { l -= nl; j++; }
  }
};

// Twiddle source of dif/dit: exp(-2 pi i t/N) from a shared-memory table
// (pointer) or from an accessor object with operator()(t).
template <typename C, typename P> __device__ __forceinline__ C tw_at(P *tw, int t) { return lds_tw(tw + t); }
template <typename C, typename TW> __device__ __forceinline__ C tw_at(const TW &tw, int t) { return tw(t); }

// Elements of a line that hold data (mask.line(l)(k) for natural index k of
// line l): dif reads only those on input (the others count as zero and need
// not be stored), dit writes only those on output.  AllElems: every element.
struct AllK {
  __device__ __forceinline__ bool operator()(int) const { return true; }
};
struct AllElems {
  __device__ __forceinline__ AllK line(int) const { return AllK{}; }
};

// P34 (R1 = 8 only): the elements j2 + R2 j1 with j1 = 3, 4 -- natural
// indices 3N/8 .. 5N/8 - 1, i.e. |k| >= 3N/8 -- hold no data on input (dif)
// and are not needed on output (dit), as for a sphere narrower than 3N/8:
// they are neither read nor written, and no mask is evaluated for them.
template <int R1> __device__ __forceinline__ constexpr bool band34(bool p34, int j1) {
  return p34 && R1 == 8 && (j1 == 3 || j1 == 4);
}

// natural -> permuted.  twN: exp(-2 pi i t/N) (shared-memory table or accessor).
template <int N, int ES, int DIR, bool P34 = false, typename C, typename LM, typename TW, typename MK = AllElems>
__device__ __forceinline__ void dif(C *buf, const LM &lm, int nl, const TW &twN, int tid, int nthr,
                                    const MK &mask = MK{}) {
  constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
  static_assert(!P34 || R1 == 8, "the j1 = 3, 4 band needs R1 = 8");
  if (nl > 0) {
#pragma unroll 1
    for (UnitIter it(tid, nthr, nl); it.j < R2; it.next()) {
      const int l = it.l, j2 = it.j;
      if (!lm.valid(l)) continue;
      C *p = buf + lm.base(l);
      C v[R1];
      const auto in = mask.line(l);
#pragma unroll
      for (int j1 = 0; j1 < R1; j1++) {
        const int k = j2 + R2 * j1;
        v[j1] = (!band34<R1>(P34, j1) && in(k)) ? p[k * ES] : cmk<C>(0.0, 0.0);
      }
      dftr<R1, DIR>(v);
      p[j2 * ES] = v[0];
#pragma unroll
      for (int k1 = 1; k1 < R1; k1++) {
        C w = tw_at<C>(twN, j2 * k1);
        if (DIR > 0) w.y = -w.y;
        p[(j2 + R2 * k1) * ES] = cmul(v[k1], w);
      }
    }
  }
  __syncthreads();
  if (nl > 0) {
#pragma unroll 1
    for (UnitIter it(tid, nthr, nl); it.j < R1; it.next()) {
      const int l = it.l, k1 = it.j;
      if (!lm.valid(l)) continue;
      C *p = buf + lm.base(l) + R2 * k1 * ES;
      C v[R2];
#pragma unroll
      for (int j = 0; j < R2; j++) v[j] = p[j * ES];
      dftr<R2, DIR>(v);
#pragma unroll
      for (int j = 0; j < R2; j++) p[j * ES] = v[j];
    }
  }
  __syncthreads();
}

// permuted -> natural
template <int N, int ES, int DIR, bool P34 = false, typename C, typename LM, typename TW, typename MK = AllElems>
__device__ __forceinline__ void dit(C *buf, const LM &lm, int nl, const TW &twN, int tid, int nthr,
                                    const MK &mask = MK{}) {
  constexpr int R1 = Plan<N>::R1, R2 = Plan<N>::R2;
  static_assert(!P34 || R1 == 8, "the j1 = 3, 4 band needs R1 = 8");
  if (nl > 0) {
#pragma unroll 1
    for (UnitIter it(tid, nthr, nl); it.j < R1; it.next()) {
      const int l = it.l, k1 = it.j;
      if (!lm.valid(l)) continue;
      C *p = buf + lm.base(l) + R2 * k1 * ES;
      C v[R2];
#pragma unroll
      for (int j = 0; j < R2; j++) v[j] = p[j * ES];
      dftr<R2, DIR>(v);
      p[0] = v[0];
#pragma unroll
      for (int j2 = 1; j2 < R2; j2++) {
        C w = tw_at<C>(twN, j2 * k1);
        if (DIR > 0) w.y = -w.y;
        p[j2 * ES] = cmul(v[j2], w);
      }
    }
  }
  __syncthreads();
  if (nl > 0) {
#pragma unroll 1
    for (UnitIter it(tid, nthr, nl); it.j < R2; it.next()) {
      const int l = it.l, j2 = it.j;
      if (!lm.valid(l)) continue;
      C *p = buf + lm.base(l);
      C v[R1];
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) v[k1] = p[(R2 * k1 + j2) * ES];
      dftr<R1, DIR>(v);
      const auto out = mask.line(l);
#pragma unroll
      for (int j1 = 0; j1 < R1; j1++) {
        const int k = j2 + R2 * j1;
        if (!band34<R1>(P34, j1) && out(k)) p[k * ES] = v[j1];
      }
    }
  }
  __syncthreads();
}

}  // namespace sdft
