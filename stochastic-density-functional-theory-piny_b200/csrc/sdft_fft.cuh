// sdft_fft.cuh -- shared-memory batched FFT building blocks (sm_100a).
//
// Lines of length n = 2^a 3^b (n <= 128) live in shared memory; element j
// of line l sits at buf[base(l) + j*es].  Each radix stage is the
// self-sorting Stockham iteration (Govindaraju et al., "High performance
// discrete Fourier transforms on graphics processors", SC'08): butterfly j
// reads x[j + q*n/R], applies twiddle w^(q*(j mod Ns)), performs an R-point
// DFT and writes y[(j/Ns)*Ns*R + (j mod Ns) + q*Ns].  The stage runs in
// place: every thread first loads all of its butterflies into registers,
// the block synchronises, then every thread stores.  dir = -1 is the
// forward transform exp(-2 pi i jk/n) (FFTW_FORWARD), dir = +1 the
// unnormalised backward one (FFTW_BACKWARD).
#pragma once
#include <cuda_runtime.h>

namespace sdft {

template <typename T> struct CT;
template <> struct CT<double> { using type = double2; };
template <> struct CT<float> { using type = float2; };

template <typename C> __device__ __forceinline__ C cmk(double r, double i) {
  C c; c.x = (decltype(c.x))r; c.y = (decltype(c.y))i; return c;
}
// FP32 complex arithmetic on the packed f32x2 pipe (sm_100): one
// instruction per complex add/sub/scale, two per complex multiply.
__device__ __forceinline__ unsigned long long pk2(float x, float y) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a.x, a.y)), "l"(pk2(b.x, b.y)));
  return upk2(r);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a.x, a.y)), "l"(pk2(b.x, b.y)));
  return upk2(r);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a.x, a.y)), "l"(pk2(b.x, b.y)));
  return upk2(r);
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk2(a.x, a.y)), "l"(pk2(b.x, b.y)), "l"(pk2(c.x, c.y)));
  return upk2(r);
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return add2(a, b); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return sub2(a, b); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// (a.x b.x - a.y b.y, a.x b.y + a.y b.x) = a.x (b.x, b.y) + a.y (-b.y, b.x)
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return fma2(make_float2(a.y, a.y), make_float2(-b.y, b.x), mul2(make_float2(a.x, a.x), b));
}
// s * (a.x, a.y) for a real s
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return mul2(a, make_float2(s, s)); }
// multiply by (dir * i): dir=-1 -> -i, dir=+1 -> +i
template <int DIR, typename C> __device__ __forceinline__ C mul_i(C a) {
  C r;
  if (DIR > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

template <int R, int DIR, typename C> __device__ __forceinline__ void dft_small(C *v) {
  if (R == 2) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    C b0 = cadd(v[1], v[3]), b1 = mul_i<DIR>(csub(v[1], v[3]));
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1);
    v[3] = csub(a1, b1);
  } else {  // R == 3: w = exp(DIR*2 pi i/3) = -1/2 + DIR*i*sqrt(3)/2
    using T = decltype(v[0].x);
    const T hs = (T)0.86602540378443864676372317075294;  // sqrt(3)/2
    C s = cadd(v[1], v[2]);
    C d = csub(v[1], v[2]);
    const C m = csub(v[0], cscale(s, (T)0.5));
    const C rot = cscale(mul_i<DIR>(d), hs);
    v[0] = cadd(v[0], s);
    v[1] = cadd(m, rot);
    v[2] = csub(m, rot);
  }
}

// Twiddle loads from shared memory.  asm volatile keeps them inside loops
// that run several transforms (otherwise they are hoisted as loop
// invariants and the live registers spill).
__device__ __forceinline__ double2 lds_tw(const double2 *p) {
  double2 r;
  unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v2.f64 {%0,%1}, [%2];" : "=d"(r.x), "=d"(r.y) : "r"(a));
  return r;
}
__device__ __forceinline__ float2 lds_tw(const float2 *p) {
  float2 r;
  unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];" : "=f"(r.x), "=f"(r.y) : "r"(a));
  return r;
}

// Line addressing: lines [0,nl1) at l*ls, lines [nl1,nl) at off2+(l-nl1)*ls.
struct LineMap {
  int nl, nl1, ls, off2, es;
  __device__ __forceinline__ int base(int l) const { return (l < nl1) ? l * ls : off2 + (l - nl1) * ls; }
};

// One in-place Stockham stage.  MAXB bounds the butterflies per thread; the
// caller guarantees ceil(nl*n/R / nthr) <= MAXB.  tw[t] = exp(-2 pi i t/n)
// must live in shared memory.
template <int R, int DIR, int MAXB, typename C>
__device__ __forceinline__ void fft_stage(C *buf, int n, const LineMap &lm, int Ns, const C *tw,
                                          int nthr, int tid) {
  const int m = n / R;
  const int total = lm.nl * m;
  const int twstep = n / (Ns * R);
  C v[MAXB][R];
#pragma unroll
  for (int i = 0; i < MAXB; i++) {
    int b = tid + i * nthr;
    if (b < total) {
      int l = b / m, j = b - l * m;
      int k = j % Ns;
      const C *p = buf + lm.base(l);
#pragma unroll
      for (int q = 0; q < R; q++) {
        C x = p[(j + q * m) * lm.es];
        if (q > 0) {
          C w = lds_tw(tw + (q * k * twstep) % n);
          if (DIR > 0) w.y = -w.y;
          x = cmul(x, w);
        }
        v[i][q] = x;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < MAXB; i++) {
    int b = tid + i * nthr;
    if (b < total) {
      int l = b / m, j = b - l * m;
      int k = j % Ns;
      dft_small<R, DIR>(v[i]);
      C *p = buf + lm.base(l);
      int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int q = 0; q < R; q++) p[(idxD + q * Ns) * lm.es] = v[i][q];
    }
  }
  __syncthreads();
}

// Full FFT of all lines described by lm.  Radix order: 4s, then 2, then 3s
// (the same order the host plan uses).  MAXE bounds elements per thread.
template <int DIR, int MAXE, typename C>
__device__ __forceinline__ void fft_lines(C *buf, int n, const LineMap &lm, const C *tw, int nthr, int tid) {
  int rem = n, Ns = 1;
  while (rem % 4 == 0) {
    fft_stage<4, DIR, (MAXE + 3) / 4>(buf, n, lm, Ns, tw, nthr, tid);
    Ns *= 4; rem /= 4;
  }
  while (rem % 2 == 0) {
    fft_stage<2, DIR, (MAXE + 1) / 2>(buf, n, lm, Ns, tw, nthr, tid);
    Ns *= 2; rem /= 2;
  }
  while (rem % 3 == 0) {
    fft_stage<3, DIR, (MAXE + 2) / 3>(buf, n, lm, Ns, tw, nthr, tid);
    Ns *= 3; rem /= 3;
  }
}

}  // namespace sdft
