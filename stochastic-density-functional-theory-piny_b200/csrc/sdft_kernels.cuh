// sdft_kernels.cuh -- device geometry + kernel launch wrappers shared by
// sdft_kernels.cu (definitions) and sdft_api.cu (context / C ABI).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace sdft {

// Column-pair batch of the column stages.
constexpr int kCPB = 8;          // column pairs per CTA (16 columns)
constexpr int kColThreads = 256; // threads of the column stages

// Device view of the G sphere and FFT grid.
struct DevGeom {
  int n1, n2, n3;       // nkf1 (a), nkf2 (b), nkf3 (c)
  int N;                // n1*n2*n3
  int ncoef;            // half sphere + G=0 (last)
  int ngp;              // pitch of one re (or im) block of an orbital
  int ncols, ncols_pad, ncp, kamax;
  int nbatch;           // ceil(ncp / kCPB)
  const int2 *kb_rng;   // [n1] per plane row a: signed kb range [x, y] of its sphere columns
  int kb_contig;        // every row's columns fill its kb range (else kb_rng is not used)
  int plane_nt;         // FP32 plane stage threads per CTA: 256 or 128
  int kbmax;            // largest |kb| of the sphere columns
  int prune34;          // 1: 8 kamax < 3 n1 and 8 kbmax < 3 n2, the plane passes skip the j1 = 3, 4 band;
                        // 2: also 4 kamax >= n1, the a-pass rows with j1 = 0, 1, 6, 7 are all inside
  const int *cp_gstart; // [ncp] first G index of the pair's direct column
  const int *cp_gcount; // [ncp]
  const int *col_ab;    // [ncols] (ka mod n1) << 16 | (kb mod n2)
  const int *gkc;       // [ncoef] kc of each G (G=0: 0)
  const double *ak2;    // [ncoef] kinetic |G|^2 (capped), G=0: 0
  const double2 *tw1, *tw2, *tw3;   // exp(-2 pi i t/n) tables, FP64
  const float2 *tw1f, *tw2f, *tw3f; // FP32 copies
};

// Epilogue modes of the unpack stage.
enum EpiMode : int {
  EPI_HPSI = 0,    // write the raw PINY force f
  EPI_CHEB1 = 1,   // T1 = s1 f + pre c               (+acc init, +dot)
  EPI_CHEBK = 2,   // T_k = s1' f + pre' c - T_{k-2}   (+acc, +dot)
  EPI_NEWTON = 3,  // P_k = s1 f + pre c              (+acc, acc init on k==1)
  EPI_MOMK = 4,    // Chebyshev step + <chi,T>, <T,Tprev>, <T,T>
  EPI_NOISE = 5,   // noise orbital from an r->G transform
};

struct EpiArgs {
  int mode;
  int nstate;
  int pair0;             // first pair handled by this launch
  const double *C;       // current vector (T_{k-1}) [S][2][ngp]
  const double *PREV;    // T_{k-2} (CHEBK/MOMK)
  double *OUT;           // output vector (may alias PREV or C)
  const double *CHI;     // chi (moment dots)
  const double *FNL;     // nonlocal force or nullptr
  const float *FNLf;     // the same in FP32 (mixed precision), or nullptr
  double *ACC;           // [nmu][S][2][ngp] or nullptr
  const double *acoef;   // device: a[k*nmu + imu] of this step (nmu values)
  const double *acoef0;  // device: a[imu] (k = 0) when initialising ACC, else nullptr
  const double *acoefp;  // device: a[(k-1)*nmu + imu] when this step also adds the
                         // previous vector (C): ACC += a_{k-1} C + a_k OUT; else nullptr
  int nmu;
  size_t acc_stride;     // elements between ACC chem-pot blocks
  double s1, s2, pre;    // G!=0 scale, G=0 scale, c coefficient
  double *dots;          // per-CTA partials [pairs][nbatch][3] or nullptr
  int ndots;             // 1 (filter moments) or 3 (doubling)
  double invN;
  void *Xnext;           // column scratch to receive the packed, c-transformed OUT
                         // (stage A of the next H application; fast path), or nullptr
  bool pack_next;        // set by the loops: a next application follows this step
  unsigned long long *omax;  // per orbital: atomicMax of max|OUT| (bits of a
                             // non-negative double; +inf if not finite), or nullptr
};

// |x| as an order-preserving key for atomicMax on the bit pattern; non-finite -> +inf
__device__ __forceinline__ double absmax_key_d(double a) { return isfinite(a) ? fabs(a) : INFINITY; }

// Block-wide max of two per-thread values, then one atomicMax per orbital
// (blockDim.x = kColThreads).
__device__ __forceinline__ void omax_flush(unsigned long long *omax, int s1, int s2, bool has2, double m1, double m2,
                                           double (*red)[2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
  }
  if (lane == 0) { red[warp][0] = m1; red[warp][1] = m2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) { m1 = fmax(m1, red[w][0]); m2 = fmax(m2, red[w][1]); }
    atomicMax(omax + s1, (unsigned long long)__double_as_longlong(m1));
    if (has2) atomicMax(omax + s2, (unsigned long long)__double_as_longlong(m2));
  }
}

// ----- launches (all on `st`) ---------------------------------------------
// Column stage A: pack pairs of orbitals into columns, backward c-FFT.
// X: [npairs][n3][ncols_pad] complex (T = double or float).
template <typename T>
void launch_stage_a(const DevGeom &g, const double *C, int nstate, int pair0, int npairs,
                    void *X, cudaStream_t st);
// Plane stage B for the local potential: b/a FFT, x V, inverse a/b FFT.
// Vp: [n3][n1][n2] potential (T).
template <typename T>
void launch_stage_b(const DevGeom &g, void *X, const T *Vp, int npairs, cudaStream_t st);
// Column stage C: forward c-FFT + unpack + epilogue.
template <typename T>
void launch_stage_c(const DevGeom &g, const void *X, const EpiArgs &e, int npairs, cudaStream_t st);
// Density: planes from X (after stage A), accumulate |psi|^2 into
// rho_part[split][N] (package layout).  Pairs [0,npairs) split in nsplit groups.
template <typename T>
void launch_stage_b_density(const DevGeom &g, const void *X, int npairs, int nsplit,
                            double *rho_part, cudaStream_t st);
void launch_density_reduce(const double *rho_part, int nsplit, int N, double scale, double *rho,
                           cudaStream_t st);
// Noise: planes of +-sqrt(N) from sign bytes [S][N] (package layout) -> forward
// a/b FFT -> X columns for stage C (mode EPI_NOISE).
template <typename T>
void launch_stage_b_noise(const DevGeom &g, const unsigned char *neg, int nstate, int pair0,
                          int npairs, void *X, cudaStream_t st);

// FP64 NT GEMM on DMMA: out[n*ldo + m] = sum_p A[m*lda + p] * B[n*ldb + p]
// (beta = 0).  M, N, K must be multiples of 128, 64, 16 (padded buffers);
// only m < Mst, n < Nst are stored.  split > 1 writes partials to
// work[split][N][ldo] and reduces in fixed order.
void launch_gemm_nt_f64(const double *A, int lda, const double *B, int ldb, double *out, int ldo,
                        int M, int N, int K, int Mst, int Nst, int split, double *work,
                        cudaStream_t st);

// sum over nparts CTA partials (3 doubles each) -> out[0, ndots); blk: kDotBlocks*3
// doubles of scratch (two launches, fixed order)
constexpr int kDotBlocks = 128;
void launch_dots_reduce(const double *part, int nparts, int ndots, double *blk, double *out, cudaStream_t st);
// E_NL = sum_u w[u] sum_{s<nstate} Z[s*ldz + u]^2 -> out[0]; out[1 .. kEnlBlocks]
// hold the partials (two launches)
constexpr int kEnlBlocks = 128;
void launch_enl(const double *Z, int ldz, const double *w, int P, int nstate, double *out,
                cudaStream_t st);
// dst[i] = a*src[i] over n doubles (acc init etc.)
void launch_scale_copy(const double *src, double *dst, double a, size_t n, cudaStream_t st);
// Vp[(ic*n1+ia)*n2+ib] = v[(ia*n2+ib)*n3+ic] (T)
template <typename T>
void launch_vks_transpose(const double *v, T *Vp, int n1, int n2, int n3, cudaStream_t st);

}  // namespace sdft
