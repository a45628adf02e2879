// sdft_mixer.cu -- density mixing (genDensityMix, stodft/diis.c:34-464) and
// its checkpoint file (checkpointOutput / checkpointInput,
// stodft/checkpointIO.c:32-533), with the densities on the device.
//
// State: the last num_diis + 1 corrected densities ("bank", newest first),
// the last num_diis errors rho_correct - rho_old and rho_old, all device
// buffers; banking rotates buffer pointers and copies the new vector in.
// One SCF step:
//   iscf == 0                : bank rho_correct, rho_old = rho_correct
//                              (the output density is not written);
//   1 <= iscf <= num_step_mix: rho = rho_correct (1 - r) + bank[0] r, r =
//                              mix_ratio_big (bank[0] is rho_correct itself
//                              after the banking, as in the reference);
//   iscf > num_step_mix      : DIIS on the n = min(iscf, num_diis) newest
//                              errors: B_ij = <err_i|err_j> (device,
//                              fixed-order reduction), the bordered system
//                              [[B, -m], [-m^T, 0]] x = (0, .., 0, -m), m =
//                              max |B_ij|, solved by pseudo-inverse (singular
//                              values below 1e-10 of the largest dropped;
//                              symmetric Jacobi eigen-decomposition on the
//                              host), rho = sum_i x_i (bank_i + (alpha - 1)
//                              err_i), alpha = mix_ratio_sm (iscf <= 10) or
//                              mix_ratio_sm2;
//   rho_old = rho.
// The elementwise arithmetic is evaluated in the reference's order without
// contraction, so the banked and simply mixed densities are bitwise those
// of the reference.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "sdft_internal.h"

struct sdft_mixer {
  int device = 0;
  cudaStream_t st = nullptr;
  long long n = 0;
  int num_diis = 0, num_step_mix = 0;
  double r_big = 0.0, r_sm = 0.0, r_sm2 = 0.0;
  int iscf = -1, num_diis_now = 0;
  std::vector<double *> bank;  // num_diis + 1 (nullptr = empty)
  std::vector<double *> err;   // num_diis
  std::vector<double> coef;    // DIIS coefficients of the last DIIS step
  double *old = nullptr, *in = nullptr, *out = nullptr;
  double *part = nullptr;      // dot partials [pairs][kMixBlocks]
  double *dots = nullptr;      // [pairs]
  double *dcoef = nullptr;     // [num_diis]
  const double **dptr = nullptr;  // [2 num_diis]: bank, err pointers for the combination
};

namespace sdft {
namespace {

constexpr int kMixBlocks = 256, kMixThreads = 256, kMaxDiis = 16;

__global__ void k_mix_err(double *__restrict__ e, const double *__restrict__ in, const double *__restrict__ old,
                          long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    e[i] = __dsub_rn(in[i], old[i]);
}

__global__ void k_mix_simple(double *__restrict__ out, const double *__restrict__ in, const double *__restrict__ b0,
                             double r2, double r1, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __dadd_rn(__dmul_rn(in[i], r2), __dmul_rn(b0[i], r1));
}

// partial[y][bx] = sum over this block's elements of a_y . b_y, pair y = blockIdx.y
__global__ void __launch_bounds__(kMixThreads) k_mix_dots(const double *const *__restrict__ vec, const int2 *pairs,
                                                          long long n, double *__restrict__ part) {
  const int2 pr = pairs[blockIdx.y];
  const double *a = vec[pr.x], *b = vec[pr.y];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)kMixThreads + threadIdx.x; i < n; i += (long long)kMixBlocks * kMixThreads)
    s += a[i] * b[i];
  __shared__ double sh[kMixThreads];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int h = kMixThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(size_t)blockIdx.y * kMixBlocks + blockIdx.x] = sh[0];
}

__global__ void k_mix_dots_finish(const double *__restrict__ part, int npairs, double *__restrict__ dots) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= npairs) return;
  double s = 0.0;
  for (int b = 0; b < kMixBlocks; b++) s += part[(size_t)y * kMixBlocks + b];
  dots[y] = s;
}

// out = sum_i c_i (bank_i + pre err_i), accumulated in i order
__global__ void k_mix_diis(double *__restrict__ out, const double *const *__restrict__ ptr, const double *__restrict__ c,
                           int nv, double pre, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nv; k++) s = __dadd_rn(s, __dmul_rn(c[k], __dadd_rn(ptr[k][i], __dmul_rn(pre, ptr[nv + k][i]))));
    out[i] = s;
  }
}

unsigned grid_of(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); }

// Symmetric eigen-decomposition A = Q diag(w) Q^T (cyclic Jacobi rotations).
void jacobi_eigen(int n, std::vector<double> a, std::vector<double> &w, std::vector<double> &q) {
  q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) q[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; i++) {
      diag += a[(size_t)i * n + i] * a[(size_t)i * n + i];
      for (int j = i + 1; j < n; j++) off += a[(size_t)i * n + j] * a[(size_t)i * n + j];
    }
    if (off <= 1e-34 * diag || off == 0.0) break;
    for (int p = 0; p < n - 1; p++)
      for (int r = p + 1; r < n; r++) {
        const double apr = a[(size_t)p * n + r];
        if (apr == 0.0) continue;
        const double th = (a[(size_t)r * n + r] - a[(size_t)p * n + p]) / (2.0 * apr);
        const double t = (th >= 0.0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; k++) {  // columns p, r
          const double akp = a[(size_t)k * n + p], akr = a[(size_t)k * n + r];
          a[(size_t)k * n + p] = c * akp - s * akr;
          a[(size_t)k * n + r] = s * akp + c * akr;
        }
        for (int k = 0; k < n; k++) {  // rows p, r
          const double apk = a[(size_t)p * n + k], ark = a[(size_t)r * n + k];
          a[(size_t)p * n + k] = c * apk - s * ark;
          a[(size_t)r * n + k] = s * apk + c * ark;
        }
        for (int k = 0; k < n; k++) {
          const double qkp = q[(size_t)k * n + p], qkr = q[(size_t)k * n + r];
          q[(size_t)k * n + p] = c * qkp - s * qkr;
          q[(size_t)k * n + r] = s * qkp + c * qkr;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; i++) w[i] = a[(size_t)i * n + i];
}

// x = pseudo-inverse(A) b for symmetric A: singular values |w_i| below
// 1e-10 of the largest are dropped (matrixInvSVD's rule)
std::vector<double> pinv_solve(int n, const std::vector<double> &a, const std::vector<double> &b) {
  std::vector<double> w, q;
  jacobi_eigen(n, a, w, q);
  double smax = 0.0;
  for (double x : w) smax = std::max(smax, std::fabs(x));
  std::vector<double> x(n, 0.0);
  for (int i = 0; i < n; i++) {
    if (smax == 0.0 || !(std::fabs(w[i]) / smax > 1e-10)) continue;
    double qb = 0.0;
    for (int k = 0; k < n; k++) qb += q[(size_t)k * n + i] * b[k];
    const double f = qb / w[i];
    for (int k = 0; k < n; k++) x[k] += f * q[(size_t)k * n + i];
  }
  return x;
}

#define MCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e__ = (call);                                                         \
    if (e__ != cudaSuccess) return set_error(SDFT_ERR_CUDA, cudaGetErrorString(e__)); \
  } while (0)

int alloc_vec(sdft_mixer *m, double **p) { return dev_alloc(m->device, m->st, (void **)p, (size_t)m->n * 8); }

// n doubles between host and device (or device and device) in the mixer's
// stream order, complete on return
bool copy_sync(sdft_mixer *m, void *dst, const void *src, cudaMemcpyKind kind) {
  return cudaMemcpyAsync(dst, src, (size_t)m->n * 8, kind, m->st) == cudaSuccess &&
         cudaStreamSynchronize(m->st) == cudaSuccess;
}

// bank <- rho (newest first); the oldest buffer is reused
int bank_push(sdft_mixer *m, const double *rho) {
  double *buf = m->bank.back();
  for (int i = m->num_diis; i > 0; i--) m->bank[i] = m->bank[i - 1];
  if (!buf) {
    int r = alloc_vec(m, &buf);
    if (r) return r;
  }
  m->bank[0] = buf;
  MCK(cudaMemcpyAsync(buf, rho, (size_t)m->n * 8, cudaMemcpyDeviceToDevice, m->st));
  return SDFT_OK;
}

// err <- rho - old (newest first)
int err_push(sdft_mixer *m, const double *rho) {
  double *buf = m->err.back();
  for (int i = m->num_diis - 1; i > 0; i--) m->err[i] = m->err[i - 1];
  if (!buf) {
    int r = alloc_vec(m, &buf);
    if (r) return r;
  }
  m->err[0] = buf;
  k_mix_err<<<grid_of(m->n), 256, 0, m->st>>>(buf, rho, m->old, m->n);
  MCK(cudaGetLastError());
  return SDFT_OK;
}

int diis(sdft_mixer *m, int iscf) {
  const int n = m->num_diis_now;
  std::vector<const double *> vp(2 * n);
  for (int i = 0; i < n; i++) { vp[i] = m->bank[i]; vp[n + i] = m->err[i]; }
  std::vector<int2> pr;
  for (int i = 0; i < n; i++)
    for (int j = i; j < n; j++) pr.push_back(make_int2(n + i, n + j));
  const int np = (int)pr.size();
  // pointer table, then the pair table (int2) behind it
  MCK(cudaMemcpyAsync(m->dptr, vp.data(), vp.size() * sizeof(void *), cudaMemcpyHostToDevice, m->st));
  int2 *dpairs = reinterpret_cast<int2 *>(m->dptr + 2 * kMaxDiis);
  MCK(cudaMemcpyAsync(dpairs, pr.data(), pr.size() * sizeof(int2), cudaMemcpyHostToDevice, m->st));
  k_mix_dots<<<dim3(kMixBlocks, np), kMixThreads, 0, m->st>>>(m->dptr, dpairs, m->n, m->part);
  k_mix_dots_finish<<<(np + 127) / 128, 128, 0, m->st>>>(m->part, np, m->dots);
  MCK(cudaGetLastError());
  std::vector<double> dots(np);
  MCK(cudaMemcpyAsync(dots.data(), m->dots, np * sizeof(double), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  const int d = n + 1;
  std::vector<double> A((size_t)d * d, 0.0), b(d, 0.0);
  double mx = -1000.0;
  for (int i = 0, k = 0; i < n; i++)
    for (int j = i; j < n; j++, k++) {
      A[(size_t)i * d + j] = A[(size_t)j * d + i] = dots[k];
      mx = std::max(mx, std::fabs(dots[k]));
    }
  for (int i = 0; i < n; i++) A[(size_t)n * d + i] = A[(size_t)i * d + n] = -mx;
  b[n] = -mx;
  const std::vector<double> x = pinv_solve(d, A, b);
  m->coef.assign(x.begin(), x.begin() + n);
  MCK(cudaMemcpyAsync(m->dcoef, m->coef.data(), n * sizeof(double), cudaMemcpyHostToDevice, m->st));
  const double pre = (iscf <= 10 ? m->r_sm : m->r_sm2) - 1.0;
  k_mix_diis<<<grid_of(m->n), 256, 0, m->st>>>(m->out, m->dptr, m->dcoef, n, pre, m->n);
  MCK(cudaGetLastError());
  return SDFT_OK;
}

// text output with a large stdio buffer; "%.16lg" per value as checkpointOutput
int write_vec(FILE *f, const double *v, long long n, double scale, bool scaled) {
  for (long long i = 0; i < n; i++) {
    double x = v[i];
    if (scaled) x *= scale;
    if (fprintf(f, "%.16lg\n", x) < 0) return set_error(SDFT_ERR_ARG, "checkpoint: write failed");
  }
  return SDFT_OK;
}

int read_vec(FILE *f, double *v, long long n) {
  for (long long i = 0; i < n; i++)
    if (fscanf(f, "%lg", &v[i]) != 1) return set_error(SDFT_ERR_ARG, "checkpoint: file too short or malformed");
  return SDFT_OK;
}

}  // namespace
}  // namespace sdft

using namespace sdft;

extern "C" int sdft_mixer_create(int device, long long n, int num_diis, int num_step_mix, double mix_ratio_big,
                                 double mix_ratio_sm, double mix_ratio_sm2, sdft_mixer **out) {
  if (!out || n < 1 || num_diis < 1 || num_diis > kMaxDiis || num_step_mix < 0)
    return set_error(SDFT_ERR_ARG, "mixer_create: n >= 1, 1 <= num_diis <= 16, num_step_mix >= 0");
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return set_error(SDFT_ERR_NODEVICE, "mixer_create: no such device");
  sdft_mixer *m = new sdft_mixer;
  m->device = device;
  m->n = n;
  m->num_diis = num_diis;
  m->num_step_mix = num_step_mix;
  m->r_big = mix_ratio_big;
  m->r_sm = mix_ratio_sm;
  m->r_sm2 = mix_ratio_sm2;
  m->bank.assign(num_diis + 1, nullptr);
  m->err.assign(num_diis, nullptr);
  int r = SDFT_OK;
  if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess)
    r = set_error(SDFT_ERR_CUDA, "mixer_create: stream");
  const int maxpairs = kMaxDiis * (kMaxDiis + 1) / 2;
  if (!r) r = alloc_vec(m, &m->old);
  if (!r) r = alloc_vec(m, &m->in);
  if (!r) r = alloc_vec(m, &m->out);
  if (!r) r = dev_alloc(device, m->st, (void **)&m->part, (size_t)maxpairs * kMixBlocks * 8);
  if (!r) r = dev_alloc(device, m->st, (void **)&m->dots, (size_t)maxpairs * 8);
  if (!r) r = dev_alloc(device, m->st, (void **)&m->dcoef, (size_t)kMaxDiis * 8);
  if (!r) r = dev_alloc(device, m->st, (void **)&m->dptr, 2 * kMaxDiis * sizeof(void *) + maxpairs * sizeof(int2));
  if (r) {
    sdft_mixer_destroy(m);
    return r;
  }
  *out = m;
  return SDFT_OK;
}

extern "C" int sdft_mixer_destroy(sdft_mixer *m) {
  if (!m) return SDFT_OK;
  cudaSetDevice(m->device);
  for (double *p : m->bank) dev_free(p, m->st);
  for (double *p : m->err) dev_free(p, m->st);
  for (void *p : {(void *)m->old, (void *)m->in, (void *)m->out, (void *)m->part, (void *)m->dots, (void *)m->dcoef,
                  (void *)m->dptr})
    dev_free(p, m->st);
  if (m->st) {
    cudaStreamSynchronize(m->st);
    cudaStreamDestroy(m->st);
  }
  delete m;
  return SDFT_OK;
}

extern "C" int sdft_mixer_step(sdft_mixer *m, int iscf, const double *rho_correct, double *rho) {
  if (!m || iscf < 0 || !rho_correct || !rho) return set_error(SDFT_ERR_ARG, "mixer_step: bad argument");
  cudaSetDevice(m->device);
  const size_t bytes = (size_t)m->n * 8;
  MCK(cudaMemcpyAsync(m->in, rho_correct, bytes, cudaMemcpyDefault, m->st));
  m->num_diis_now = std::min(iscf, m->num_diis);
  m->iscf = iscf;
  int r;
  if (iscf == 0) {
    if ((r = bank_push(m, m->in))) return r;
    MCK(cudaMemcpyAsync(m->old, m->in, bytes, cudaMemcpyDeviceToDevice, m->st));
    MCK(cudaStreamSynchronize(m->st));
    return SDFT_OK;
  }
  if ((r = err_push(m, m->in)) || (r = bank_push(m, m->in))) return r;
  if (iscf <= m->num_step_mix) {
    k_mix_simple<<<grid_of(m->n), 256, 0, m->st>>>(m->out, m->in, m->bank[0], 1.0 - m->r_big, m->r_big, m->n);
    MCK(cudaGetLastError());
  } else if ((r = diis(m, iscf))) {
    return r;
  }
  MCK(cudaMemcpyAsync(m->old, m->out, bytes, cudaMemcpyDeviceToDevice, m->st));
  MCK(cudaMemcpyAsync(rho, m->out, bytes, cudaMemcpyDefault, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return SDFT_OK;
}

extern "C" int sdft_mixer_state(const sdft_mixer *m, int *iscf, int *num_diis_now, double *coef) {
  if (!m) return set_error(SDFT_ERR_ARG, "mixer_state: null");
  if (iscf) *iscf = m->iscf;
  if (num_diis_now) *num_diis_now = m->num_diis_now;
  if (coef)
    for (size_t i = 0; i < m->coef.size(); i++) coef[i] = m->coef[i];
  return SDFT_OK;
}

extern "C" int sdft_mixer_write_checkpoint(sdft_mixer *m, const char *path, const double *rho, double vol) {
  if (!m || !path || !rho || m->iscf < 0) return set_error(SDFT_ERR_ARG, "write_checkpoint: no mixer step yet");
  cudaSetDevice(m->device);
  const int nd = m->num_diis_now;
  const int nout = nd < m->num_diis ? nd + 1 : nd;
  std::vector<double> h((size_t)m->n);
  FILE *f = fopen(path, "w");
  if (!f) return set_error(SDFT_ERR_ARG, "write_checkpoint: cannot open file");
  std::vector<char> iobuf(1 << 22);
  setvbuf(f, iobuf.data(), _IOFBF, iobuf.size());
  int r = fprintf(f, "%i %i\n", m->iscf, nd) < 0 ? set_error(SDFT_ERR_ARG, "write_checkpoint: write failed") : 0;
  if (!r && !copy_sync(m, h.data(), rho, cudaMemcpyDefault))
    r = set_error(SDFT_ERR_CUDA, "write_checkpoint: copy");
  if (!r) r = write_vec(f, h.data(), m->n, vol, true);
  for (int k = 0; !r && k < nout + nd; k++) {
    const double *src = k < nout ? m->bank[k] : m->err[k - nout];
    if (!src) { r = set_error(SDFT_ERR_STATE, "write_checkpoint: bank entry missing"); break; }
    if (!copy_sync(m, h.data(), src, cudaMemcpyDeviceToHost))
      r = set_error(SDFT_ERR_CUDA, "write_checkpoint: copy");
    else
      r = write_vec(f, h.data(), m->n, 1.0, false);
  }
  if (fclose(f) != 0 && !r) r = set_error(SDFT_ERR_ARG, "write_checkpoint: close failed");
  return r;
}

extern "C" int sdft_mixer_read_checkpoint(sdft_mixer *m, const char *path, double *rho) {
  if (!m || !path || !rho) return set_error(SDFT_ERR_ARG, "read_checkpoint: bad argument");
  cudaSetDevice(m->device);
  FILE *f = fopen(path, "r");
  if (!f) return set_error(SDFT_ERR_ARG, "read_checkpoint: cannot open file");
  std::vector<char> iobuf(1 << 22);
  setvbuf(f, iobuf.data(), _IOFBF, iobuf.size());
  int iscf = 0, nd = 0, r = SDFT_OK;
  if (fscanf(f, "%i %i", &iscf, &nd) != 2 || iscf < 0 || nd < 0 || nd > m->num_diis)
    r = set_error(SDFT_ERR_ARG, "read_checkpoint: bad header");
  std::vector<double> h((size_t)m->n);
  if (!r) r = read_vec(f, h.data(), m->n);
  if (!r && !copy_sync(m, rho, h.data(), cudaMemcpyDefault))
    r = set_error(SDFT_ERR_CUDA, "read_checkpoint: copy");
  if (!r && !copy_sync(m, m->old, h.data(), cudaMemcpyHostToDevice))
    r = set_error(SDFT_ERR_CUDA, "read_checkpoint: copy");
  const int nout = nd < m->num_diis ? nd + 1 : nd;
  for (int k = 0; !r && k < nout + nd; k++) {
    double **slot = k < nout ? &m->bank[k] : &m->err[k - nout];
    if (!*slot && (r = alloc_vec(m, slot))) break;
    if ((r = read_vec(f, h.data(), m->n))) break;
    if (!copy_sync(m, *slot, h.data(), cudaMemcpyHostToDevice))
      r = set_error(SDFT_ERR_CUDA, "read_checkpoint: copy");
  }
  fclose(f);
  if (r) return r;
  m->iscf = iscf;
  m->num_diis_now = nd;
  return SDFT_OK;
}
