// sdft_kernels2.cuh -- fast-path (compile-time edge) stage launches.
// Supported: every edge in {24, 48, 72, 96}, planes (n1,n2) in
// {24,48,72}^2 or (96,96).  Launchers return false if the size is not
// instantiated; the context then uses the generic kernels.
#pragma once
#include "sdft_kernels.cuh"

namespace sdft {
bool fast_supported(int n1, int n2, int n3);
// twiddle tables of the compile-time FFT edges in constant memory, once per
// device (call with the device current); nonzero on failure
int init_const_twiddles();
template <typename T>
bool fast_stage_a(const DevGeom &g, const double *C, int nstate, int pair0, int npairs, void *X, cudaStream_t st);
template <typename T>
bool fast_stage_b(const DevGeom &g, void *X, const T *Vp, int npairs, cudaStream_t st);
template <typename T>
bool fast_stage_c(const DevGeom &g, const void *X, const EpiArgs &e, int npairs, cudaStream_t st);
template <typename T>
bool fast_stage_b_density(const DevGeom &g, const void *X, int npairs, double *rho_pair, cudaStream_t st);
template <typename T>
bool fast_stage_b_noise(const DevGeom &g, const unsigned char *neg, int nstate, int pair0, int npairs, void *X,
                        cudaStream_t st);
template <typename T>
bool fast_vks_perm(const DevGeom &g, const double *v, T *Vp, cudaStream_t st);
}  // namespace sdft
