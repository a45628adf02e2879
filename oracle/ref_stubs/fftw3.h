/* fftw3.h -- project-written stand-in declaring the FFTW3 subset the
 * reference's hot-path sources call (FFTW itself is not installed here).
 * The implementations live in oracle/ref_harness.c (a plain FP64 DFT). */
#ifndef SDFT_REF_FFTW3_STUB_H
#define SDFT_REF_FFTW3_STUB_H
#include <complex.h>
typedef double _Complex fftw_complex;
typedef struct sdft_fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed, int istride,
                             int idist, fftw_complex *out, const int *onembed, int ostride, int odist, int sign,
                             unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int n);
void fftw_cleanup_threads(void);
#endif
