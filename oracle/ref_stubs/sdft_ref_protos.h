/* sdft_ref_protos.h -- prototypes that MKL and OpenMP headers supply in the
 * reference's own build (its sources call these without including them;
 * without a prototype C would assume an int return).  Force-included by
 * oracle/build_ref.sh. */
#ifndef SDFT_REF_PROTOS_H
#define SDFT_REF_PROTOS_H
double ddot_(int *n, double *x, int *incx, double *y, int *incy);
void daxpy_(int *n, double *a, double *x, int *incx, double *y, int *incy);
void mkl_set_dynamic(int);
void mkl_set_num_threads(int);
double omp_get_wtime(void);
void omp_set_num_threads(int);
int omp_get_thread_num(void);
void omp_set_max_active_levels(int);
#endif
