/* omp.h -- project-written single-thread stand-in for the OpenMP runtime
 * calls made by the reference's sources (pragmas are ignored without
 * -fopenmp).  Implementations in oracle/ref_harness.c. */
#ifndef SDFT_REF_OMP_STUB_H
#define SDFT_REF_OMP_STUB_H
double omp_get_wtime(void);
void omp_set_num_threads(int n);
int omp_get_thread_num(void);
int omp_get_num_threads(void);
int omp_get_max_threads(void);
#endif
