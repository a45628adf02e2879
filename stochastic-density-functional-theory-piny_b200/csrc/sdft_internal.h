// sdft_internal.h -- shared declarations of the B200 filter-path library.
#pragma once
#include <cstddef>
#include <cstdint>
#include "../../include/sdft_b200.h"

namespace sdft {

int set_error(int code, const char *msg);

// Stream-ordered device memory from the library's per-device pool; complete
// (usable from any stream) on return.  dev_free releases in stream order.
int dev_alloc(int device, void *stream, void **p, size_t bytes);
void dev_free(void *p, void *stream);

// host helpers (sdft_host.cpp)
void invert_cell(const double *h, double *hi);
double cell_volume(const double *h);
double ran_uniform(double *qseed);
void gaussran2(int nran, double *qseed, double *gauss);
void noise_rank_seeds(double seed, int np_states, double *out);
void gauss_signs(long long nran, double *qseed, unsigned char *neg);
// DURAND state q on the lattice q = Q/128 (Q integer, 1 <= q <= 2147483646):
// from there the FP64 generator follows Q <- 16807 Q mod 128 (2^31 - 1)
// exactly until a draw finds q outside [1, 2147483646].
bool durand_on_lattice(double q);
// gauss_signs pairs p, p+1, ... (two draws each) from *qseed until the state
// is on the lattice or pend is reached; bytes of pair i go to
// out[2 (i - p)], out[2 (i - p) + 1] (the second only below nran).  Returns
// the first pair not generated.
long long gauss_signs_to_lattice(long long nran, long long p, long long pend, double *qseed, unsigned char *out);
// Signs of one pair (r != 1) from its phi, as gauss_signs decides them.
void gauss_signs_from_phi(double phi, unsigned char *b);
int cheby_coeff(int L, int ngrid, double energy_diff, double energy_mean, double beta,
                double chem_pot, int fun_flag, double *coeffs);

// Largest supported FFT edge; every edge must be 2^a 3^b.
constexpr int kMaxEdge = 128;

// Column decomposition of the G sphere (see sdft_api.cu).  Columns are the
// (ka,kb) lines of the full sphere {G} U {-G}; they are stored as mirror
// pairs (ka,kb),(-ka,-kb) followed by the single (0,0) column.
struct SphereCols {
  int ncols = 0;       // 2*(ncp-1)+1
  int ncp = 0;         // column pairs (the last one is the (0,0) column)
  int ncols_pad = 0;   // row pitch of the column scratch
  int kamax = 0;       // max |ka| over columns
};

}  // namespace sdft
