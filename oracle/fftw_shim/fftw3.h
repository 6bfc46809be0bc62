/*
 * FFTW-API shim used only by the CPU oracle (test infrastructure).
 *
 * FFTW3 is not installed on the build or GPU hosts, so the reference's
 * sfac.cpp (which includes <fftw3.h>, sfac.hpp:5) is compiled against this
 * header instead.  Only the entry points the reference uses are declared
 * (sfac.hpp:13, sfac.cpp:71-81,125,171-175,392):
 *   fftw_malloc, fftw_free, fftw_plan_dft_r2c_3d, fftw_plan_dft_c2r_3d,
 *   fftw_execute, fftw_destroy_plan, fftw_cleanup, FFTW_PATIENT.
 * Semantics follow FFTW's documented conventions: unnormalised transforms,
 * r2c uses sign -1, c2r uses sign +1, the half-complex last dimension holds
 * n2/2+1 values, and an in-place r2c pads each real row to 2*(n2/2+1).
 * The arithmetic is FP64 (see fftw_shim.c).
 */
#ifndef SPME_ORACLE_FFTW_SHIM_H
#define SPME_ORACLE_FFTW_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct shim_fftw_plan_s *fftw_plan;

/* Planner flags: accepted and ignored (the shim has a single algorithm). */
#define FFTW_MEASURE (0U)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);

/* Shim-only: plain 1D complex FFT (out-of-place, unnormalised).
 * sign = -1 (forward) or +1 (backward).  Used by the oracle's self-tests. */
void shim_fft1d(int n, const double *in, double *out, int sign);

#ifdef __cplusplus
}
#endif

#endif
