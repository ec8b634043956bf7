/* oracle/shims/fftw3.h -- the subset of the FFTW3 API the reference calls
 * (fftw_plan_dft_1d/2d, fftw_execute, fftw_destroy_plan, fftw_malloc, fftw_free),
 * implemented in fftw_shim.c on oracle/fft_d.c.  Test infrastructure only. */
#ifndef SWD_SHIM_FFTW3_H
#define SWD_SHIM_FFTW3_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct swd_fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
#ifdef __cplusplus
}
#endif
#endif
