/* oracle/shims/fftw_shim.c -- FFTW3-API plans executed by oracle/fft_d.c (O(n log n) for any n). */
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"
#include "../fft_d.h"
struct swd_fftw_plan_s { int rank, n0, n1, sign; fftw_complex *in, *out; };
static fftw_plan mk(int rank, int n0, int n1, fftw_complex *in, fftw_complex *out, int sign)
{
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->rank = rank; p->n0 = n0; p->n1 = n1; p->sign = sign; p->in = in; p->out = out;
    return p;
}
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{ (void)flags; return mk(1, n, 1, in, out, sign); }
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{ (void)flags; return mk(2, n0, n1, in, out, sign); }
void fftw_execute(const fftw_plan p)
{
    size_t n = (size_t)p->n0 * p->n1;
    if (p->out != p->in) memcpy(p->out, p->in, n * sizeof(fftw_complex));
    if (p->rank == 1) orc_fft(p->n0, (double *)p->out, p->sign);
    else orc_fft2(p->n0, p->n1, (double *)p->out, p->sign);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }
void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }
