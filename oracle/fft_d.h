/* oracle/fft_d.h -- double FFT for the oracle and the FFTW-API shim (test infrastructure). */
#ifndef SWD_ORACLE_FFT_D_H
#define SWD_ORACLE_FFT_D_H
#ifdef __cplusplus
extern "C" {
#endif
void orc_fft(int n, double *x, int sign);
void orc_fft_strided(int n, double *x, int stride, int sign, double *scratch);
void orc_fft2(int n0, int n1, double *x, int sign);
#ifdef __cplusplus
}
#endif
#endif
