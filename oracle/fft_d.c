/*
 * oracle/fft_d.c -- double-precision complex FFT of any length, test infrastructure only.
 *
 * This is the FFT used by the CPU oracle (oracle/swd_oracle.c) and by the FFTW-API shim
 * (oracle/shims/fftw_shim.c) that lets the reference's kk_decon_interp_psf_minewindow.cpp
 * build without FFTW3.  It is never linked into the product library.
 *
 * Convention (same as FFTW3's documented one, which the reference relies on at
 * kkdecon_acoustic/kk_decon_interp_psf_minewindow.cpp:490-493 and
 * forward/acoustic_hilbert_fftkz_HLForLc.cu:1291,1308 via cuFFT):
 *   sign = -1 : X[k] = sum_j x[j] exp(-2 pi i j k / n)
 *   sign = +1 : X[k] = sum_j x[j] exp(+2 pi i j k / n)
 * Both directions are unnormalised.  Data are interleaved (re, im) doubles.
 *
 * Algorithm: iterative radix-2 Cooley-Tukey for powers of two; Bluestein's chirp-z
 * algorithm (L. Bluestein, 1970) on a power-of-two convolution for every other n, so
 * prime sizes such as the reference's 101-point decon windows stay O(n log n).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fft_d.h"

static const double TWO_PI = 6.283185307179586476925286766559;

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void fft_pow2(int n, double *x, int sign)
{
    /* bit reversal */
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = x[2 * i], ti = x[2 * i + 1];
            x[2 * i] = x[2 * j]; x[2 * i + 1] = x[2 * j + 1];
            x[2 * j] = tr; x[2 * j + 1] = ti;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1;
        double ang = sign * TWO_PI / len;
        for (int k = 0; k < half; k++) {
            double wr = cos(ang * k), wi = sin(ang * k);
            for (int s = 0; s < n; s += len) {
                double *a = x + 2 * (s + k), *b = x + 2 * (s + k + half);
                double br = b[0] * wr - b[1] * wi;
                double bi = b[0] * wi + b[1] * wr;
                b[0] = a[0] - br; b[1] = a[1] - bi;
                a[0] += br; a[1] += bi;
            }
        }
    }
}

static void fft_bluestein(int n, double *x, int sign)
{
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    double *w = (double *)malloc(sizeof(double) * 2 * n);   /* chirp exp(sign*i*pi*k^2/n) */
    double *a = (double *)calloc((size_t)2 * m, sizeof(double));
    double *b = (double *)calloc((size_t)2 * m, sizeof(double));
    for (int k = 0; k < n; k++) {
        /* k*k mod 2n keeps the angle argument small and exact */
        long long kk = ((long long)k * k) % (2LL * n);
        double ang = sign * TWO_PI * 0.5 * (double)kk / n;
        w[2 * k] = cos(ang); w[2 * k + 1] = sin(ang);
    }
    for (int k = 0; k < n; k++) {   /* a = x * w */
        a[2 * k] = x[2 * k] * w[2 * k] - x[2 * k + 1] * w[2 * k + 1];
        a[2 * k + 1] = x[2 * k] * w[2 * k + 1] + x[2 * k + 1] * w[2 * k];
    }
    b[0] = w[0]; b[1] = -w[1];      /* b = conj(w), wrapped */
    for (int k = 1; k < n; k++) {
        b[2 * k] = w[2 * k]; b[2 * k + 1] = -w[2 * k + 1];
        b[2 * (m - k)] = w[2 * k]; b[2 * (m - k) + 1] = -w[2 * k + 1];
    }
    fft_pow2(m, a, -1);
    fft_pow2(m, b, -1);
    for (int k = 0; k < m; k++) {
        double ar = a[2 * k], ai = a[2 * k + 1];
        a[2 * k] = ar * b[2 * k] - ai * b[2 * k + 1];
        a[2 * k + 1] = ar * b[2 * k + 1] + ai * b[2 * k];
    }
    fft_pow2(m, a, +1);
    double inv = 1.0 / m;
    for (int k = 0; k < n; k++) {
        double cr = a[2 * k] * inv, ci = a[2 * k + 1] * inv;
        x[2 * k] = cr * w[2 * k] - ci * w[2 * k + 1];
        x[2 * k + 1] = cr * w[2 * k + 1] + ci * w[2 * k];
    }
    free(w); free(a); free(b);
}

void orc_fft(int n, double *x, int sign)
{
    if (n <= 1) return;
    if (is_pow2(n)) fft_pow2(n, x, sign);
    else fft_bluestein(n, x, sign);
}

void orc_fft_strided(int n, double *x, int stride, int sign, double *scratch)
{
    for (int i = 0; i < n; i++) {
        scratch[2 * i] = x[2 * (size_t)i * stride];
        scratch[2 * i + 1] = x[2 * (size_t)i * stride + 1];
    }
    orc_fft(n, scratch, sign);
    for (int i = 0; i < n; i++) {
        x[2 * (size_t)i * stride] = scratch[2 * i];
        x[2 * (size_t)i * stride + 1] = scratch[2 * i + 1];
    }
}

/* Row-major n0 x n1 array (element [i0][i1] at i0*n1+i1), the layout of FFTW's
 * fftw_plan_dft_2d(n0, n1, ...). */
void orc_fft2(int n0, int n1, double *x, int sign)
{
    int nmax = n0 > n1 ? n0 : n1;
    double *scratch = (double *)malloc(sizeof(double) * 2 * nmax);
    for (int r = 0; r < n0; r++) orc_fft(n1, x + 2 * (size_t)r * n1, sign);
    for (int c = 0; c < n1; c++) orc_fft_strided(n0, x + 2 * (size_t)c, n1, sign, scratch);
    free(scratch);
}
