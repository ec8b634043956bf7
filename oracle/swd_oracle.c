/*
 * oracle/swd_oracle.c -- CPU oracle (TEST INFRASTRUCTURE, never part of the product).
 *
 * Host preparation and the windowed PSF deconvolution are restated here with the
 * reference's own float/double arithmetic; the propagation/imaging loops live in
 * oracle/prop_impl.h and are compiled twice (float and double) at the end of this file.
 * Build with -ffp-contract=off so that float expressions round exactly as written.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "swd_oracle.h"
#include "fft_d.h"

#define ORC_PI 3.1415926   /* the reference's PI macro (acoustic_HLVSPRTMC.cpp:7) */

/* Staggered-grid Taylor coefficients of order 2*Lc.  acoustic_HLVSPRTMC.cpp:1858-1878. */
void orc_cal_xishu(int Lx, float *rx)
{
    int m, i;
    float s1, s2;
    for (m = 1; m <= Lx; m++) {
        s1 = 1.0; s2 = 1.0;
        for (i = 1; i < m; i++) {
            s1 = s1 * (2.0 * i - 1) * (2.0 * i - 1);
            s2 = s2 * ((2.0 * m - 1) * (2.0 * m - 1) - (2.0 * i - 1) * (2.0 * i - 1));
        }
        for (i = m + 1; i <= Lx; i++) {
            s1 = s1 * (2.0 * i - 1) * (2.0 * i - 1);
            s2 = s2 * ((2.0 * m - 1) * (2.0 * m - 1) - (2.0 * i - 1) * (2.0 * i - 1));
        }
        s2 = fabsf(s2);
        rx[m - 1] = pow(-1.0, m + 1) * s1 / (s2 * (2.0 * m - 1));
    }
}

/* CPML a/b profiles at integer and half nodes.  acoustic_HLVSPRTMC.cpp:891-1129 (`pml`
 * there is the padded width pmlc, passed at :467).  Vpmax=5500, Rc=1e-5, N=2,
 * alpha_max=15*pi and kappa=1 are the reference's hard-coded constants; the layer
 * thickness uses dz for both axes (:925). */
void orc_cpml(int ntx, int ntz, int pml, float dx, float dz, float dt,
              float *a_x, float *a_x_half, float *a_z, float *a_z_half,
              float *b_x, float *b_x_half, float *b_z, float *b_z_half)
{
    int N = 2;
    int iz, ix;
    float thickness_of_pml;
    float Rc = 1.0e-5;
    float d0;
    float pi = 3.1415927;
    float alpha_max = pi * 15;
    float Vpmax;
    float x_start, x_end, delta_x;
    float z_start, z_end, delta_z;
    float x_current, z_current;
    float *d_x = (float *)malloc(sizeof(float) * ntx), *d_x_half = (float *)malloc(sizeof(float) * ntx);
    float *d_z = (float *)malloc(sizeof(float) * ntz), *d_z_half = (float *)malloc(sizeof(float) * ntz);
    float *k_x = (float *)malloc(sizeof(float) * ntx), *k_x_half = (float *)malloc(sizeof(float) * ntx);
    float *k_z = (float *)malloc(sizeof(float) * ntz), *k_z_half = (float *)malloc(sizeof(float) * ntz);
    float *alpha_x = (float *)malloc(sizeof(float) * ntx), *alpha_x_half = (float *)malloc(sizeof(float) * ntx);
    float *alpha_z = (float *)malloc(sizeof(float) * ntz), *alpha_z_half = (float *)malloc(sizeof(float) * ntz);

    Vpmax = 5500;
    thickness_of_pml = pml * dz;
    /* the reference is C++: log/exp of a float argument resolve to the float overloads */
    d0 = -(N + 1) * Vpmax * logf(Rc) / (2.0 * thickness_of_pml);

    for (ix = 0; ix < ntx; ix++) {
        a_x[ix] = 0.0; a_x_half[ix] = 0.0; b_x[ix] = 0.0; b_x_half[ix] = 0.0;
        d_x[ix] = 0.0; d_x_half[ix] = 0.0; k_x[ix] = 1.0; k_x_half[ix] = 1.0;
        alpha_x[ix] = 0.0; alpha_x_half[ix] = 0.0;
    }
    for (iz = 0; iz < ntz; iz++) {
        a_z[iz] = 0.0; a_z_half[iz] = 0.0; b_z[iz] = 0.0; b_z_half[iz] = 0.0;
        d_z[iz] = 0.0; d_z_half[iz] = 0.0; k_z[iz] = 1.0; k_z_half[iz] = 1.0;
        alpha_z[iz] = 0.0; alpha_z_half[iz] = 0.0;
    }

    x_start = pml * dx;
    x_end = (ntx - pml - 1) * dx;
    for (ix = 0; ix < ntx; ix++) {
        x_current = ix * dx;
        if (x_current <= x_start) {
            delta_x = x_start - x_current;
            d_x[ix] = d0 * pow(delta_x / thickness_of_pml, 2);
            k_x[ix] = 1.0;
            alpha_x[ix] = alpha_max * (1.0 - (delta_x / thickness_of_pml)) + 0.1 * alpha_max;
        }
        if (x_current >= x_end) {
            delta_x = x_current - x_end;
            d_x[ix] = d0 * pow(delta_x / thickness_of_pml, 2);
            k_x[ix] = 1.0;
            alpha_x[ix] = alpha_max * (1.0 - (delta_x / thickness_of_pml)) + 0.1 * alpha_max;
        }
    }
    for (ix = 0; ix < ntx; ix++) {
        x_current = (ix + 0.5) * dx;
        if (x_current <= x_start) {
            delta_x = x_start - x_current;
            d_x_half[ix] = d0 * pow(delta_x / thickness_of_pml, 2);
            k_x_half[ix] = 1.0;
            alpha_x_half[ix] = alpha_max * (1.0 - (delta_x / thickness_of_pml)) + 0.1 * alpha_max;
        }
        if (x_current >= x_end) {
            delta_x = x_current - x_end;
            d_x_half[ix] = d0 * pow(delta_x / thickness_of_pml, 2);
            k_x_half[ix] = 1.0;
            alpha_x_half[ix] = alpha_max * (1.0 - (delta_x / thickness_of_pml)) + 0.1 * alpha_max;
        }
    }
    for (ix = 0; ix < ntx; ix++) {
        if (alpha_x[ix] < 0.0) alpha_x[ix] = 0.0;
        if (alpha_x_half[ix] < 0.0) alpha_x_half[ix] = 0.0;
        b_x[ix] = expf(-(d_x[ix] / k_x[ix] + alpha_x[ix]) * dt);
        if (d_x[ix] > 1.0e-6)
            a_x[ix] = d_x[ix] / (k_x[ix] * (d_x[ix] + k_x[ix] * alpha_x[ix])) * (b_x[ix] - 1.0);
        b_x_half[ix] = expf(-(d_x_half[ix] / k_x_half[ix] + alpha_x_half[ix]) * dt);
        if (d_x_half[ix] > 1.0e-6)
            a_x_half[ix] = d_x_half[ix] / (k_x_half[ix] * (d_x_half[ix] + k_x_half[ix] * alpha_x_half[ix])) * (b_x_half[ix] - 1.0);
    }

    z_start = pml * dz;
    z_end = (ntz - pml - 1) * dz;
    for (iz = 0; iz < ntz; iz++) {
        z_current = iz * dz;
        if (z_current <= z_start) {
            delta_z = z_start - z_current;
            d_z[iz] = d0 * pow(delta_z / thickness_of_pml, 2);
            k_z[iz] = 1.0;
            alpha_z[iz] = alpha_max * (1.0 - (delta_z / thickness_of_pml)) + 0.1 * alpha_max;
        }
        if (z_current >= z_end) {
            delta_z = z_current - z_end;
            d_z[iz] = d0 * pow(delta_z / thickness_of_pml, 2);
            k_z[iz] = 1.0;
            alpha_z[iz] = alpha_max * (1.0 - (delta_z / thickness_of_pml)) + 0.1 * alpha_max;
        }
    }
    for (iz = 0; iz < ntz; iz++) {
        z_current = (iz + 0.5) * dz;
        if (z_current <= z_start) {
            delta_z = z_start - z_current;
            d_z_half[iz] = d0 * pow(delta_z / thickness_of_pml, 2);
            k_z_half[iz] = 1.0;
            alpha_z_half[iz] = alpha_max * (1.0 - (delta_z / thickness_of_pml)) + 0.1 * alpha_max;
        }
        if (z_current >= z_end) {
            delta_z = z_current - z_end;
            d_z_half[iz] = d0 * pow(delta_z / thickness_of_pml, 2);
            k_z_half[iz] = 1.0;
            alpha_z_half[iz] = alpha_max * (1.0 - (delta_z / thickness_of_pml)) + 0.1 * alpha_max;
        }
    }
    for (iz = 0; iz < ntz; iz++) {
        if (alpha_z[iz] < 0.0) alpha_z[iz] = 0.0;
        if (alpha_z_half[iz] < 0.0) alpha_z_half[iz] = 0.0;
        b_z[iz] = expf(-(d_z[iz] / k_z[iz] + alpha_z[iz]) * dt);
        if (d_z[iz] > 1.0e-6)
            a_z[iz] = d_z[iz] / (k_z[iz] * (d_z[iz] + k_z[iz] * alpha_z[iz])) * (b_z[iz] - 1.0);
        b_z_half[iz] = expf(-(d_z_half[iz] / k_z_half[iz] + alpha_z_half[iz]) * dt);
        if (d_z_half[iz] > 1.0e-6)
            a_z_half[iz] = d_z_half[iz] / (k_z_half[iz] * (d_z_half[iz] + k_z_half[iz] * alpha_z_half[iz])) * (b_z_half[iz] - 1.0);
    }
    free(d_x); free(d_x_half); free(d_z); free(d_z_half);
    free(k_x); free(k_x_half); free(k_z); free(k_z_half);
    free(alpha_x); free(alpha_x_half); free(alpha_z); free(alpha_z_half);
}

/* Ricker wavelet, flag 2, t0 = 1/f0.  acoustic_HLVSPRTMC.cpp:1249-1299 (called at :359
 * with t0 = 1.0/f0 from :96). */
void orc_ricker2(int itmax, float f0, float dt, float *rick)
{
    float pi = 3.1415927;
    float t0 = 1.0 / f0;
    float temp;
    for (int it = 0; it < itmax; it++) {
        temp = pi * f0 * (it * dt - t0);
        temp = temp * temp;
        rick[it] = (1.0 - 2.0 * temp) * expf(-temp);   /* C++ float overload */
    }
}

/* Read-in interior + edge replication into the padded frame.
 * get_acc_model, acoustic_HLVSPRTMC.cpp:1136-1196 (`pml` there is pmlc, :376). */
void orc_pad_model(int nx, int nz, int pml, const float *v_in, float *vp)
{
    int ntx = nx + 2 * pml, ntz = nz + 2 * pml;
    int ip, ipp, ix, iz, k = 0;
    for (ix = pml; ix < ntx - pml; ix++)
        for (iz = pml; iz < ntz - pml; iz++) vp[ix * ntz + iz] = v_in[k++];
    for (iz = pml; iz <= ntz - pml - 1; iz++) {
        for (ix = 0; ix <= pml - 1; ix++) { ip = ix * ntz + iz; ipp = pml * ntz + iz; vp[ip] = vp[ipp]; }
        for (ix = ntx - pml; ix < ntx; ix++) { ip = ix * ntz + iz; ipp = (ntx - pml - 1) * ntz + iz; vp[ip] = vp[ipp]; }
    }
    for (ix = 0; ix < ntx; ix++) {
        for (iz = 0; iz <= pml - 1; iz++) { ip = ix * ntz + iz; ipp = ix * ntz + pml; vp[ip] = vp[ipp]; }
        for (iz = ntz - pml; iz < ntz; iz++) { ip = ix * ntz + iz; ipp = ix * ntz + (ntz - pml - 1); vp[ip] = vp[ipp]; }
    }
}

static void model_in_pml(float *vp, int ntz, int ntx, int pml)
{
    /* acoustic_HLVSPRTMC.cpp:1428-1468 */
    int iz, ix, ip, ipp;
    for (iz = pml; iz <= ntz - pml - 1; iz++) {
        for (ix = 0; ix <= pml - 1; ix++) { ip = ix * ntz + iz; ipp = pml * ntz + iz; vp[ip] = vp[ipp]; }
        for (ix = ntx - pml; ix < ntx; ix++) { ip = ix * ntz + iz; ipp = (ntx - pml - 1) * ntz + iz; vp[ip] = vp[ipp]; }
    }
    for (ix = 0; ix < ntx; ix++) {
        for (iz = 0; iz <= pml - 1; iz++) { ip = ix * ntz + iz; ipp = ix * ntz + pml; vp[ip] = vp[ipp]; }
        for (iz = ntz - pml; iz < ntz; iz++) { ip = ix * ntz + iz; ipp = ix * ntz + (ntz - pml - 1); vp[ip] = vp[ipp]; }
    }
}

/* Gaussian (2w+1)^2 smoothing with double accumulation and clamped indices; rows
 * iz < pml+8 keep the original value.  ini_model_mine, acoustic_HLVSPRTMC.cpp:1473-1569. */
void orc_smooth(int ntx, int ntz, int pml, int window, float *vp)
{
    int windxz = 2 * window + 1;
    double sigma = window / 2.0;
    int ntp = ntx * ntz;
    double sum;
    double *coef = (double *)malloc(sizeof(double) * windxz * windxz);
    double *vp_old1 = (double *)malloc(sizeof(double) * ntp);
    sum = 0.0;
    for (int ix = 0; ix < windxz; ix++)
        for (int iz = 0; iz < windxz; iz++) {
            int ip = ix * windxz + iz;
            coef[ip] = 1.0 / (2.0 * ORC_PI * sigma * sigma) *
                       exp(-((ix - window) * (ix - window) + (iz - window) * (iz - window)) / (2.0 * sigma * sigma));
            sum += coef[ip];
        }
    for (int ip = 0; ip < windxz * windxz; ip++) coef[ip] /= sum;
    for (int ip = 0; ip < ntp; ip++) vp_old1[ip] = vp[ip];
#pragma omp parallel for schedule(static)
    for (int iz = pml; iz <= ntz - pml - 1; iz++) {
        for (int ix = pml; ix <= ntx - pml - 1; ix++) {
            double s = 0.0;
            for (int izw = iz - window; izw <= iz + window; izw++) {
                for (int ixw = ix - window; ixw <= ix + window; ixw++) {
                    int ipp = (izw - iz + window) * windxz + (ixw - ix + window);
                    int iz1 = izw < 0 ? 0 : (izw > ntz - 1 ? ntz - 1 : izw);
                    int ix1 = ixw < 0 ? 0 : (ixw > ntx - 1 ? ntx - 1 : ixw);
                    s += vp_old1[ix1 * ntz + iz1] * coef[ipp];
                }
            }
            int ip = ix * ntz + iz;
            vp[ip] = s;
            if (iz < pml + 8) vp[ip] = vp_old1[ip];
        }
    }
    model_in_pml(vp, ntz, ntx, pml);
    free(coef);
    free(vp_old1);
}

/* nfftz / NZ rule: (int)pow(2, (int)ceil(log(1.0*n)/log(2.0))).
 * forward/acoustic_hilbert_fftkz_HLForC.cpp:299-300, forward/...HLForLc.cu:1263-1264. */
int orc_pow2_len(int n)
{
    int K = (int)ceil(log(1.0 * n) / log(2.0));
    return (int)pow(2.0, K);
}

/* Cosine kz taper near kz=0 for the up/down split.  forward/...HLForC.cpp:354-377.
 * Returns layerz, or -1 when the reference would abort (layerz > nfftz/6). */
int orc_kz_taper(int nfftz, float dz, float *coef)
{
    float dkz = 1.0 / (nfftz * dz);
    float kcut = 1.0 / 15.0 / dz;
    int layerz = kcut / dkz;
    if (layerz > nfftz / 6) return -1;
    int upz = layerz, downz = nfftz - layerz;
    for (int iz = 0; iz < nfftz; iz++) {
        if (iz <= upz) coef[iz] = 0.5000 - 0.5 * cos(ORC_PI * iz / layerz);
        if (iz > upz && iz < downz) coef[iz] = 1.0;
        if (iz >= downz) coef[iz] = 0.5000 + 0.5 * cos(ORC_PI * (iz - downz) / layerz);
    }
    return layerz;
}

/* Time-Hilbert transform of the wavelet: zero-pad to NZ, -i on bins [1,NZ/2), +i on
 * [NZ/2,NZ), bin 0 zeroed, inverse, /NZ.  forward/...HLForLc.cu:1257-1324 (cuFFT there,
 * double FFT here). */
void orc_hilbert1d(int itmax, const float *rick, float *rick_hilbert)
{
    int NZ = orc_pow2_len(itmax);
    double *f = (double *)calloc((size_t)2 * NZ, sizeof(double));
    double *h = (double *)calloc((size_t)2 * NZ, sizeof(double));
    for (int it = 0; it < itmax; it++) f[2 * it] = rick[it];
    orc_fft(NZ, f, -1);
    for (int it = 1; it < NZ / 2; it++) { h[2 * it] = f[2 * it + 1]; h[2 * it + 1] = -f[2 * it]; }
    for (int it = NZ / 2; it < NZ; it++) { h[2 * it] = -f[2 * it + 1]; h[2 * it + 1] = f[2 * it]; }
    orc_fft(NZ, h, +1);
    for (int it = 0; it < itmax; it++) rick_hilbert[it] = (float)(h[2 * it] / NZ);
    free(f);
    free(h);
}

/* Receiver count and depths of the two edge wells (left well ix=pmlc, right well
 * ix=ntx-pmlc-1; the reference records there, not at r_ix).
 * acoustic_HLVSPRTMC.cpp:153-200 with the recording columns of acoustic_HLVSPRTMLc.cu:180-197. */
int orc_well_count(int nz, int pmlc, float dz, float shotdep, float offsetz)
{
    int s_iz = pmlc + (int)(shotdep / dz), i = 0;
    for (int iz = 0; iz < nz; iz++)
        if (fabs((double)(s_iz - iz - pmlc)) * dz <= offsetz) i++;
    return 2 * i;
}

void orc_well_geometry(int nx, int nz, int pmlc, float dz, float shotdep, float offsetz,
                       int *r_ix, int *r_iz)
{
    int ntx = nx + 2 * pmlc;
    int r_n = orc_well_count(nz, pmlc, dz, shotdep, offsetz);
    int s_iz = pmlc + (int)(shotdep / dz), i = 0;
    for (int iz = 0; iz < nz; iz++) {
        if (fabs((double)(s_iz - iz - pmlc)) * dz <= offsetz) {
            r_iz[i] = pmlc + iz; r_ix[i] = pmlc;
            r_iz[i + r_n / 2] = pmlc + iz; r_ix[i + r_n / 2] = ntx - pmlc - 1;
            i++;
        }
    }
}

int orc_strip_len(const orc_model *m)
{
    int nx = m->ntx - 2 * m->pmlc, nz = m->ntz - 2 * m->pmlc;
    return 2 * m->Lc * nx + 2 * m->Lc * (nz - 2 * m->Lc);
}

/* Stacked-image edge zeroing.  acoustic_HLVSPRTMC.cpp:754-768. */
void orc_edge_zero(int nx, int nz, int Lc, float *img)
{
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++)
            if (ix <= 3 || ix >= nx - Lc || iz < 7 || iz >= nz - Lc) img[ix * nz + iz] = 0.0;
}

/* ------------------------------------------------------------------------------------
 * Windowed wavenumber PSF deconvolution.
 * kkdecon_acoustic/kk_decon_interp_psf_minewindow.cpp: geometry :84-124, expansion
 * :303-339, taper :355-383, window loop :543-674, outputs :692-731.
 * ---------------------------------------------------------------------------------- */
typedef struct {
    int halfpsfwx, halfpsfwz, halfltwx, halfltwz, nzwpsf, nxwpsf;
    int fullwx, fullwz, FX, FZ, n0, n1, midpx, midpz;
    int outwinx, outwinz, halfoutwx, halfoutwz, stepwinx, stepwinz;
    int stepnumx, stepnumz, totalnum, nxp, nzp, ocx, ocz;
} decon_geom;

static int decon_geom_fill(const orc_decon_params *p, decon_geom *g)
{
    if (p->psfwinx % 2 == 0 || p->psfwinz % 2 == 0 || p->filterwinx % 2 == 0 || p->filterwinz % 2 == 0)
        return -1;
    g->halfpsfwx = p->psfwinx / 2; g->halfpsfwz = p->psfwinz / 2;
    g->halfltwx = p->filterwinx / 2; g->halfltwz = p->filterwinz / 2;
    g->nzwpsf = (int)ceil(1.0 * p->nz / p->psfwinz);
    g->nxwpsf = (int)ceil(1.0 * p->nx / p->psfwinx);
    g->fullwx = p->filterwinx + p->psfwinx - 1;
    g->fullwz = p->filterwinz + p->psfwinz - 1;
    if (p->fft_n0 > 0 && p->fft_n1 > 0) {
        /* project option: zero-padded FFT of FX x FZ, a true 2D DFT over (x, z) */
        g->FX = p->fft_n0; g->FZ = p->fft_n1;
        if (g->FX < g->fullwx || g->FZ < g->fullwz) return -2;
        g->n0 = g->FX; g->n1 = g->FZ;
    } else {
        /* reference: buffer indexed ixx*fullwz+izz, planned as fftw_plan_dft_2d(fullwz, fullwx) */
        g->FX = g->fullwx; g->FZ = g->fullwz;
        g->n0 = g->fullwz; g->n1 = g->fullwx;
    }
    g->midpx = g->FX / 2; g->midpz = g->FZ / 2;
    g->outwinx = 2 * (p->psfwinx / 10) + 2 * p->snapwinx + 1;
    g->outwinz = 2 * (p->psfwinz / 10) + 2 * p->snapwinz + 1;
    g->halfoutwx = g->outwinx / 2; g->halfoutwz = g->outwinz / 2;
    g->stepwinx = g->outwinx - p->snapwinx; g->stepwinz = g->outwinz - p->snapwinz;
    g->stepnumx = (int)ceil(1.0 * (p->nx + g->fullwx) / g->stepwinx) + 1;
    g->stepnumz = (int)ceil(1.0 * (p->nz + g->fullwz) / g->stepwinz) + 1;
    g->totalnum = g->stepnumx * g->stepnumz;
    g->nxp = g->stepnumx * g->stepwinx; g->nzp = g->stepnumz * g->stepwinz;
    /* deconvolved-patch centre inside the FFT buffer: midp - halfpsfw (== halfltw for the
       reference size, which is the offset the reference uses at :659) */
    g->ocx = g->midpx - g->halfpsfwx; g->ocz = g->midpz - g->halfpsfwz;
    if (p->filterwinx < p->psfwinx || p->filterwinz < p->psfwinz) return -3;
    if (p->filterwinx < g->outwinx || p->filterwinz < g->outwinz) return -4;
    return 0;
}

int orc_decon_geometry(const orc_decon_params *p, int *out)
{
    decon_geom g;
    int rc = decon_geom_fill(p, &g);
    if (rc) return rc;
    int v[16] = {g.fullwx, g.fullwz, g.FX, g.FZ, g.outwinx, g.outwinz, g.stepwinx, g.stepwinz,
                 g.stepnumx, g.stepnumz, g.totalnum, g.nxp, g.nzp, g.nxwpsf, g.nzwpsf, g.n0};
    memcpy(out, v, sizeof(v));
    return 0;
}

/* Bracketing lattice points of a window-centre coordinate for PSF interpolation (project
 * option): f0 = floor((c - h)/w) and f1 = f0 + 1 clamped to [3, n - 4] (the reference's
 * range), t the fractional position between them in [0, 1] (0 when they coincide). */
static void orc_psf_bracket(int c, int h, int w, int n, int *f0, int *f1, double *t)
{
    const double pos = (double)(c - h) / (double)w;
    int a = (int)floor(pos);
    if (a < 3) a = 3;
    if (a > n - 4) a = n - 4;
    int b = a + 1 > n - 4 ? n - 4 : a + 1;
    double u = pos - (double)a;
    if (u < 0.0) u = 0.0;
    if (u > 1.0) u = 1.0;
    if (b == a) u = 0.0;
    *f0 = a;
    *f1 = b;
    *t = u;
}

int orc_decon(const orc_decon_params *p, const float *migreal, const float *migpsf,
              float *out_dec, float *out_coef, int nthreads)
{
    decon_geom g;
    int rc = decon_geom_fill(p, &g);
    if (rc) return rc;
    const int nx = p->nx, nz = p->nz, nxp = g.nxp, nzp = g.nzp;
    const size_t npf = (size_t)nxp * nzp, nbuf = (size_t)g.FX * g.FZ;
    float *migrealf = (float *)malloc(sizeof(float) * npf);
    float *migpsff = (float *)malloc(sizeof(float) * npf);
    float *coefr = (float *)malloc(sizeof(float) * g.outwinx * g.outwinz);
    float *mig_dec = (float *)calloc(npf, sizeof(float));
    float *mig_coef = (float *)calloc(npf, sizeof(float));
    /* expansion by edge replication (:303-339) */
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            migrealf[ix * nzp + iz] = migreal[ix * nz + iz];
            migpsff[ix * nzp + iz] = migpsf[ix * nz + iz];
        }
    for (int ix = nx; ix < nxp; ix++)
        for (int iz = 0; iz < nz; iz++) {
            migrealf[ix * nzp + iz] = migrealf[(nx - 1) * nzp + iz];
            migpsff[ix * nzp + iz] = migpsff[(nx - 1) * nzp + iz];
        }
    for (int iz = nz; iz < nzp; iz++)
        for (int ix = 0; ix < nxp; ix++) {
            migrealf[ix * nzp + iz] = migrealf[ix * nzp + nz - 1];
            migpsff[ix * nzp + iz] = migpsff[ix * nzp + nz - 1];
        }
    /* Hann-edged output taper (:355-383) */
    for (int ix = 0; ix < g.outwinx; ix++)
        for (int iz = 0; iz < g.outwinz; iz++) {
            float coefx, coefz;
            if (ix <= p->snapwinx - 1) coefx = 0.5000 - 0.5 * cos(ORC_PI * ix / (p->snapwinx - 1));
            else if (ix >= g.outwinx - p->snapwinx) coefx = 0.5000 + 0.5 * cos(ORC_PI * (ix - g.outwinx + p->snapwinx) / (p->snapwinx - 1));
            else coefx = 1.0;
            if (iz <= p->snapwinz - 1) coefz = 0.5000 - 0.5 * cos(ORC_PI * iz / (p->snapwinz - 1));
            else if (iz >= g.outwinz - p->snapwinz) coefz = 0.5000 + 0.5 * cos(ORC_PI * (iz - g.outwinz + p->snapwinz) / (p->snapwinz - 1));
            else coefz = 1.0;
            coefr[ix * g.outwinz + iz] = coefx * coefz;
        }
    const int nout = g.outwinx * g.outwinz;
    double *winout = (double *)malloc(sizeof(double) * (size_t)g.totalnum * nout);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel
    {
        double *snapm = (double *)malloc(sizeof(double) * 2 * nbuf);
        double *snapsf = (double *)malloc(sizeof(double) * 2 * nbuf);
        double *decon = (double *)malloc(sizeof(double) * 2 * nbuf);
        /* iterative option: B = M^ conj S^, P = |S^|^2, iterates, and a transform buffer */
        double *itB = NULL, *itP = NULL, *itX = NULL, *itXP = NULL, *itW = NULL;
        if (p->iters > 0) {
            itB = (double *)malloc(sizeof(double) * 2 * nbuf);
            itP = (double *)malloc(sizeof(double) * nbuf);
            itX = (double *)malloc(sizeof(double) * nbuf);
            itXP = (double *)malloc(sizeof(double) * nbuf);
            itW = (double *)malloc(sizeof(double) * 2 * nbuf);
        }
#pragma omp for schedule(dynamic, 4)
        for (int stepindex = 0; stepindex < g.totalnum; stepindex++) {
            int ix = g.stepwinx * (stepindex / g.stepnumz);
            int iz = g.stepwinz * (stepindex % g.stepnumz);
            memset(snapm, 0, sizeof(double) * 2 * nbuf);
            memset(snapsf, 0, sizeof(double) * 2 * nbuf);
            float pp_max = 0.0;
            for (int ixx = 0; ixx < p->filterwinx; ixx++)
                for (int izz = 0; izz < p->filterwinz; izz++) {
                    int iix = ix - g.halfltwx + ixx, iiz = iz - g.halfltwz + izz;
                    int ip = (g.midpx - g.halfltwx + ixx) * g.FZ + g.midpz - g.halfltwz + izz;
                    if (iix >= 0 && iix < nxp && iiz >= 0 && iiz < nzp) {
                        snapm[2 * ip] = migrealf[(size_t)iix * nzp + iiz];
                        pp_max += fabs(snapm[2 * ip]);
                    }
                }
            if (pp_max <= 1.0e-15) pp_max = 1.0e-10;
            for (size_t ip = 0; ip < nbuf; ip++) snapm[2 * ip] /= pp_max;
            orc_fft2(g.n0, g.n1, snapm, -1);

            if (!p->psf_interp) {
                int ixf = (ix - g.halfpsfwx) / p->psfwinx;
                int izf = (iz - g.halfpsfwz) / p->psfwinz;
                if (ixf <= 2) ixf = 3;
                if (ixf >= g.nxwpsf - 3) ixf = g.nxwpsf - 4;
                if (izf <= 2) izf = 3;
                if (izf >= g.nzwpsf - 3) izf = g.nzwpsf - 4;
                int ixp = g.halfpsfwx + ixf * p->psfwinx;
                int izp = g.halfpsfwz + izf * p->psfwinz;
                for (int ixx = 0; ixx < p->psfwinx; ixx++)
                    for (int izz = 0; izz < p->psfwinz; izz++) {
                        int ip = ixx * g.FZ + izz;
                        snapsf[2 * ip] = migpsff[(size_t)(ixp + ixx - g.halfpsfwx) * nzp + (izp + izz - g.halfpsfwz)];
                    }
            } else {
                /* project option: bilinear weights of the two lattice points bracketing the
                 * window centre on each axis, inside the clamped range [3, nwpsf-4] */
                int fx0, fx1, fz0, fz1;
                double tx, tz;
                orc_psf_bracket(ix, g.halfpsfwx, p->psfwinx, g.nxwpsf, &fx0, &fx1, &tx);
                orc_psf_bracket(iz, g.halfpsfwz, p->psfwinz, g.nzwpsf, &fz0, &fz1, &tz);
                const int xa = g.halfpsfwx + fx0 * p->psfwinx - g.halfpsfwx, xb = g.halfpsfwx + fx1 * p->psfwinx - g.halfpsfwx;
                const int za = g.halfpsfwz + fz0 * p->psfwinz - g.halfpsfwz, zb = g.halfpsfwz + fz1 * p->psfwinz - g.halfpsfwz;
                for (int ixx = 0; ixx < p->psfwinx; ixx++)
                    for (int izz = 0; izz < p->psfwinz; izz++) {
                        const double a = migpsff[(size_t)(xa + ixx) * nzp + za + izz];
                        const double b = migpsff[(size_t)(xb + ixx) * nzp + za + izz];
                        const double c = migpsff[(size_t)(xa + ixx) * nzp + zb + izz];
                        const double d = migpsff[(size_t)(xb + ixx) * nzp + zb + izz];
                        snapsf[2 * (ixx * g.FZ + izz)] =
                            (float)((1.0 - tz) * ((1.0 - tx) * a + tx * b) + tz * ((1.0 - tx) * c + tx * d));
                    }
            }
            float psf_max = 0.0;
            for (size_t ip = 0; ip < nbuf; ip++) psf_max += fabs(snapsf[2 * ip]);
            for (size_t ip = 0; ip < nbuf; ip++) snapsf[2 * ip] /= psf_max;
            orc_fft2(g.n0, g.n1, snapsf, -1);

            float fft_max = 0.0, tmpfloat;
            for (size_t ip = 0; ip < nbuf; ip++) {
                tmpfloat = (snapsf[2 * ip] * snapsf[2 * ip] + snapsf[2 * ip + 1] * snapsf[2 * ip + 1]);
                if (fft_max < tmpfloat) fft_max = tmpfloat;
            }
            const double smax2 = fft_max;   /* max |S^|^2 before the damping factor */
            fft_max *= p->epsilon;
            if (fft_max == 0.0) fft_max = 1.0e-15;
            for (size_t ip = 0; ip < nbuf; ip++) {
                tmpfloat = (snapsf[2 * ip] * snapsf[2 * ip] + snapsf[2 * ip + 1] * snapsf[2 * ip + 1]) + fft_max;
                decon[2 * ip] = (snapm[2 * ip] * snapsf[2 * ip] + snapm[2 * ip + 1] * snapsf[2 * ip + 1]) / tmpfloat;
                decon[2 * ip + 1] = (-snapm[2 * ip] * snapsf[2 * ip + 1] + snapm[2 * ip + 1] * snapsf[2 * ip]) / tmpfloat;
            }
            orc_fft2(g.n0, g.n1, decon, +1);
            if (p->iters > 0 && smax2 > 0.0) {
                /* FISTA from x0 = IDFT2(D)/n; gradient IDFT2((P + mu) Y^ - B)/n */
                const double n = (double)nbuf, mu = p->reg_l2 * smax2, tau = 1.0 / (smax2 + mu);
                double xmax = 0.0, t = 1.0;
                for (size_t ip = 0; ip < nbuf; ip++) {
                    itB[2 * ip] = snapm[2 * ip] * snapsf[2 * ip] + snapm[2 * ip + 1] * snapsf[2 * ip + 1];
                    itB[2 * ip + 1] = snapm[2 * ip + 1] * snapsf[2 * ip] - snapm[2 * ip] * snapsf[2 * ip + 1];
                    itP[ip] = snapsf[2 * ip] * snapsf[2 * ip] + snapsf[2 * ip + 1] * snapsf[2 * ip + 1];
                    itX[ip] = itXP[ip] = decon[2 * ip] / n;
                    if (fabs(itX[ip]) > xmax) xmax = fabs(itX[ip]);
                }
                const double thr = p->reg_l1 * xmax;
                for (int k = 0; k < p->iters; k++) {
                    const double tn = 0.5 * (1.0 + sqrt(1.0 + 4.0 * t * t)), beta = (t - 1.0) / tn;
                    t = tn;
                    for (size_t ip = 0; ip < nbuf; ip++) {
                        itW[2 * ip] = itX[ip] + beta * (itX[ip] - itXP[ip]);
                        itW[2 * ip + 1] = 0.0;
                    }
                    orc_fft2(g.n0, g.n1, itW, -1);
                    for (size_t ip = 0; ip < nbuf; ip++) {
                        const double q = itP[ip] + mu;
                        itW[2 * ip] = q * itW[2 * ip] - itB[2 * ip];
                        itW[2 * ip + 1] = q * itW[2 * ip + 1] - itB[2 * ip + 1];
                    }
                    orc_fft2(g.n0, g.n1, itW, +1);
                    for (size_t ip = 0; ip < nbuf; ip++) {
                        const double x = itX[ip], y = x + beta * (x - itXP[ip]);
                        const double v = y - tau * itW[2 * ip] / n;
                        itXP[ip] = x;
                        itX[ip] = v > thr ? v - thr : (v < -thr ? v + thr : 0.0);
                    }
                }
                for (size_t ip = 0; ip < nbuf; ip++) decon[2 * ip] = itX[ip] * n;
            }
            double *wo = winout + (size_t)stepindex * nout;
            for (int ixx = 0; ixx < g.outwinx; ixx++)
                for (int izz = 0; izz < g.outwinz; izz++) {
                    int ip = (g.ocx - g.halfoutwx + ixx) * g.FZ + g.ocz - g.halfoutwz + izz;
                    wo[ixx * g.outwinz + izz] = decon[2 * ip];
                }
        }
        free(snapm); free(snapsf); free(decon);
        free(itB); free(itP); free(itX); free(itXP); free(itW);
    }
    /* overlap-add in window order, float accumulators as in the reference (:656-673) */
    for (int stepindex = 0; stepindex < g.totalnum; stepindex++) {
        int ix = g.stepwinx * (stepindex / g.stepnumz);
        int iz = g.stepwinz * (stepindex % g.stepnumz);
        const double *wo = winout + (size_t)stepindex * nout;
        for (int ixx = 0; ixx < g.outwinx; ixx++)
            for (int izz = 0; izz < g.outwinz; izz++) {
                int ipc = ixx * g.outwinz + izz;
                int iix = ix - g.halfoutwx + ixx, iiz = iz - g.halfoutwz + izz;
                if (iix >= 0 && iix < nxp && iiz >= 0 && iiz < nzp) {
                    size_t ipp = (size_t)iix * nzp + iiz;
                    mig_dec[ipp] += wo[ipc] * coefr[ipc];
                    mig_coef[ipp] += coefr[ipc];
                }
            }
    }
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            out_dec[ix * nz + iz] = mig_dec[(size_t)ix * nzp + iz];
            out_coef[ix * nz + iz] = mig_coef[(size_t)ix * nzp + iz];
        }
    free(winout); free(migrealf); free(migpsff); free(coefr); free(mig_dec); free(mig_coef);
    return 0;
}

/* ---------------- propagation / imaging restatements, float and double ---------------- */
#define T float
#define SFX f32
#include "prop_impl.h"
#undef T
#undef SFX
#define T double
#define SFX f64
#include "prop_impl.h"
#undef T
#undef SFX
