// host_prep.cpp -- the reference's host-side preparation, restated for libswd.
//
// These run once per model/shot on the host, exactly as in the reference programs: the
// stencil coefficients, CPML profiles, Ricker wavelet, model padding, kz taper and the
// two-edge-well receiver geometry.  They are written in C++ with the reference's float /
// double types so that overloads (std::exp(float) -> expf, std::log(float) -> logf, ...)
// resolve as they do in acoustic_HLVSPRTMC.cpp, and the results are bit-identical.
#include <math.h>
#include <string.h>
#include <vector>
#include "../../include/swd.h"

extern "C" {

// cal_xishu, acoustic_HLVSPRTMC.cpp:1858-1878
void swd_prep_xishu(int Lx, float *rx)
{
    for (int m = 1; m <= Lx; m++) {
        float s1 = 1.0, s2 = 1.0;
        for (int i = 1; i < m; i++) {
            s1 = s1 * (2.0 * i - 1) * (2.0 * i - 1);
            s2 = s2 * ((2.0 * m - 1) * (2.0 * m - 1) - (2.0 * i - 1) * (2.0 * i - 1));
        }
        for (int i = m + 1; i <= Lx; i++) {
            s1 = s1 * (2.0 * i - 1) * (2.0 * i - 1);
            s2 = s2 * ((2.0 * m - 1) * (2.0 * m - 1) - (2.0 * i - 1) * (2.0 * i - 1));
        }
        s2 = fabs(s2);
        rx[m - 1] = pow(-1.0, m + 1) * s1 / (s2 * (2.0 * m - 1));
    }
}

// One axis of get_absorbing_parameters, acoustic_HLVSPRTMC.cpp:967-1120.  Both axes use
// the same d0 (thickness pml*dz, :925) and the same constants.
static void cpml_axis(int n, int pml, float h, float d0, float thickness_of_pml, float dt,
                      float *a, float *a_half, float *b, float *b_half)
{
    float pi = 3.1415927;
    float alpha_max = pi * 15;
    std::vector<float> d(n, 0.0f), d_half(n, 0.0f), k(n, 1.0f), k_half(n, 1.0f), al(n, 0.0f), al_half(n, 0.0f);
    for (int i = 0; i < n; i++) { a[i] = 0.0; a_half[i] = 0.0; b[i] = 0.0; b_half[i] = 0.0; }
    float start = pml * h;
    float end = (n - pml - 1) * h;
    float cur, delta;
    for (int i = 0; i < n; i++) {
        cur = i * h;
        if (cur <= start) {
            delta = start - cur;
            d[i] = d0 * pow(delta / thickness_of_pml, 2);
            k[i] = 1.0;
            al[i] = alpha_max * (1.0 - (delta / thickness_of_pml)) + 0.1 * alpha_max;
        }
        if (cur >= end) {
            delta = cur - end;
            d[i] = d0 * pow(delta / thickness_of_pml, 2);
            k[i] = 1.0;
            al[i] = alpha_max * (1.0 - (delta / thickness_of_pml)) + 0.1 * alpha_max;
        }
    }
    for (int i = 0; i < n; i++) {
        cur = (i + 0.5) * h;
        if (cur <= start) {
            delta = start - cur;
            d_half[i] = d0 * pow(delta / thickness_of_pml, 2);
            k_half[i] = 1.0;
            al_half[i] = alpha_max * (1.0 - (delta / thickness_of_pml)) + 0.1 * alpha_max;
        }
        if (cur >= end) {
            delta = cur - end;
            d_half[i] = d0 * pow(delta / thickness_of_pml, 2);
            k_half[i] = 1.0;
            al_half[i] = alpha_max * (1.0 - (delta / thickness_of_pml)) + 0.1 * alpha_max;
        }
    }
    for (int i = 0; i < n; i++) {
        if (al[i] < 0.0) al[i] = 0.0;
        if (al_half[i] < 0.0) al_half[i] = 0.0;
        b[i] = exp(-(d[i] / k[i] + al[i]) * dt);
        if (d[i] > 1.0e-6) a[i] = d[i] / (k[i] * (d[i] + k[i] * al[i])) * (b[i] - 1.0);
        b_half[i] = exp(-(d_half[i] / k_half[i] + al_half[i]) * dt);
        if (d_half[i] > 1.0e-6) a_half[i] = d_half[i] / (k_half[i] * (d_half[i] + k_half[i] * al_half[i])) * (b_half[i] - 1.0);
    }
}

// get_absorbing_parameters, acoustic_HLVSPRTMC.cpp:891-1129 (pml = pmlc, Vpmax = 5500).
void swd_prep_cpml(int ntx, int ntz, int pml, float dx, float dz, float dt,
                   float *a_x, float *a_x_half, float *a_z, float *a_z_half,
                   float *b_x, float *b_x_half, float *b_z, float *b_z_half)
{
    int N = 2;
    float Rc = 1.0e-5;
    float Vpmax = 5500;
    float thickness_of_pml = pml * dz;
    float d0 = -(N + 1) * Vpmax * log(Rc) / (2.0 * thickness_of_pml);
    cpml_axis(ntx, pml, dx, d0, thickness_of_pml, dt, a_x, a_x_half, b_x, b_x_half);
    cpml_axis(ntz, pml, dz, d0, thickness_of_pml, dt, a_z, a_z_half, b_z, b_z_half);
}

// ricker_wave(flag = 2) with t0 = 1.0/f0, acoustic_HLVSPRTMC.cpp:96,1249-1299
void swd_prep_ricker(int itmax, float f0, float dt, float *rick)
{
    float pi = 3.1415927;
    float t0 = 1.0 / f0;
    float temp;
    for (int it = 0; it < itmax; it++) {
        temp = pi * f0 * (it * dt - t0);
        temp = temp * temp;
        rick[it] = (1.0 - 2.0 * temp) * exp(-temp);
    }
}

// get_acc_model: interior read-in and edge replication, acoustic_HLVSPRTMC.cpp:1136-1196
void swd_prep_pad(int nx, int nz, int pml, const float *v_in, float *vp)
{
    int ntx = nx + 2 * pml, ntz = nz + 2 * pml;
    size_t k = 0;
    for (int ix = pml; ix < ntx - pml; ix++)
        for (int iz = pml; iz < ntz - pml; iz++) vp[(size_t)ix * ntz + iz] = v_in[k++];
    for (int iz = pml; iz <= ntz - pml - 1; iz++) {
        for (int ix = 0; ix <= pml - 1; ix++) vp[(size_t)ix * ntz + iz] = vp[(size_t)pml * ntz + iz];
        for (int ix = ntx - pml; ix < ntx; ix++) vp[(size_t)ix * ntz + iz] = vp[(size_t)(ntx - pml - 1) * ntz + iz];
    }
    for (int ix = 0; ix < ntx; ix++) {
        for (int iz = 0; iz <= pml - 1; iz++) vp[(size_t)ix * ntz + iz] = vp[(size_t)ix * ntz + pml];
        for (int iz = ntz - pml; iz < ntz; iz++) vp[(size_t)ix * ntz + iz] = vp[(size_t)ix * ntz + (ntz - pml - 1)];
    }
}

// (int)pow(2.0, (int)ceil(log(1.0*n)/log(2.0))), forward/...HLForC.cpp:299-300 and
// forward/...HLForLc.cu:1263-1264
int swd_prep_pow2(int n)
{
    int K = (int)ceil(log(1.0 * n) / log(2.0));
    return (int)pow(2.0, K);
}

// kz taper, forward/acoustic_hilbert_fftkz_HLForC.cpp:354-377 (PI = 3.1415926)
int swd_prep_kz_taper(int nfftz, float dz, float *coef)
{
    const double PI = 3.1415926;
    float dkz = 1.0 / (nfftz * dz);
    float kcut = 1.0 / 15.0 / dz;
    int layerz = kcut / dkz;
    if (layerz > nfftz / 6) return -1;
    int upz = layerz, downz = nfftz - layerz;
    for (int iz = 0; iz < nfftz; iz++) {
        if (iz <= upz) coef[iz] = 0.5000 - 0.5 * cos(PI * iz / layerz);
        if (iz > upz && iz < downz) coef[iz] = 1.0;
        if (iz >= downz) coef[iz] = 0.5000 + 0.5 * cos(PI * (iz - downz) / layerz);
    }
    return layerz;
}

// Two edge wells: depth list of acoustic_HLVSPRTMC.cpp:153-200 recorded at ix = pmlc and
// ix = ntx-pmlc-1 (acoustic_HLVSPRTMLc.cu:180-197).  Traces [0, r_n/2) are the left well.
int swd_prep_wells(int nx, int nz, int pmlc, float dz, float shotdep, float offsetz, int *r_ix, int *r_iz)
{
    int ntx = nx + 2 * pmlc;
    int s_iz = pmlc + (int)(shotdep / dz);
    int cnt = 0;
    for (int iz = 0; iz < nz; iz++)
        if (fabs(s_iz - iz - pmlc) * dz <= offsetz) cnt++;
    int r_n = 2 * cnt;
    if (r_ix && r_iz) {
        int i = 0;
        for (int iz = 0; iz < nz; iz++) {
            if (fabs(s_iz - iz - pmlc) * dz <= offsetz) {
                r_iz[i] = pmlc + iz; r_ix[i] = pmlc;
                r_iz[i + r_n / 2] = pmlc + iz; r_ix[i + r_n / 2] = ntx - pmlc - 1;
                i++;
            }
        }
    }
    return r_n;
}

}  // extern "C"
