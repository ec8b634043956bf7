// ref_rtm_abi.cpp -- libswd_refrtm.so: the GPU entry points that the reference's AVSPRTM host
// program calls (headrtm.h: getdevice, variables_malloc, variables_free,
// fdtd_2d_GPU_forward, fdtd_2d_GPU_backward), implemented over libswd.  Linking the
// unmodified acoustic_HLVSPRTMC.cpp against this library instead of acoustic_HLVSPRTMLc.cu
// runs the reference's own shot loop, I/O and per-shot post on this engine.
//
// Differences a caller can see: none in the results the host reads (seismogram_obs / _syn,
// image_pp, image_sources, image_receivers; the FP64 image accumulators are rounded to the
// reference's float arrays, image_ppcig stays zero as the reference's launched kernels leave
// it).  The final forward wavefield stays in device memory between the two calls instead of
// ./output/wavefield*_itmax*.dat, and no device arrays are allocated in plan[].
#include <string.h>
#include "compat_common.h"

using namespace swd_compat;

extern "C" {

void getdevice(int *GPU_N)
{
    int n = 0;
    if (swd_device_count(&n) != SWD_OK) n = 0;
    *GPU_N = n;
}

void variables_malloc(int ntx, int ntz, int ntp, int nx, int nz, int pml, int Lc, float dx, float dz, int itmax,
                      int thetan, int delt, RtmPlan plan[], int GPU_N, int rnmax)
{
    (void)ntx; (void)ntz; (void)ntp; (void)thetan; (void)delt; (void)plan; (void)GPU_N; (void)rnmax;
    record_dims(nx, nz, pml, Lc, dx, dz, itmax);
}

void variables_free(int ntx, int ntz, int ntp, int nx, int nz, int pml, int Lc, float dx, float dz, int itmax,
                    RtmPlan plan[], int GPU_N, int rnmax)
{
    (void)ntx; (void)ntz; (void)ntp; (void)nx; (void)nz; (void)pml; (void)Lc; (void)dx; (void)dz; (void)itmax;
    (void)plan; (void)GPU_N; (void)rnmax;
    release_all();
}

// inv_flag 0: observed data into seismogram_obs; 1: the RTM forward pass (synthetic data into
// seismogram_syn, final wavefield and boundary strips kept for fdtd_2d_GPU_backward)
void fdtd_2d_GPU_forward(int ntx, int ntz, int ntp, int nx, int nz, int pml, int Lc, float *rc, float dx, float dz,
                         float *rick, int itmax, float dt, int myid, int is, RefSource ss[], RtmPlan plan[], int GPU_N,
                         int rnmax, float *vp, float *rho, int *mx, float *k_x, float *k_x_half, float *k_z,
                         float *k_z_half, float *a_x, float *a_x_half, float *a_z, float *a_z_half, float *b_x,
                         float *b_x_half, float *b_z, float *b_z_half, float *c, int inv_flag)
{
    (void)ntz; (void)ntp; (void)nx; (void)nz; (void)dx; (void)dz; (void)myid; (void)rnmax; (void)mx;
    (void)k_x; (void)k_x_half; (void)k_z; (void)k_z_half; (void)c;
    for (int i = 0; i < GPU_N; i++) {
        swd_ctx *ctx = context(i, dt);
        load_operator(ctx, rc, vp, rho, a_x, a_x_half, a_z, a_z_half, b_x, b_x_half, b_z, b_z_half);
        ShotCells sc;
        shot_cells(ss[is + i], ntx, pml + Lc, itmax, sc);
        if (inv_flag == 0)
            check(ctx, swd_forward(ctx, &sc.shot, rick, nullptr, nullptr, plan[i].seismogram_obs, nullptr, nullptr),
                  "swd_forward");
        else
            check(ctx, swd_rtm_forward(ctx, &sc.shot, rick, plan[i].seismogram_syn), "swd_rtm_forward");
    }
}

// Backward pass of the shots of the preceding forward call: the host's preprocessed data in
// seismogram_rms are injected; raw I, S and R go to image_pp, image_sources, image_receivers.
void fdtd_2d_GPU_backward(int ntx, int ntz, int ntp, int nx, int nz, int pml, int Lc, float *rc, float dx, float dz,
                          float *rick, int itmax, float dt, int myid, int thetan, int delt, int is, RefSource ss[],
                          RtmPlan plan[], int GPU_N, int rnmax, float *vp, float *rho, int *mx, float *k_x,
                          float *k_x_half, float *k_z, float *k_z_half, float *a_x, float *a_x_half, float *a_z,
                          float *a_z_half, float *b_x, float *b_x_half, float *b_z, float *b_z_half)
{
    (void)nx; (void)nz; (void)rc; (void)dx; (void)dz; (void)rick; (void)myid; (void)delt; (void)rnmax; (void)vp;
    (void)rho; (void)mx; (void)k_x; (void)k_x_half; (void)k_z; (void)k_z_half; (void)a_x; (void)a_x_half;
    (void)a_z; (void)a_z_half; (void)b_x; (void)b_x_half; (void)b_z; (void)b_z_half;
    std::vector<double> I((size_t)ntp), S((size_t)ntp), R((size_t)ntp);
    for (int i = 0; i < GPU_N; i++) {
        swd_ctx *ctx = context(i, dt);
        ShotCells sc;
        shot_cells(ss[is + i], ntx, pml + Lc, itmax, sc);
        check(ctx, swd_rtm_backward(ctx, &sc.shot, plan[i].seismogram_rms, SWD_RTM_ILLUM_RCV | SWD_RTM_NO_STACK,
                                    nullptr, nullptr, nullptr),
              "swd_rtm_backward");
        check(ctx, swd_rtm_raw(ctx, I.data(), S.data(), R.data()), "swd_rtm_raw");
        for (int ip = 0; ip < ntp; ip++) {
            plan[i].image_pp[ip] = (float)I[ip];
            plan[i].image_sources[ip] = (float)S[ip];
            plan[i].image_receivers[ip] = (float)R[ip];
        }
        memset(plan[i].image_ppcig, 0, sizeof(float) * (size_t)ntp * thetan);
        (void)ntz;
    }
}

}  // extern "C"
