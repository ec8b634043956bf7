// ref_fwd_abi.cpp -- libswd_reffwd.so: the GPU entry points that the reference's AFor host
// program calls (forward/headrtm.h: getdevice, variables_malloc, variables_free,
// fdtd_2d_GPU_forward with the Hilbert twin, hilbert_transform1d), implemented over libswd.
// Linking the unmodified forward/acoustic_hilbert_fftkz_HLForC.cpp against this library
// instead of forward/acoustic_hilbert_fftkz_HLForLc.cu runs AFor's own flow on this engine:
// full, up-going and down-going data (kz split with the host's taper plan[i].coef, scaled by
// nfftz like the reference's unnormalised inverse FFT).
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
                      int thetan, int delt, FwdPlan plan[], int GPU_N, int rnmax)
{
    (void)ntx; (void)ntz; (void)ntp; (void)thetan; (void)delt; (void)plan; (void)GPU_N; (void)rnmax;
    record_dims(nx, nz, pml, Lc, dx, dz, itmax);
}

void variables_free(int ntx, int ntz, int ntp, int nx, int nz, int pml, int Lc, float dx, float dz, int itmax,
                    FwdPlan plan[], int GPU_N, int rnmax)
{
    (void)ntx; (void)ntz; (void)ntp; (void)nx; (void)nz; (void)pml; (void)Lc; (void)dx; (void)dz; (void)itmax;
    (void)plan; (void)GPU_N; (void)rnmax;
    release_all();
}

// The wavelet's Hilbert transform (forward/...HLForLc.cu:1257-1324).  The host calls it before
// any propagation, when dt is not yet known; the transform does not depend on dt, so a
// context with a placeholder step serves (it is rebuilt when the first shot brings dt).
void hilbert_transform1d(float *rick, float *rick_hilbert, int itmax)
{
    swd_ctx *ctx = context(0, session().dev.empty() || !session().dev[0].ctx ? 1.0f : session().dev[0].grid.dt);
    check(ctx, swd_hilbert(ctx, itmax, rick, rick_hilbert), "swd_hilbert");
}

void fdtd_2d_GPU_forward(int ntx, int ntz, int ntp, int nx, int nz, int pml, int Lc, float *rc, float dx, float dz,
                         float *rick, float *hrick, int itmax, float dt, int myid, int is, RefSource ss[],
                         FwdPlan plan[], int GPU_N, int rnmax, float *vp, float *rho, int *mx, float *k_x,
                         float *k_x_half, float *k_z, float *k_z_half, float *a_x, float *a_x_half, float *a_z,
                         float *a_z_half, float *b_x, float *b_x_half, float *b_z, float *b_z_half, float *c,
                         int inv_flag)
{
    (void)ntz; (void)ntp; (void)nx; (void)nz; (void)dx; (void)dz; (void)myid; (void)rnmax; (void)mx;
    (void)k_x; (void)k_x_half; (void)k_z; (void)k_z_half; (void)c; (void)inv_flag;
    for (int i = 0; i < GPU_N; i++) {
        swd_ctx *ctx = context(i, dt);
        load_operator(ctx, rc, vp, rho, a_x, a_x_half, a_z, a_z_half, b_x, b_x_half, b_z, b_z_half);
        ShotCells sc;
        shot_cells(ss[is + i], ntx, pml + Lc, itmax, sc);
        check(ctx,
              swd_forward(ctx, &sc.shot, rick, hrick, plan[i].coef, plan[i].seismogram_obs, plan[i].seismogram_up,
                          plan[i].seismogram_down),
              "swd_forward");
    }
}

}  // extern "C"
