// ref_layouts.h -- the memory layouts of the reference's `struct Source` and of its two
// `struct MultiGPU` bundles, as the unmodified reference host programs pass them to the GPU
// entry points.  The compat libraries (libswd_refrtm.so, libswd_reffwd.so) read and write
// these structs, so field order and types follow the reference headers exactly: every
// member is a pointer except the trailing cuFFT plan handles (int).  Only the host-side
// result arrays are used here; the device pointers are never touched.
//   Source:              headrtm.h:8-13, forward/headrtm.h:12-18
//   MultiGPU (RTM):      headrtm.h:16-98
//   MultiGPU (forward):  forward/headrtm.h:20-127
#pragma once

namespace swd_compat {

struct RefSource {
    int s_iz, s_ix, r_ix, r_n;
    int *r_iz;
};

// AVSPRTM's bundle: 80 pointers, then one plan handle
struct RtmPlan {
    float *vx, *vz, *p;
    float *vx_inv, *vz_inv, *p_inv;
    float *phi_vx_x, *phi_vz_z, *phi_p_x, *phi_p_z;
    float *seismogram_obs, *seismogram_dir, *seismogram_syn, *seismogram_rms, *seismogram_rmsup,
        *seismogram_rmsdown, *seismogram_frms;
    float *p_borders_up, *p_borders_bottom, *p_borders_left, *p_borders_right;
    float *image_pp, *image_ppcig, *image_sources, *image_receivers;
    void *device_pointers[55];   // d_r_iz .. d_fxzr (device arrays of the reference engine)
    int forward_z;
};
static_assert(sizeof(RtmPlan) == 80 * sizeof(void *) + 8, "RTM MultiGPU layout");

// AFor's bundle: 103 pointers, then two plan handles
struct FwdPlan {
    float *coef;
    float *vx, *vz;
    void *p, *htp, *spu, *spd, *rpu, *rpd;   // cufftComplex host arrays
    float *vx_inv, *vz_inv, *p_inv;
    float *phi_vx_x, *phi_vz_z, *phi_p_x, *phi_p_z;
    float *seismogram_obs, *seismogram_up, *seismogram_down, *seismogram_dir, *seismogram_dirup,
        *seismogram_dirdown, *seismogram_syn, *seismogram_rms, *seismogram_rmsup, *seismogram_rmsdown,
        *seismogram_hrms;
    float *p_borders_up, *p_borders_bottom, *p_borders_left, *p_borders_right;
    float *image_pp, *image_ppdu, *image_ppud, *image_ppcig, *image_sources, *image_receivers;
    void *device_pointers[66];   // d_coef .. d_fxzr
    int forward_z, backward_z;
};
static_assert(sizeof(FwdPlan) == 103 * sizeof(void *) + 8, "forward MultiGPU layout");

}  // namespace swd_compat
