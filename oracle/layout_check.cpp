// layout_check.cpp -- TEST INFRASTRUCTURE.  Compiled against one of the reference's own
// headers (headrtm.h of the RTM program, or forward/headrtm.h of AFor with -DFWD) and the
// package's compat layouts (csrc/compat/ref_layouts.h).  For every named member of the compat
// structs it prints the member's offset in the reference's struct and in the compat struct,
// and the sizes of both, as lines "<struct> <member> <reference> <compat>"; the tests require
// the two columns to agree.
#include <cstddef>
#include <cstdio>
#include "headrtm.h"
#include "compat/ref_layouts.h"

#define ROW(REF, OURS, f) std::printf("%s %s %zu %zu\n", #OURS, #f, offsetof(REF, f), offsetof(swd_compat::OURS, f))

int main()
{
    std::printf("RefSource size %zu %zu\n", sizeof(Source), sizeof(swd_compat::RefSource));
    ROW(Source, RefSource, s_iz);
    ROW(Source, RefSource, s_ix);
    ROW(Source, RefSource, r_ix);
    ROW(Source, RefSource, r_n);
    ROW(Source, RefSource, r_iz);
#ifdef FWD
#define M(f) ROW(MultiGPU, FwdPlan, f);
    std::printf("FwdPlan size %zu %zu\n", sizeof(MultiGPU), sizeof(swd_compat::FwdPlan));
    M(coef) M(vx) M(vz) M(p) M(htp) M(spu) M(spd) M(rpu) M(rpd)
    M(vx_inv) M(vz_inv) M(p_inv) M(phi_vx_x) M(phi_vz_z) M(phi_p_x) M(phi_p_z)
    M(seismogram_obs) M(seismogram_up) M(seismogram_down) M(seismogram_dir) M(seismogram_dirup)
    M(seismogram_dirdown) M(seismogram_syn) M(seismogram_rms) M(seismogram_rmsup) M(seismogram_rmsdown)
    M(seismogram_hrms)
    M(p_borders_up) M(p_borders_bottom) M(p_borders_left) M(p_borders_right)
    M(image_pp) M(image_ppdu) M(image_ppud) M(image_ppcig) M(image_sources) M(image_receivers)
    M(forward_z) M(backward_z)
#else
#define M(f) ROW(MultiGPU, RtmPlan, f);
    std::printf("RtmPlan size %zu %zu\n", sizeof(MultiGPU), sizeof(swd_compat::RtmPlan));
    M(vx) M(vz) M(p) M(vx_inv) M(vz_inv) M(p_inv) M(phi_vx_x) M(phi_vz_z) M(phi_p_x) M(phi_p_z)
    M(seismogram_obs) M(seismogram_dir) M(seismogram_syn) M(seismogram_rms) M(seismogram_rmsup)
    M(seismogram_rmsdown) M(seismogram_frms)
    M(p_borders_up) M(p_borders_bottom) M(p_borders_left) M(p_borders_right)
    M(image_pp) M(image_ppcig) M(image_sources) M(image_receivers)
    M(forward_z)
#endif
    return 0;
}
