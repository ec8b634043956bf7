// AFor -- drop-in forward-modelling program (the reference's forward/AFor,
// forward/acoustic_hilbert_fftkz_HLForC.cpp:13-892) on libswd.
//
// Run from the `forward/` directory of a project tree: reads ../parameter.txt and
// ../input/acc_vp.bin, writes ../output/.  For every shot it propagates the pressure field
// and its time-Hilbert twin, records the two edge wells, and splits them into up- and
// down-going traces in kz (scaled by nfftz like the reference's unnormalised inverse FFT).
//   scatter_flag = 0: %dsource_seismogram_{obs,obsup,obsdown}.bin
//   scatter_flag = 1: smoothed model, background run (%dsource_seismogram_sobs*), scatter
//     points added on the swin lattice, perturbed run, differences written as
//     %dsource_seismogram_scatter{,up,down}.bin.  The reference perturbs density
//     (rho += 1e-3*vp, :697-705); `swd.perturb = velocity` in parameter.txt multiplies vp by
//     (1 + swd.perturb_amp, default 0.01) instead.
// Extensions (parameter.txt lines `swd.key = value`): device, perturb (density|velocity; an
// unknown value is an error), perturb_amp.
#include <math.h>
#include "common.h"

using namespace drv;

int main(int, char **)
{
    const std::string up = "..";
    ModelParams m;
    if (!read_model_params((up + "/parameter.txt").c_str(), m)) {
        printf("Cannot open the parameters1 file!\n");
        return 1;
    }
    auto ext = extensions((up + "/parameter.txt").c_str());
    const int device = ext_int(ext, "device", 0);
    std::string perturb;
    if (!ext_choice(ext, "perturb", {"density", "velocity"}, perturb)) return 1;
    const float perturb_amp = (float)atof(ext_str(ext, "perturb_amp", "0.01").c_str());
    printf("Number of MPI thread is 1\n");
    printf("The simulation time step is %d\n", m.itmax);

    const int pmlc = m.pml + m.Lc;
    const int ntz = m.nz + 2 * pmlc, ntx = m.nx + 2 * pmlc;
    const size_t ntp = (size_t)ntz * ntx;
    Operator op = make_operator(m, ntx, ntz, pmlc);

    // shots and the two edge wells (forward/...HLForC.cpp:144-191)
    const int r_n = swd_prep_wells(m.nx, m.nz, pmlc, m.dz, m.shotdep, m.offsetz, nullptr, nullptr);
    std::vector<int> r_ix(r_n), r_iz(r_n);
    swd_prep_wells(m.nx, m.nz, pmlc, m.dz, m.shotdep, m.offsetz, r_ix.data(), r_iz.data());
    printf("The maximum trace number for source is %d\n", r_n);
    if (r_n < 2) {
        printf("No receiver depth lies within the maximum offset\n");
        return 1;
    }

    // kz taper (forward/...HLForC.cpp:354-377)
    const int nfftz = swd_prep_pow2(ntz);
    std::vector<float> coef(nfftz);
    const int layerz = swd_prep_kz_taper(nfftz, m.dz, coef.data());
    {
        float dkz = 1.0 / (nfftz * m.dz);
        float kcut = 1.0 / 15.0 / m.dz;
        printf("\nDamping wavenumber point No. = %d; NFFTz = %d\n\n", (int)(kcut / dkz), nfftz);
    }
    if (layerz < 0) {
        printf("Damping wavenumber is to long !\nBreak up!\n");
        return 0;
    }

    swd_ctx *ctx = make_context(m, device);
    // wavelet and its Hilbert twin (:385-403)
    std::vector<float> rick(m.itmax), hrick(m.itmax);
    swd_prep_ricker(m.itmax, m.f0, m.dt, rick.data());
    write_f32(up + "/output/rick_second_derive.bin", rick.data(), m.itmax);
    printf("Ricker wave is done\n");
    die_on(ctx, swd_hilbert(ctx, m.itmax, rick.data(), hrick.data()), "swd_hilbert");
    write_f32(up + "/output/rick_hilbert.bin", hrick.data(), m.itmax);

    // true model (get_acc_model, :412-439)
    std::vector<float> vin((size_t)m.nx * m.nz), vp(ntp), rho(ntp, 1000.0f);
    if (!read_f32(up + "/input/acc_vp.bin", vin.data(), vin.size())) return 1;
    swd_prep_pad(m.nx, m.nz, pmlc, vin.data(), vp.data());
    write_f32(up + "/output/acc_vp.bin", interior(vp, ntx, ntz, pmlc).data(), (size_t)m.nx * m.nz);
    write_f32(up + "/output/acc_vpful.bin", vp.data(), ntp);
    write_f32(up + "/output/acc_rho.bin", interior(rho, ntx, ntz, pmlc).data(), (size_t)m.nx * m.nz);
    printf("The true model is done\n");
    float vmax = 0, vmin = 5000, rmax = 0, rmin = 5000;
    for (size_t ip = 0; ip < ntp; ip++) {
        if (vp[ip] >= vmax) vmax = vp[ip];
        if (vp[ip] <= vmin) vmin = vp[ip];
        if (rho[ip] >= rmax) rmax = rho[ip];
        if (rho[ip] <= rmin) rmin = rho[ip];
    }
    printf("vp_max = %f\nrho_max = %f\nvp_min = %f\nrho_min = %f\n", vmax, rmax, vmin, rmin);
    die_on(ctx, swd_set_stencil(ctx, op.rc.data()), "swd_set_stencil");
    die_on(ctx, swd_set_cpml(ctx, op.ax.data(), op.axh.data(), op.az.data(), op.azh.data(), op.bx.data(),
                             op.bxh.data(), op.bz.data(), op.bzh.data()), "swd_set_cpml");
    printf("ABC parameters are done\n");

    const size_t ntr = (size_t)r_n * m.itmax;
    std::vector<float> obs(ntr), obsup(ntr), obsdown(ntr);
    auto shot_of = [&](int is) {
        swd_shot s;
        s.s_ix = pmlc + (int)(m.sx0 / m.dx) + (int)(m.shotdx / m.dx) * is;
        s.s_iz = pmlc + (int)(m.shotdep / m.dz);
        s.nt = m.itmax;
        s.r_n = r_n;
        s.r_ix = r_ix.data();
        s.r_iz = r_iz.data();
        return s;
    };
    auto run = [&](int is, std::vector<float> &a, std::vector<float> &b, std::vector<float> &c) {
        swd_shot s = shot_of(is);
        die_on(ctx, swd_forward(ctx, &s, rick.data(), hrick.data(), coef.data(), a.data(), b.data(), c.data()),
               "swd_forward");
    };
    auto shotfile = [&](int is, const char *kind) {
        char name[64];
        snprintf(name, sizeof name, "/output/%dsource_seismogram_%s.bin", is + 1, kind);
        return up + name;
    };
    printf("====================\n");
    if (m.scatter_flag == 0) {
        printf("    The Scatter Flag == %d--- NORMAL\n====================\n", m.scatter_flag);
        printf("Obtain the observed seismogram !\n");
        die_on(ctx, swd_set_model(ctx, vp.data(), rho.data()), "swd_set_model");
        for (int is = 0; is < m.ns; is++) {
            run(is, obs, obsup, obsdown);
            write_f32(shotfile(is, "obs"), obs.data(), ntr);
            write_f32(shotfile(is, "obsup"), obsup.data(), ntr);
            write_f32(shotfile(is, "obsdown"), obsdown.data(), ntr);
        }
    } else {
        printf("    The Scatter Flag == %d--- PSF\n====================\n", m.scatter_flag);
        die_on(ctx, swd_smooth(ctx, ntx, ntz, pmlc, m.window, vp.data()), "swd_smooth");
        write_f32(up + "/output/ini_vp.bin", interior(vp, ntx, ntz, pmlc).data(), (size_t)m.nx * m.nz);
        printf("Obtain the background scatter seismogram !\n");
        die_on(ctx, swd_set_model(ctx, vp.data(), rho.data()), "swd_set_model");
        std::vector<std::vector<float>> bg(3 * (size_t)m.ns);
        for (int is = 0; is < m.ns; is++) {
            run(is, obs, obsup, obsdown);
            write_f32(shotfile(is, "sobs"), obs.data(), ntr);
            write_f32(shotfile(is, "sobsup"), obsup.data(), ntr);
            write_f32(shotfile(is, "sobsdown"), obsdown.data(), ntr);
            bg[3 * is] = obs;
            bg[3 * is + 1] = obsup;
            bg[3 * is + 2] = obsdown;
        }
        printf("The scatter model is done\n");
        std::vector<float> vps = vp, rhos = rho;
        for (int ix = pmlc + m.swin / 2; ix < ntx - pmlc - m.swin / 2; ix++)
            for (int iz = pmlc + m.swin / 2; iz < ntz - pmlc - 5; iz++)
                if ((ix - (pmlc + m.swin / 2)) % m.swin == 0 && (iz - (pmlc + m.swin / 2)) % m.swin == 0) {
                    const size_t ip = (size_t)ix * ntz + iz;
                    if (perturb == "velocity") vps[ip] *= (1.0f + perturb_amp);
                    else rhos[ip] += vp[ip] * 1.0e-3f;
                }
        write_f32(up + "/output/ini_scatter_vp.bin", interior(vps, ntx, ntz, pmlc).data(), (size_t)m.nx * m.nz);
        write_f32(up + "/output/rho_scatter.bin", interior(rhos, ntx, ntz, pmlc).data(), (size_t)m.nx * m.nz);
        printf("Obtain the observed scatter seismogram !\n");
        die_on(ctx, swd_set_model(ctx, vps.data(), rhos.data()), "swd_set_model");
        for (int is = 0; is < m.ns; is++) {
            run(is, obs, obsup, obsdown);
            for (size_t ip = 0; ip < ntr; ip++) {
                obs[ip] -= bg[3 * is][ip];
                obsup[ip] -= bg[3 * is + 1][ip];
                obsdown[ip] -= bg[3 * is + 2][ip];
            }
            write_f32(shotfile(is, "scatter"), obs.data(), ntr);
            write_f32(shotfile(is, "scatterup"), obsup.data(), ntr);
            write_f32(shotfile(is, "scatterdown"), obsdown.data(), ntr);
        }
    }
    printf("====================\n      THE END\n====================\n");
    swd_destroy(ctx);
    return 0;
}
