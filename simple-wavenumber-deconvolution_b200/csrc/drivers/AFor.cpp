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
// unknown value is an error), perturb_amp, scatter_field (difference|exact): `difference`, the
// default, forms the scatter records as the reference does, perturbed run minus background run;
// `exact` propagates the difference field itself (swd_forward_scatter), whose FP32 error is
// relative to the scatter data instead of to the records.
// Per-shot receivers: ../input/%dsource_receivers.txt, when present, gives that shot its own
// receiver list (count, then "ix iz" interior cells); its records then hold that many traces.
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
    std::string perturb, sfield;
    if (!ext_choice(ext, "perturb", {"density", "velocity"}, perturb) ||
        !ext_choice(ext, "scatter_field", {"difference", "exact"}, sfield))
        return 1;
    const float perturb_amp = (float)atof(ext_str(ext, "perturb_amp", "0.01").c_str());
    printf("Number of MPI thread is 1\n");
    printf("The simulation time step is %d\n", m.itmax);

    const int pmlc = m.pml + m.Lc;
    const int ntz = m.nz + 2 * pmlc, ntx = m.nx + 2 * pmlc;
    const size_t ntp = (size_t)ntz * ntx;
    Operator op = make_operator(m, ntx, ntz, pmlc);

    // shots and their receivers: the two edge wells (forward/...HLForC.cpp:144-191) or the
    // shot's own list; every file is checked before any device work
    std::vector<Receivers> recv(m.ns);
    int rnmax = 0;
    for (int is = 0; is < m.ns; is++) {
        if (!shot_receivers(up, is, m, recv[is])) return 1;
        rnmax = (int)recv[is].ix.size() > rnmax ? (int)recv[is].ix.size() : rnmax;
    }
    printf("The maximum trace number for source is %d\n", rnmax);

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

    std::vector<float> obs, obsup, obsdown;
    auto shot_of = [&](int is) {
        swd_shot s;
        s.s_ix = pmlc + (int)(m.sx0 / m.dx) + (int)(m.shotdx / m.dx) * is;
        s.s_iz = pmlc + (int)(m.shotdep / m.dz);
        s.nt = m.itmax;
        s.r_n = (int)recv[is].ix.size();
        s.r_ix = recv[is].ix.data();
        s.r_iz = recv[is].iz.data();
        return s;
    };
    // records of shot is, sized for its receivers
    auto run = [&](int is, std::vector<float> &a, std::vector<float> &b, std::vector<float> &c, bool scat = false) {
        swd_shot s = shot_of(is);
        const size_t n = (size_t)s.r_n * m.itmax;
        a.resize(n);
        b.resize(n);
        c.resize(n);
        if (scat)
            die_on(ctx, swd_forward_scatter(ctx, &s, rick.data(), hrick.data(), coef.data(), a.data(), b.data(), c.data()),
                   "swd_forward_scatter");
        else
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
            write_f32(shotfile(is, "obs"), obs.data(), obs.size());
            write_f32(shotfile(is, "obsup"), obsup.data(), obsup.size());
            write_f32(shotfile(is, "obsdown"), obsdown.data(), obsdown.size());
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
            write_f32(shotfile(is, "sobs"), obs.data(), obs.size());
            write_f32(shotfile(is, "sobsup"), obsup.data(), obsup.size());
            write_f32(shotfile(is, "sobsdown"), obsdown.data(), obsdown.size());
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
        const bool exact = sfield == "exact";
        // exact: the background stays and the perturbed model drives the scattered field
        if (exact) die_on(ctx, swd_set_scatter_model(ctx, vps.data(), rhos.data()), "swd_set_scatter_model");
        else die_on(ctx, swd_set_model(ctx, vps.data(), rhos.data()), "swd_set_model");
        for (int is = 0; is < m.ns; is++) {
            run(is, obs, obsup, obsdown, exact);
            if (!exact)
                for (size_t ip = 0; ip < obs.size(); ip++) {
                    obs[ip] -= bg[3 * is][ip];
                    obsup[ip] -= bg[3 * is + 1][ip];
                    obsdown[ip] -= bg[3 * is + 2][ip];
                }
            write_f32(shotfile(is, "scatter"), obs.data(), obs.size());
            write_f32(shotfile(is, "scatterup"), obsup.data(), obsup.size());
            write_f32(shotfile(is, "scatterdown"), obsdown.data(), obsdown.size());
        }
    }
    printf("====================\n      THE END\n====================\n");
    swd_destroy(ctx);
    return 0;
}
