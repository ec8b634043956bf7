// AVSPRTM -- drop-in RTM / PSF-imaging program (the reference's AVSPRTM,
// acoustic_HLVSPRTMC.cpp:15-883) on libswd.
//
// Run from the project root: reads ./parameter.txt, ./input/acc_vp.bin and, per shot,
// ./output/%dsource_seismogram_obsup.bin (scatter_flag = 0) or ..._scatterup.bin
// (scatter_flag = 1) as written by AFor.  The migration model is the Gaussian smoothing of
// the true model (window from parameter.txt).  Per shot it writes image_pp%d / image_psf%d
// (normalised image), image_sources%d (source illumination), fimage_pp%d / fimage_psf%d
// (-vp^2 Laplacian), and, for every 20th shot, the synthetic and preprocessed data; at the
// end the stacked, edge-zeroed migration_pp.bin / migration_psf.bin.
// The final forward wavefield stays in GPU memory; the reference's wavefield%d_itmax%d.dat
// disk round trip is not needed.
// Extensions (parameter.txt lines `swd.key = value`): device, strip_precision
// (f32|f16|bf16|i16), data (up|full|down: which AFor record to migrate; the reference always
// uses up).  An unknown value of either is an error.
// Per-shot receivers: ./input/%dsource_receivers.txt, when present, gives that shot its own
// receiver list (count, then "ix iz" interior cells; AFor reads the same file); every record
// must hold exactly r_n x itmax floats of its shot.  All shots' geometry and record files are
// checked before any device work.
#include <math.h>
#include "common.h"

using namespace drv;

int main(int, char **)
{
    ModelParams m;
    if (!read_model_params("./parameter.txt", m)) {
        printf("Cannot open the parameters1 file!\n");
        return 1;
    }
    auto ext = extensions("./parameter.txt");
    const int device = ext_int(ext, "device", 0);
    std::string sp, which;
    if (!ext_choice(ext, "strip_precision", {"f32", "f16", "bf16", "i16"}, sp) ||
        !ext_choice(ext, "data", {"up", "full", "down"}, which))
        return 1;
    printf("Number of MPI thread is 1\n");
    printf("The simulation time step is %d\n", m.itmax);

    const int pmlc = m.pml + m.Lc;
    const int ntz = m.nz + 2 * pmlc, ntx = m.nx + 2 * pmlc;
    const size_t ntp = (size_t)ntz * ntx, np = (size_t)m.nx * m.nz;
    Operator op = make_operator(m, ntx, ntz, pmlc);
    // every shot's receivers and record, checked before any device work
    const char *suffix = which == "full" ? "" : (which == "down" ? "down" : "up");
    std::vector<Receivers> recv(m.ns);
    std::vector<std::string> files(m.ns);
    int rnmax = 0;
    for (int is = 0; is < m.ns; is++) {
        if (!shot_receivers(".", is, m, recv[is])) return 1;
        const int r_n = (int)recv[is].ix.size();
        rnmax = r_n > rnmax ? r_n : rnmax;
        char name[128];
        snprintf(name, sizeof name, "./output/%dsource_seismogram_%s%s.bin", is + 1, m.scatter_flag ? "scatter" : "obs",
                 suffix);
        files[is] = name;
        if (!check_record(files[is], r_n, m.itmax)) return 1;
    }
    printf("The maximum trace number for source is %d\n", rnmax);

    swd_ctx *ctx = make_context(m, device);
    if (sp == "f16") die_on(ctx, swd_set_strip_precision(ctx, SWD_STRIP_F16), "strip precision");
    else if (sp == "bf16") die_on(ctx, swd_set_strip_precision(ctx, SWD_STRIP_BF16), "strip precision");
    else if (sp == "i16") die_on(ctx, swd_set_strip_precision(ctx, SWD_STRIP_I16), "strip precision");

    std::vector<float> rick(m.itmax);
    swd_prep_ricker(m.itmax, m.f0, m.dt, rick.data());
    write_f32("./output/rick_second_derive.bin", rick.data(), m.itmax);
    printf("Ricker wave is done\n");

    std::vector<float> vin(np), vp(ntp), rho(ntp, 1000.0f);
    if (!read_f32("./input/acc_vp.bin", vin.data(), np)) return 1;
    swd_prep_pad(m.nx, m.nz, pmlc, vin.data(), vp.data());
    write_f32("./output/acc_vp.bin", interior(vp, ntx, ntz, pmlc).data(), np);
    write_f32("./output/acc_rho.bin", interior(rho, ntx, ntz, pmlc).data(), np);
    printf("The true model is done\n");
    float vmax = 0, vmin = 5000;
    for (size_t ip = 0; ip < ntp; ip++) {
        if (vp[ip] >= vmax) vmax = vp[ip];
        if (vp[ip] <= vmin) vmin = vp[ip];
    }
    printf("vp_max = %f\nrho_max = %f\nvp_min = %f\nrho_min = %f\n", vmax, 1000.0, vmin, 1000.0);
    die_on(ctx, swd_smooth(ctx, ntx, ntz, pmlc, m.window, vp.data()), "swd_smooth");
    write_f32("./output/ini_vp.bin", interior(vp, ntx, ntz, pmlc).data(), np);
    printf("The initial model is done\n");
    die_on(ctx, swd_set_stencil(ctx, op.rc.data()), "swd_set_stencil");
    die_on(ctx, swd_set_cpml(ctx, op.ax.data(), op.axh.data(), op.az.data(), op.azh.data(), op.bx.data(),
                             op.bxh.data(), op.bz.data(), op.bzh.data()), "swd_set_cpml");
    die_on(ctx, swd_set_model(ctx, vp.data(), rho.data()), "swd_set_model");
    printf("ABC parameters are done\n");
    printf("====================\n%s\n====================\n", m.scatter_flag ? " PSF RTM BEGIN" : " NORMAL RTM BEGIN");

    std::vector<float> data, syn, rms, img(np), src(np), fim(np);
    const char *tag = m.scatter_flag ? "psf" : "pp";
    die_on(ctx, swd_stack_reset(ctx), "swd_stack_reset");
    for (int is = 0; is < m.ns; is++) {
        char name[128];
        const int r_n = (int)recv[is].ix.size();
        const size_t ntr = (size_t)r_n * m.itmax;
        data.resize(ntr);
        syn.resize(ntr);
        rms.resize(ntr);
        if (!read_f32(files[is], data.data(), ntr)) return 1;
        swd_shot s;
        s.s_ix = pmlc + (int)(m.sx0 / m.dx) + (int)(m.shotdx / m.dx) * is;
        s.s_iz = pmlc + (int)(m.shotdep / m.dz);
        s.nt = m.itmax;
        s.r_n = r_n;
        s.r_ix = recv[is].ix.data();
        s.r_iz = recv[is].iz.data();
        die_on(ctx, swd_rtm_shot(ctx, &s, rick.data(), data.data(), SWD_RTM_PREPROCESS, syn.data(), img.data(),
                                 src.data(), fim.data()), "swd_rtm_shot");
        if (is % 20 == 0) {
            snprintf(name, sizeof name, "./output/%dsource_seismogram_syn.bin", is + 1);
            write_f32(name, syn.data(), ntr);
            die_on(ctx, swd_preprocess(ctx, r_n, m.itmax, m.dt, data.data(), rms.data()), "swd_preprocess");
            snprintf(name, sizeof name, "./output/%dsource_seismogram_frms.bin", is + 1);
            write_f32(name, rms.data(), ntr);
        }
        snprintf(name, sizeof name, "./output/image_%s%d.bin", tag, is + 1);
        write_f32(name, img.data(), np);
        snprintf(name, sizeof name, "./output/image_sources%d.bin", is + 1);
        write_f32(name, src.data(), np);
        snprintf(name, sizeof name, "./output/fimage_%s%d.bin", tag, is + 1);
        write_f32(name, fim.data(), np);
    }
    std::vector<float> mig(np);
    die_on(ctx, swd_stack_get(ctx, 1, mig.data()), "swd_stack_get");
    write_f32(m.scatter_flag ? "./output/migration_psf.bin" : "./output/migration_pp.bin", mig.data(), np);
    printf("====================\n      THE END\n====================\n");
    swd_destroy(ctx);
    return 0;
}
