// decon2d_mine -- drop-in windowed wavenumber PSF deconvolution (the reference's
// kkdecon_acoustic/decon2d_mine, kk_decon_interp_psf_minewindow.cpp:17-785) on libswd.
//
// Run from the kkdecon_acoustic/ directory: reads ./parameter.txt (window sizes, epsilon and
// the file names), the true and migration velocity models, the RTM image and the PSF image;
// writes the reference's diagnostics and the deconvolved image (the decon file named in
// parameter.txt) plus migration_coef.{bin,txt}, start.flag and end.flag into ./output/.
// All windows run as one batched launch on the GPU (swd_decon).
// Extensions (parameter.txt lines `swd.key = value`): device, psf_interp (1: bilinear blend of
// the lattice PSFs around each window, a project option), fft_nx / fft_nz (zero-padded
// FFT size instead of filterwin + psfwin - 1), iterative (1: the regularised deconvolution with
// the parameter file's own L1 coefficient reg_eps, L2 coefficient and iteration count, which
// the reference reads in part but never uses; reg_l1 / reg_l2 / iters override them).
#include <math.h>
#include "common.h"

using namespace drv;

int main(int, char **)
{
    int nx, nz, psfwinx, psfwinz, filterwinx, filterwinz, snapwinx, snapwinz, shift_flag;
    float epsilon, reg_eps, reg_l2_file = 0.0f;
    int itn_file = 0;
    char vp_file[150], vp0_file[150], rho_file[150], migreal_file[150], migpsf_file[150], decon_file[150], ipsf_file[150];
    {
        ParamReader r("parameter.txt");
        if (!r.fp) {
            printf("Cannot open the parameters file!\n");
            return 1;
        }
        r.get(&nx); r.get(&nz); r.get(&psfwinx); r.get(&psfwinz); r.get(&filterwinx); r.get(&filterwinz);
        r.get(&snapwinx); r.get(&snapwinz); r.get(&epsilon); r.get(vp_file); r.get(vp0_file); r.get(rho_file);
        r.get(migreal_file); r.get(migpsf_file); r.get(decon_file); r.get(ipsf_file); r.get(&shift_flag);
        r.get(&reg_eps);
        if (!r.ok) {
            printf("parameter.txt is incomplete\n");
            return 1;
        }
        // the two entries after reg_eps (L2 coefficient, iteration count) are optional
        r.get(&reg_l2_file);
        r.get(&itn_file);
        if (!r.ok) {
            reg_l2_file = 0.0f;
            itn_file = 0;
        }
    }
    auto ext = extensions("parameter.txt");
    const int device = ext_int(ext, "device", 0);
    printf("Number of MPI thread is 1\n");
    if (psfwinx % 2 == 0 || psfwinz % 2 == 0 || filterwinx % 2 == 0 || filterwinz % 2 == 0) {
        printf("All the PSF and Fitler Windows Should Be Odd Number !\n");
        return 0;
    }
    const int fullwx = filterwinx + psfwinx - 1, fullwz = filterwinz + psfwinz - 1;
    const int outwinx = 2 * (psfwinx / 10) + 2 * snapwinx + 1, outwinz = 2 * (psfwinz / 10) + 2 * snapwinz + 1;
    const int stepwinx = outwinx - snapwinx, stepwinz = outwinz - snapwinz;
    if (filterwinx < psfwinx || filterwinz < psfwinz) {
        printf("Filter length < psf's window length !\nBreak up!\n");
        return 0;
    }
    if (filterwinx < outwinx || filterwinz < outwinz) {
        printf("Filter length < output window length !\nBreak up!\n");
        return 0;
    }
    printf("Full window size -- (%d,  %d)\nFilter window size -- (%d,  %d)\nOutput size -- (%d,  %d)\n"
           "Step window size -- (%d,  %d)\n", fullwz, fullwx, filterwinz, filterwinx, outwinz, outwinx, stepwinx, stepwinz);

    const size_t np = (size_t)nx * nz;
    std::vector<float> vp_old(np), vp(np), mn(np, 0.0f), rho(np, 1000.0f), migreal(np), migpsf(np);
    if (!read_f32(vp_file, vp_old.data(), np)) return 1;
    write_f32("./output/acc_vp.bin", vp_old.data(), np);
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 1; iz < nz; iz++) {
            const size_t ip = (size_t)ix * nz + iz;
            mn[ip] = (vp_old[ip] - vp_old[ip - 1]) / (vp_old[ip] + vp_old[ip - 1]);
        }
    write_f32("./output/true_vertical_ref.bin", mn.data(), np);
    if (!read_f32(vp0_file, vp.data(), np)) return 1;
    write_f32("./output/ini_vp.bin", vp.data(), np);
    for (size_t ip = 0; ip < np; ip++) mn[ip] = (vp_old[ip] - vp[ip]) / vp_old[ip];
    write_f32("./output/acc_ref.bin", mn.data(), np);
    write_f32("./output/acc_rho.bin", rho.data(), np);
    printf("The true model is done\n");
    if (!read_f32(migreal_file, migreal.data(), np)) return 1;
    if (!read_f32(migpsf_file, migpsf.data(), np)) return 1;
    float vp_max = 0.0;
    for (size_t ip = 0; ip < np; ip++)
        if (vp[ip] >= vp_max) vp_max = vp[ip];
    printf("vp_max = %f\n", vp_max);

    swd_decon_params p{nx, nz, psfwinx, psfwinz, filterwinx, filterwinz, snapwinx, snapwinz, epsilon,
                       ext_int(ext, "fft_nx", 0), ext_int(ext, "fft_nz", 0), ext_int(ext, "psf_interp", 0)};
    if (ext_int(ext, "iterative", 0)) {
        p.iters = ext_int(ext, "iters", itn_file);
        p.reg_l1 = ext_float(ext, "reg_l1", reg_eps);
        p.reg_l2 = ext_float(ext, "reg_l2", reg_l2_file);
        printf("Iterative regularised deconvolution: %d iterations, L1 %g, L2 %g\n", p.iters, p.reg_l1, p.reg_l2);
    }
    int windows = 0, fx = 0, fz = 0;
    if (swd_decon_geometry(&p, &windows, &fx, &fz) != SWD_OK) {
        printf("Invalid deconvolution window geometry\n");
        return 1;
    }
    const int stepnumx = (int)ceil(1.0 * (nx + fullwx) / stepwinx) + 1, stepnumz = (int)ceil(1.0 * (nz + fullwz) / stepwinz) + 1;
    printf("The expaned nxp == %d, nzp == %d\n", stepnumx * stepwinx, stepnumz * stepwinz);
    write_f32("./output/migration_psf.bin", migpsf.data(), np);

    // output taper and PSF window weights (:355-408)
    std::vector<float> coefr((size_t)outwinx * outwinz), coefp((size_t)psfwinx * psfwinz, 1.0f);
    const double PI = 3.1415926;
    for (int ix = 0; ix < outwinx; ix++)
        for (int iz = 0; iz < outwinz; iz++) {
            float cx, cz;
            if (ix <= snapwinx - 1) cx = 0.5000 - 0.5 * cos(PI * ix / (snapwinx - 1));
            else if (ix >= outwinx - snapwinx) cx = 0.5000 + 0.5 * cos(PI * (ix - outwinx + snapwinx) / (snapwinx - 1));
            else cx = 1.0;
            if (iz <= snapwinz - 1) cz = 0.5000 - 0.5 * cos(PI * iz / (snapwinz - 1));
            else if (iz >= outwinz - snapwinz) cz = 0.5000 + 0.5 * cos(PI * (iz - outwinz + snapwinz) / (snapwinz - 1));
            else cz = 1.0;
            coefr[(size_t)ix * outwinz + iz] = cx * cz;
        }
    write_f32("./output/coefr.bin", coefr.data(), coefr.size());
    write_f32("./output/psfcoef.bin", coefp.data(), coefp.size());
    // the PSF lattice windows tile the whole image, so the "filtered PSF" diagnostic of
    // :410-457 is the PSF image itself with unit weights
    std::vector<float> ones(np, 1.0f);
    write_f32("./output/migration_psf_filt.bin", migpsf.data(), np);
    write_f32("./output/migration_coefp.bin", ones.data(), np);
    printf("=========================================\n      =============================\n"
           "      Calculate the Deconvolution \n      with Point Spread Functions !\n"
           "  -------------------------------------\n");
    if (FILE *f = fopen("./output/start.flag", "w")) fclose(f);
    printf("Caculate the Deconvolution with the Wavenumber-domain PSFs ! (%d windows of %d x %d)\n", windows, fx, fz);

    swd_grid g{nx, nz, 0, 1, 1.0f, 1.0f, 1.0f, 2, device};
    swd_ctx *ctx = nullptr;
    if (nx < 3 || nz < 3 || swd_create(&ctx, &g) != SWD_OK) {
        fprintf(stderr, "swd_create failed: no usable CUDA device\n");
        return 1;
    }
    std::vector<float> dec(np), coef(np);
    die_on(ctx, swd_decon(ctx, &p, migreal.data(), migpsf.data(), dec.data(), coef.data()), "swd_decon");
    printf("\n");
    if (FILE *f = fopen("./output/end.flag", "w")) fclose(f);
    write_f32("./output/migration_pp.bin", migreal.data(), np);
    write_f32("./output/migration_coef.bin", coef.data(), np);
    if (FILE *f = fopen("./output/migration_coef.txt", "w")) {
        for (int iz = 0; iz < nz; iz++) {
            for (int ix = 0; ix < nx; ix++) fprintf(f, "%f  ", coef[(size_t)ix * nz + iz]);
            fprintf(f, "\r\t\n");
        }
        fclose(f);
    }
    write_f32(decon_file, dec.data(), np);
    printf("            Deconvolution END!     \n      =============================\n"
           "=========================================\n");
    swd_destroy(ctx);
    (void)shift_flag;
    (void)reg_eps;
    (void)rho_file;
    (void)ipsf_file;
    return 0;
}
