// compat_common.h -- shared pieces of the compat libraries that give the reference's
// unmodified host programs (AVSPRTM, AFor) this engine in place of their CUDA files.
//
// The reference's GPU entry points return nothing and report no errors; here any libswd
// error is printed with its message and ends the program, so a failure never leaves the
// host program writing unset result arrays.
#pragma once
#include <stdio.h>
#include <stdlib.h>
#include <vector>
#include "swd.h"
#include "ref_layouts.h"

namespace swd_compat {

// One libswd context per GPU index of the host program, created when the time step is
// known (the reference passes dt only to the propagation calls).
struct Device {
    swd_ctx *ctx = nullptr;
    swd_grid grid{};
};

struct Session {
    int nx = 0, nz = 0, pml = 0, Lc = 0, itmax = 0;
    float dx = 0.f, dz = 0.f;
    std::vector<Device> dev;
};

inline Session &session()
{
    static Session s;
    return s;
}

inline void check(swd_ctx *ctx, int rc, const char *what)
{
    if (rc != SWD_OK) {
        fprintf(stderr, "libswd compat: %s failed (%d): %s\n", what, rc, ctx ? swd_last_error(ctx) : "");
        exit(1);
    }
}

// the context of GPU i for time step dt, (re)created when the grid changes
inline swd_ctx *context(int i, float dt)
{
    Session &s = session();
    if ((int)s.dev.size() <= i) s.dev.resize(i + 1);
    Device &d = s.dev[i];
    const swd_grid g{s.nx, s.nz, s.pml, s.Lc, s.dx, s.dz, dt, s.itmax, i};
    const bool same = d.ctx && d.grid.nx == g.nx && d.grid.nz == g.nz && d.grid.pml == g.pml && d.grid.Lc == g.Lc &&
                      d.grid.dx == g.dx && d.grid.dz == g.dz && d.grid.dt == g.dt && d.grid.nt_max == g.nt_max;
    if (!same) {
        if (d.ctx) swd_destroy(d.ctx);
        d.ctx = nullptr;
        check(nullptr, swd_create(&d.ctx, &g), "swd_create");
        d.grid = g;
    }
    return d.ctx;
}

inline void record_dims(int nx, int nz, int pml, int Lc, float dx, float dz, int itmax)
{
    Session &s = session();
    s.nx = nx; s.nz = nz; s.pml = pml; s.Lc = Lc; s.dx = dx; s.dz = dz; s.itmax = itmax;
}

inline void release_all()
{
    for (Device &d : session().dev)
        if (d.ctx) swd_destroy(d.ctx);
    session().dev.clear();
}

// stencil, CPML profiles and model as the reference uploads them before every shot
inline void load_operator(swd_ctx *ctx, const float *rc, const float *vp, const float *rho, const float *a_x,
                          const float *a_x_half, const float *a_z, const float *a_z_half, const float *b_x,
                          const float *b_x_half, const float *b_z, const float *b_z_half)
{
    check(ctx, swd_set_stencil(ctx, rc), "swd_set_stencil");
    check(ctx, swd_set_cpml(ctx, a_x, a_x_half, a_z, a_z_half, b_x, b_x_half, b_z, b_z_half), "swd_set_cpml");
    check(ctx, swd_set_model(ctx, vp, rho), "swd_set_model");
}

// The reference records the traces [0, r_n/2) in the well at ix = pmlc and the rest at
// ix = ntx-pmlc-1, at the depths r_iz (acoustic_HLVSPRTMLc.cu:180-197).
struct ShotCells {
    std::vector<int> rix, riz;
    swd_shot shot{};
};

inline void shot_cells(const RefSource &s, int ntx, int pmlc, int nt, ShotCells &c)
{
    c.rix.resize(s.r_n);
    c.riz.assign(s.r_iz, s.r_iz + s.r_n);
    for (int t = 0; t < s.r_n; t++) c.rix[t] = t < s.r_n / 2 ? pmlc : ntx - pmlc - 1;
    c.shot = swd_shot{s.s_ix, s.s_iz, nt, s.r_n, c.rix.data(), c.riz.data()};
}

}  // namespace swd_compat
