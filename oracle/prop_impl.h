/*
 * oracle/prop_impl.h -- propagation, imaging and kz-split loops of the reference,
 * restated for the CPU oracle.  TEST INFRASTRUCTURE.  Included twice by swd_oracle.c
 * with T = float / SFX = f32 (the FP32 oracle and OpenMP CPU baseline) and
 * T = double / SFX = f64 (the FP64 oracle).
 *
 * Expressions are written in the reference's order so the float build rounds like the
 * reference kernels (the reference's nvcc build additionally contracts some mul+add
 * pairs into FMAs; that difference is the expected ~1e-6 FP32 noise).
 */
#define ORC_CAT_(a, b) a##_##b
#define ORC_CAT(a, b) ORC_CAT_(a, b)
#define FN(name) ORC_CAT(name, SFX)

typedef struct {
    int ntx, ntz, Lc, pmlc, nt;
    T dt;
    float dx, dz;
    T rc[16];
    T *vp, *rho, *ax, *axh, *az, *azh, *bx, *bxh, *bz, *bzh;
} FN(orc_mdl);

static T *FN(cvt)(const float *src, size_t n)
{
    T *d = (T *)malloc(sizeof(T) * (n ? n : 1));
    for (size_t i = 0; i < n; i++) d[i] = (T)src[i];
    return d;
}

static void FN(mdl_init)(FN(orc_mdl) *M, const orc_model *m)
{
    size_t ntp = (size_t)m->ntx * m->ntz;
    M->ntx = m->ntx; M->ntz = m->ntz; M->Lc = m->Lc; M->pmlc = m->pmlc; M->nt = m->nt;
    M->dt = (T)m->dt; M->dx = m->dx; M->dz = m->dz;
    for (int i = 0; i < m->Lc && i < 16; i++) M->rc[i] = (T)m->rc[i];
    M->vp = FN(cvt)(m->vp, ntp); M->rho = FN(cvt)(m->rho, ntp);
    M->ax = FN(cvt)(m->a_x, m->ntx); M->axh = FN(cvt)(m->a_x_half, m->ntx);
    M->az = FN(cvt)(m->a_z, m->ntz); M->azh = FN(cvt)(m->a_z_half, m->ntz);
    M->bx = FN(cvt)(m->b_x, m->ntx); M->bxh = FN(cvt)(m->b_x_half, m->ntx);
    M->bz = FN(cvt)(m->b_z, m->ntz); M->bzh = FN(cvt)(m->b_z_half, m->ntz);
}

static void FN(mdl_free)(FN(orc_mdl) *M)
{
    free(M->vp); free(M->rho); free(M->ax); free(M->axh); free(M->az); free(M->azh);
    free(M->bx); free(M->bxh); free(M->bz); free(M->bzh);
}

typedef struct { T *p, *vx, *vz, *ppx, *ppz, *pvx, *pvz; } FN(orc_fld);

static void FN(fld_alloc)(FN(orc_fld) *f, size_t ntp)
{
    f->p = (T *)calloc(ntp, sizeof(T)); f->vx = (T *)calloc(ntp, sizeof(T));
    f->vz = (T *)calloc(ntp, sizeof(T)); f->ppx = (T *)calloc(ntp, sizeof(T));
    f->ppz = (T *)calloc(ntp, sizeof(T)); f->pvx = (T *)calloc(ntp, sizeof(T));
    f->pvz = (T *)calloc(ntp, sizeof(T));
}

static void FN(fld_free)(FN(orc_fld) *f)
{
    free(f->p); free(f->vx); free(f->vz); free(f->ppx); free(f->ppz); free(f->pvx); free(f->pvz);
}

/* vx += dt/rho_x * (dp/dx + phi_p_x), with CPML memory.  acoustic_HLVSPRTMLc.cu:24-69
 * (guard iz in [Lc, ntz-Lc], ix in [Lc-1, ntx-Lc-1]); the receiver back-propagation uses
 * the same body with -dx and the wider guard of :623-667. */
static void FN(upd_vx)(const FN(orc_mdl) *M, FN(orc_fld) *f, float dx, int iz0, int iz1, int ix0, int ix1)
{
    const int ntz = M->ntz, Lc = M->Lc;
    const T odx = (T)(1.0 / (double)dx);
    const T dt = M->dt;
#pragma omp parallel for schedule(static)
    for (int ix = ix0; ix <= ix1; ix++)
        for (int iz = iz0; iz <= iz1; iz++) {
            size_t ip = (size_t)ix * ntz + iz;
            T d = 0.0;
            for (int ic = 0; ic < Lc; ic++) d += M->rc[ic] * (f->p[ip + (ic + 1) * ntz] - f->p[ip - ic * ntz]) * odx;
            f->ppx[ip] = M->bxh[ix] * f->ppx[ip] + M->axh[ix] * d;
            T orho = (T)(1 / (0.5 * (M->rho[ip] + M->rho[ip + 1 * ntz])));
            f->vx[ip] = dt * orho * (d + f->ppx[ip]) + f->vx[ip];
        }
}

/* vz analogue.  acoustic_HLVSPRTMLc.cu:72-118 (guard iz in [Lc-1, ntz-Lc-1], ix in
 * [Lc, ntx-Lc]); receiver variant :670-715. */
static void FN(upd_vz)(const FN(orc_mdl) *M, FN(orc_fld) *f, float dz, int iz0, int iz1, int ix0, int ix1)
{
    const int ntz = M->ntz, Lc = M->Lc;
    const T odz = (T)(1.0 / (double)dz);
    const T dt = M->dt;
#pragma omp parallel for schedule(static)
    for (int ix = ix0; ix <= ix1; ix++)
        for (int iz = iz0; iz <= iz1; iz++) {
            size_t ip = (size_t)ix * ntz + iz;
            T d = 0.0;
            for (int ic = 0; ic < Lc; ic++) d += M->rc[ic] * (f->p[ip + (ic + 1)] - f->p[ip - ic]) * odz;
            f->ppz[ip] = M->bzh[iz] * f->ppz[ip] + M->azh[iz] * d;
            T orho = (T)(1 / (0.5 * (M->rho[ip] + M->rho[ip + 1])));
            f->vz[ip] = dt * orho * (d + f->ppz[ip]) + f->vz[ip];
        }
}

/* p += dt*rho*vp^2*(dvx/dx + phi_vx_x + dvz/dz + phi_vz_z).  acoustic_HLVSPRTMLc.cu:121-173
 * (guard iz in [Lc, ntz-Lc], ix in [Lc, ntx-Lc]); receiver variant :717-762.
 * Born extensions (project operator): s_out receives the p-update sum S per updated cell;
 * with dk, p additionally receives dt*dk*s_in (the scattered field's secondary source). */
static void FN(upd_p_born)(const FN(orc_mdl) *M, FN(orc_fld) *f, float dx, float dz, T *s_out, const T *dk,
                           const T *s_in)
{
    const int ntz = M->ntz, ntx = M->ntx, Lc = M->Lc;
    const T odx = (T)(1.0 / (double)dx), odz = (T)(1.0 / (double)dz);
    const T dt = M->dt;
#pragma omp parallel for schedule(static)
    for (int ix = Lc; ix <= ntx - Lc; ix++)
        for (int iz = Lc; iz <= ntz - Lc; iz++) {
            size_t ip = (size_t)ix * ntz + iz;
            T dvx = 0.0, dvz = 0.0;
            for (int ic = 0; ic < Lc; ic++) {
                dvx += M->rc[ic] * (f->vx[ip + ic * ntz] - f->vx[ip - (ic + 1) * ntz]) * odx;
                dvz += M->rc[ic] * (f->vz[ip + ic] - f->vz[ip - (ic + 1)]) * odz;
            }
            f->pvx[ip] = M->bx[ix] * f->pvx[ip] + M->ax[ix] * dvx;
            f->pvz[ip] = M->bz[iz] * f->pvz[ip] + M->az[iz] * dvz;
            const T S = dvx + f->pvx[ip] + dvz + f->pvz[ip];
            if (s_out) s_out[ip] = S;
            f->p[ip] = dt * M->rho[ip] * M->vp[ip] * M->vp[ip] * S + f->p[ip];
            if (dk) f->p[ip] += dt * dk[ip] * s_in[ip];
        }
}

static void FN(upd_p)(const FN(orc_mdl) *M, FN(orc_fld) *f, float dx, float dz)
{
    const int ntz = M->ntz, ntx = M->ntx, Lc = M->Lc;
    const T odx = (T)(1.0 / (double)dx), odz = (T)(1.0 / (double)dz);
    const T dt = M->dt;
#pragma omp parallel for schedule(static)
    for (int ix = Lc; ix <= ntx - Lc; ix++)
        for (int iz = Lc; iz <= ntz - Lc; iz++) {
            size_t ip = (size_t)ix * ntz + iz;
            T dvx = 0.0, dvz = 0.0;
            for (int ic = 0; ic < Lc; ic++) {
                dvx += M->rc[ic] * (f->vx[ip + ic * ntz] - f->vx[ip - (ic + 1) * ntz]) * odx;
                dvz += M->rc[ic] * (f->vz[ip + ic] - f->vz[ip - (ic + 1)]) * odz;
            }
            f->pvx[ip] = M->bx[ix] * f->pvx[ip] + M->ax[ix] * dvx;
            f->pvz[ip] = M->bz[iz] * f->pvz[ip] + M->az[iz] * dvz;
            f->p[ip] = dt * M->rho[ip] * M->vp[ip] * M->vp[ip] * (dvx + f->pvx[ip] + dvz + f->pvz[ip]) + f->p[ip];
        }
}

/* boundary strips of p, saved (dir=0) or restored (dir=1).  Save:
 * acoustic_HLVSPRTMLc.cu:199-219; restore: fdtd_2d_GPU_kernel_borders_backward :575-620.
 * The per-step layout here is [top Lc x nx][bottom Lc x nx][left Lc x (nz-2Lc)][right]. */
static void FN(strips_io)(const FN(orc_mdl) *M, T *p, T *s, int dir)
{
    const int ntz = M->ntz, ntx = M->ntx, Lc = M->Lc, pmlc = M->pmlc;
    const int nx = ntx - 2 * pmlc, nz = ntz - 2 * pmlc, nzs = nz - 2 * Lc;
    size_t k = 0;
    for (int iz = pmlc; iz <= pmlc + Lc - 1; iz++)
        for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++, k++) {
            size_t ip = (size_t)ix * ntz + iz;
            if (dir) p[ip] = s[k]; else s[k] = p[ip];
        }
    for (int iz = ntz - pmlc - Lc; iz <= ntz - pmlc - 1; iz++)
        for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++, k++) {
            size_t ip = (size_t)ix * ntz + iz;
            if (dir) p[ip] = s[k]; else s[k] = p[ip];
        }
    for (int ix = pmlc; ix <= pmlc + Lc - 1; ix++)
        for (int iz = pmlc + Lc; iz <= ntz - pmlc - Lc - 1; iz++, k++) {
            size_t ip = (size_t)ix * ntz + iz;
            if (dir) p[ip] = s[k]; else s[k] = p[ip];
        }
    for (int ix = ntx - pmlc - Lc; ix <= ntx - pmlc - 1; ix++)
        for (int iz = pmlc + Lc; iz <= ntz - pmlc - Lc - 1; iz++, k++) {
            size_t ip = (size_t)ix * ntz + iz;
            if (dir) p[ip] = s[k]; else s[k] = p[ip];
        }
    (void)nx; (void)nzs;
}

void FN(orc_forward)(const orc_model *m, const orc_geom *g, const float *rick,
                     const float *hrick, T *seis, T *strips, T *final_state,
                     int ncol, const int *col_ix, T *cols)
{
    FN(orc_mdl) M;
    FN(mdl_init)(&M, m);
    const int ntx = M.ntx, ntz = M.ntz, Lc = M.Lc, nt = M.nt;
    const size_t ntp = (size_t)ntx * ntz;
    const int slen = orc_strip_len(m);
    FN(orc_fld) f, h;
    FN(fld_alloc)(&f, ntp);
    if (hrick) FN(fld_alloc)(&h, ntp);
    const size_t src = (size_t)g->s_ix * ntz + g->s_iz;
    for (int it = 0; it < nt; it++) {
        /* vx, vz, p, source, record -- the launch order of acoustic_HLVSPRTMLc.cu:320-354 */
        FN(upd_vx)(&M, &f, m->dx, Lc, ntz - Lc, Lc - 1, ntx - Lc - 1);
        FN(upd_vz)(&M, &f, m->dz, Lc - 1, ntz - Lc - 1, Lc, ntx - Lc);
        FN(upd_p)(&M, &f, m->dx, m->dz);
        f.p[src] += rick[it];
        if (hrick) {   /* Hilbert twin, forward/...HLForLc.cu:724-760 */
            FN(upd_vx)(&M, &h, m->dx, Lc, ntz - Lc, Lc - 1, ntx - Lc - 1);
            FN(upd_vz)(&M, &h, m->dz, Lc - 1, ntz - Lc - 1, Lc, ntx - Lc);
            FN(upd_p)(&M, &h, m->dx, m->dz);
            h.p[src] += hrick[it];
        }
        if (seis)
            for (int r = 0; r < g->nrec; r++)
                seis[(size_t)r * nt + it] = f.p[(size_t)g->r_ix[r] * ntz + g->r_iz[r]];
        if (strips) FN(strips_io)(&M, f.p, strips + (size_t)it * slen, 0);
        if (cols)
            for (int c = 0; c < ncol; c++) {
                T *dst = cols + ((size_t)c * nt + it) * ntz * 2;
                const size_t base = (size_t)col_ix[c] * ntz;
                for (int iz = 0; iz < ntz; iz++) {
                    dst[2 * iz] = f.p[base + iz];
                    dst[2 * iz + 1] = hrick ? h.p[base + iz] : (T)0;
                }
            }
    }
    if (final_state) {
        memcpy(final_state, f.vx, sizeof(T) * ntp);
        memcpy(final_state + ntp, f.vz, sizeof(T) * ntp);
        memcpy(final_state + 2 * ntp, f.p, sizeof(T) * ntp);
    }
    FN(fld_free)(&f);
    if (hrick) FN(fld_free)(&h);
    FN(mdl_free)(&M);
}

void FN(orc_kzsep)(int ntz, int nfftz, int nt, int ncol, const T *cols,
                   const float *coef, int nrec, const int *rec_col, const int *r_iz,
                   T *up, T *down)
{
    const int halfz = nfftz / 2;   /* ceilf(nfftz/2.0) for the power-of-two nfftz */
#pragma omp parallel
    {
        double *F = (double *)malloc(sizeof(double) * 2 * nfftz);
        double *U = (double *)malloc(sizeof(double) * 2 * nfftz);
        double *D = (double *)malloc(sizeof(double) * 2 * nfftz);
#pragma omp for schedule(static) collapse(2)
        for (int c = 0; c < ncol; c++)
            for (int it = 0; it < nt; it++) {
                const T *src = cols + ((size_t)c * nt + it) * ntz * 2;
                memset(F, 0, sizeof(double) * 2 * nfftz);
                for (int iz = 0; iz < ntz; iz++) { F[2 * iz] = src[2 * iz]; F[2 * iz + 1] = src[2 * iz + 1]; }
                orc_fft(nfftz, F, -1);
                for (int k = 0; k < nfftz; k++) {
                    double re = F[2 * k] * coef[k], im = F[2 * k + 1] * coef[k];
                    if (k <= halfz) { U[2 * k] = re; U[2 * k + 1] = im; D[2 * k] = 0; D[2 * k + 1] = 0; }
                    else { D[2 * k] = re; D[2 * k + 1] = im; U[2 * k] = 0; U[2 * k + 1] = 0; }
                }
                orc_fft(nfftz, U, +1);
                orc_fft(nfftz, D, +1);
                for (int r = 0; r < nrec; r++)
                    if (rec_col[r] == c) {
                        up[(size_t)r * nt + it] = (T)U[2 * r_iz[r]];
                        down[(size_t)r * nt + it] = (T)D[2 * r_iz[r]];
                    }
            }
        free(F); free(U); free(D);
    }
}

void FN(orc_preprocess)(int nrec, int nt, float dtf, const float *d, T *rms)
{
    const T dt = (T)dtf;
    T *frms = FN(cvt)(d, (size_t)nrec * nt);
    for (int ix = 0; ix < nrec; ix++) {
        T tmp = 0.0;
        for (int it = 0; it < nt; it++) {
            size_t ip = (size_t)ix * nt + it;
            tmp += frms[ip] * dt;
            frms[ip] = tmp;
        }
    }
    for (int ix = 0; ix < nrec; ix++) {
        T tmp = 0.0;
        for (int it = 0; it < nt; it++) {
            size_t ip = (size_t)ix * nt + it;
            tmp += frms[ip] * dt;
            rms[ip] = -tmp;
        }
    }
    free(frms);
}

/* Angle-domain common-image gathers of one backward step (sum_image_GPU_kernel_imageCIG,
 * acoustic_HLVSPRTMLc.cu:819-905; the reference never launches it): Poynting vectors -p*v of
 * the source and receiver wavefields, their dot product and magnitude product kept over the
 * last delt steps, the reflection half-angle ftheta = 0.5*acos(dot/mag) in degrees, and
 * p_s*p_r spread over the five 1-degree bins around it with weights exp(-ii^2/18); bins < 2 and
 * >= thetan are dropped, as are cells whose angle is undefined (zero magnitude).  Float
 * arithmetic with the reference's mixed float/double expressions. */
static void FN(cig_step)(const FN(orc_mdl) *M, const FN(orc_fld) *s, const FN(orc_fld) *r, int it, int nt, int thetan,
                         int delt, float *ring, float *cig)
{
    const int ntx = M->ntx, ntz = M->ntz, pmlc = M->pmlc;
    const size_t ntp = (size_t)ntx * ntz;
    for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++)
        for (int iz = pmlc; iz <= ntz - pmlc - 1; iz++) {
            const size_t ip = (size_t)ix * ntz + iz;
            const float ps = (float)s->p[ip], pr = (float)r->p[ip];
            const float fx = -ps * (float)s->vx[ip], fz = -ps * (float)s->vz[ip];
            const float fxr = -pr * (float)r->vx[ip], fzr = -pr * (float)r->vz[ip];
            ring[(size_t)(it % delt) * 2 * ntp + ip] = fx * fxr + fz * fzr;
            ring[((size_t)(it % delt) * 2 + 1) * ntp + ip] = sqrtf(fx * fx + fz * fz) * sqrtf(fxr * fxr + fzr * fzr);
            if (nt - 2 - it + 1 < delt) continue;
            float pre = 0.0f, pst = 0.0f;
            for (int ii = 0; ii < delt; ii++) {
                pre += ring[(size_t)ii * 2 * ntp + ip];
                pst += ring[((size_t)ii * 2 + 1) * ntp + ip];
            }
            const float tht = pre / pst;
            const float ftheta = (float)(0.5 * acosf(tht) * 180.0 / 3.1415926);
            if (!(ftheta == ftheta)) continue;   /* undefined angle */
            for (int ii = -2; ii <= 2; ii++) {
                const int itheta = (int)ceilf((float)(ftheta + ii - 0.5));
                const float betaf = (float)(1.0 * ii * ii / (2.0 * 9.0));
                if (itheta >= 2 && itheta < thetan) cig[ip * thetan + itheta] += ps * pr * expf(-betaf);
            }
        }
}

void FN(orc_rtm_backward)(const orc_model *m, const orc_geom *g, const float *rick,
                          const T *rms, const T *strips, const T *final_state,
                          T *img, T *illum_s, T *illum_r, int thetan, int delt, float *cig)
{
    FN(orc_mdl) M;
    FN(mdl_init)(&M, m);
    const int ntx = M.ntx, ntz = M.ntz, Lc = M.Lc, nt = M.nt, pmlc = M.pmlc;
    const size_t ntp = (size_t)ntx * ntz;
    const int slen = orc_strip_len(m);
    FN(orc_fld) s, r;
    FN(fld_alloc)(&s, ntp);
    FN(fld_alloc)(&r, ntp);
    T *dpdt = (T *)calloc(ntp, sizeof(T));
    memcpy(s.vx, final_state, sizeof(T) * ntp);
    memcpy(s.vz, final_state + ntp, sizeof(T) * ntp);
    memcpy(s.p, final_state + 2 * ntp, sizeof(T) * ntp);
    memset(img, 0, sizeof(T) * ntp);
    memset(illum_s, 0, sizeof(T) * ntp);
    if (illum_r) memset(illum_r, 0, sizeof(T) * ntp);
    const size_t src = (size_t)g->s_ix * ntz + g->s_iz;
    const T odx = (T)(1.0 / (double)m->dx), odz = (T)(1.0 / (double)m->dz);
    const T mdt = -M.dt;
    float *ring = cig ? (float *)calloc((size_t)2 * delt * ntp, sizeof(float)) : NULL;
    if (cig) memset(cig, 0, sizeof(float) * ntp * thetan);
    for (int it = nt - 2; it >= 0; it--) {
        /* source wavefield: p (interior, -dt) and dp_dt -- fdtd_2d_GPU_kernel_p_backward :434-485 */
#pragma omp parallel for schedule(static)
        for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++)
            for (int iz = pmlc; iz <= ntz - pmlc - 1; iz++) {
                size_t ip = (size_t)ix * ntz + iz;
                T dvx = 0.0, dvz = 0.0;
                for (int ic = 0; ic < Lc; ic++) {
                    dvx += M.rc[ic] * (s.vx[ip + ic * ntz] - s.vx[ip - (ic + 1) * ntz]) * odx;
                    dvz += M.rc[ic] * (s.vz[ip + ic] - s.vz[ip - (ic + 1)]) * odz;
                }
                s.p[ip] = mdt * M.rho[ip] * M.vp[ip] * M.vp[ip] * (dvx + dvz) + s.p[ip];
                dpdt[ip] = M.rho[ip] * M.vp[ip] * M.vp[ip] * (dvx + dvz);
            }
        s.p[src] -= rick[it + 1];
        /* strip overwrite -- :575-620 */
        FN(strips_io)(&M, s.p, (T *)strips + (size_t)it * slen, 1);
        /* vx, vz (interior, -dt) -- :488-573 */
#pragma omp parallel for schedule(static)
        for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++)
            for (int iz = pmlc; iz <= ntz - pmlc - 1; iz++) {
                size_t ip = (size_t)ix * ntz + iz;
                T d = 0.0;
                for (int ic = 0; ic < Lc; ic++) d += M.rc[ic] * (s.p[ip + (ic + 1) * ntz] - s.p[ip - ic * ntz]) * odx;
                T orho = (T)(1 / (0.5 * (M.rho[ip] + M.rho[ip + 1 * ntz])));
                s.vx[ip] = mdt * orho * d + s.vx[ip];
            }
#pragma omp parallel for schedule(static)
        for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++)
            for (int iz = pmlc; iz <= ntz - pmlc - 1; iz++) {
                size_t ip = (size_t)ix * ntz + iz;
                T d = 0.0;
                for (int ic = 0; ic < Lc; ic++) d += M.rc[ic] * (s.p[ip + (ic + 1)] - s.p[ip - ic]) * odz;
                T orho = (T)(1 / (0.5 * (M.rho[ip] + M.rho[ip + 1])));
                s.vz[ip] = mdt * orho * d + s.vz[ip];
            }
        /* receiver wavefield with -dx,-dz and hard injection -- :623-782, launches :1111-1140 */
        FN(upd_vx)(&M, &r, -m->dx, 0, ntz - 1, Lc - 1, ntx - Lc - 1);
        FN(upd_vz)(&M, &r, -m->dz, Lc - 1, ntz - Lc - 1, 0, ntx - 1);
        FN(upd_p)(&M, &r, -m->dx, -m->dz);
        for (int k = 0; k < g->nrec; k++)
            r.p[(size_t)g->r_ix[k] * ntz + g->r_iz[k]] = rms[(size_t)k * nt + it];
        /* imaging condition -- sum_image_GPU_kernel_image :785-817 */
#pragma omp parallel for schedule(static)
        for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++)
            for (int iz = pmlc; iz <= ntz - pmlc - 1; iz++) {
                size_t ip = (size_t)ix * ntz + iz;
                img[ip] += dpdt[ip] * r.p[ip];
                illum_s[ip] += dpdt[ip] * dpdt[ip];
                if (illum_r) illum_r[ip] += r.p[ip] * r.p[ip];
            }
        if (cig) FN(cig_step)(&M, &s, &r, it, nt, thetan, delt, ring, cig);
    }
    free(ring);
    free(dpdt);
    FN(fld_free)(&s);
    FN(fld_free)(&r);
    FN(mdl_free)(&M);
}

void FN(orc_rtm_post)(const orc_model *m, const T *img, const T *illum_s, T *img_norm, T *fimage)
{
    const int ntx = m->ntx, ntz = m->ntz, pmlc = m->pmlc;
    const int nz = ntz - 2 * pmlc;
    const size_t ntp = (size_t)ntx * ntz;
    const T dx = (T)m->dx, dz = (T)m->dz;
    T remax = 0;
    for (size_t ip = 0; ip < ntp; ip++) {
        T a = illum_s[ip] < 0 ? -illum_s[ip] : illum_s[ip];
        if (remax < a) remax = a;
    }
    for (size_t ip = 0; ip < ntp; ip++) img_norm[ip] = (T)(img[ip] / (illum_s[ip] + 1.0e-3 * remax));
    for (int iz = pmlc; iz <= ntz - pmlc - 1; iz++)
        for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++) {
            size_t ip = (size_t)ix * ntz + iz;
            size_t ipp = (size_t)(ix - pmlc) * nz + iz - pmlc;
            const T *I = img_norm;
            T v = (T)m->vp[ip];
            fimage[ipp] = (T)(-((I[ip + ntz] - 2.0 * I[ip] + I[ip - ntz]) / (dx * dx) +
                                (I[ip + 1] - 2.0 * I[ip] + I[ip - 1]) / (dz * dz)) * v * v);
        }
}


/* ---------------- Born modelling and its adjoint (project operators) ----------------
 * The forward step above is linear in the state (p, vx, vz and the four CPML memories) and
 * in kappa = rho*vp^2.  Born: the scattered field b steps beside the background f and gets
 * dt*dkappa*S0 after its p update; the receivers record b.p after each step.  The adjoint
 * below is the transpose written as scatters of each forward loop body, applied in reverse
 * order (P^T then V^T per step), so its correctness rests on the dot-product identity, not
 * on matching the device's gathers. */
void FN(orc_born)(const orc_model *m, const orc_geom *g, const float *rick, const float *dkappa, T *dseis)
{
    FN(orc_mdl) M;
    FN(mdl_init)(&M, m);
    const int ntx = M.ntx, ntz = M.ntz, Lc = M.Lc, nt = M.nt;
    const size_t ntp = (size_t)ntx * ntz;
    T *dk = FN(cvt)(dkappa, ntp);
    T *s0 = (T *)calloc(ntp, sizeof(T));
    FN(orc_fld) f, b;
    FN(fld_alloc)(&f, ntp);
    FN(fld_alloc)(&b, ntp);
    const size_t src = (size_t)g->s_ix * ntz + g->s_iz;
    for (int it = 0; it < nt; it++) {
        FN(upd_vx)(&M, &f, m->dx, Lc, ntz - Lc, Lc - 1, ntx - Lc - 1);
        FN(upd_vz)(&M, &f, m->dz, Lc - 1, ntz - Lc - 1, Lc, ntx - Lc);
        FN(upd_p_born)(&M, &f, m->dx, m->dz, s0, NULL, NULL);
        f.p[src] += rick[it];
        FN(upd_vx)(&M, &b, m->dx, Lc, ntz - Lc, Lc - 1, ntx - Lc - 1);
        FN(upd_vz)(&M, &b, m->dz, Lc - 1, ntz - Lc - 1, Lc, ntx - Lc);
        FN(upd_p_born)(&M, &b, m->dx, m->dz, NULL, dk, s0);
        for (int r = 0; r < g->nrec; r++) dseis[(size_t)r * nt + it] = b.p[(size_t)g->r_ix[r] * ntz + g->r_iz[r]];
    }
    FN(fld_free)(&f);
    FN(fld_free)(&b);
    free(dk);
    free(s0);
    FN(mdl_free)(&M);
}

void FN(orc_born_adjoint)(const orc_model *m, const orc_geom *g, const float *rick, const float *resid, T *grad)
{
    FN(orc_mdl) M;
    FN(mdl_init)(&M, m);
    const int ntx = M.ntx, ntz = M.ntz, Lc = M.Lc, nt = M.nt;
    const size_t ntp = (size_t)ntx * ntz;
    const T odx = (T)(1.0 / (double)m->dx), odz = (T)(1.0 / (double)m->dz), dt = M.dt;
    /* background pass, S0 of every step stored */
    T *s0 = (T *)calloc(ntp * nt, sizeof(T));
    FN(orc_fld) f, l;
    FN(fld_alloc)(&f, ntp);
    const size_t src = (size_t)g->s_ix * ntz + g->s_iz;
    for (int it = 0; it < nt; it++) {
        FN(upd_vx)(&M, &f, m->dx, Lc, ntz - Lc, Lc - 1, ntx - Lc - 1);
        FN(upd_vz)(&M, &f, m->dz, Lc - 1, ntz - Lc - 1, Lc, ntx - Lc);
        FN(upd_p_born)(&M, &f, m->dx, m->dz, s0 + (size_t)it * ntp, NULL, NULL);
        f.p[src] += rick[it];
    }
    FN(fld_free)(&f);
    /* adjoint: l.p = p^, l.vx/vz = v^, l.ppx/ppz = psi^ (velocity CPML), l.pvx/pvz = phi^ */
    FN(fld_alloc)(&l, ntp);
    memset(grad, 0, sizeof(T) * ntp);
    for (int k = nt - 1; k >= 0; k--) {
        /* P^T: p' = p + c*(Dx- vx + phi_x' + Dz- vz + phi_z'), phi' = b*phi + a*D- v on Gp */
        for (int ix = Lc; ix <= ntx - Lc; ix++)
            for (int iz = Lc; iz <= ntz - Lc; iz++) {
                const size_t ip = (size_t)ix * ntz + iz;
                const T q = dt * M.rho[ip] * M.vp[ip] * M.vp[ip] * l.p[ip];
                const T qx = q + M.ax[ix] * (q + l.pvx[ip]);
                const T qz = q + M.az[iz] * (q + l.pvz[ip]);
                l.pvx[ip] = M.bx[ix] * (q + l.pvx[ip]);
                l.pvz[ip] = M.bz[iz] * (q + l.pvz[ip]);
                for (int ic = 0; ic < Lc; ic++) {
                    l.vx[ip + (size_t)ic * ntz] += M.rc[ic] * odx * qx;
                    l.vx[ip - (size_t)(ic + 1) * ntz] -= M.rc[ic] * odx * qx;
                    l.vz[ip + ic] += M.rc[ic] * odz * qz;
                    l.vz[ip - (ic + 1)] -= M.rc[ic] * odz * qz;
                }
            }
        /* V^T: vx' = vx + dt/rho_x*(Dx+ p + psi_x'), psi_x' = b'*psi_x + a'*Dx+ p on Gx */
        for (int ix = Lc - 1; ix <= ntx - Lc - 1; ix++)
            for (int iz = Lc; iz <= ntz - Lc; iz++) {
                const size_t ip = (size_t)ix * ntz + iz;
                const T orho = (T)(1 / (0.5 * (M.rho[ip] + M.rho[ip + ntz])));
                const T r = dt * orho * l.vx[ip];
                const T R = r + M.axh[ix] * (r + l.ppx[ip]);
                l.ppx[ip] = M.bxh[ix] * (r + l.ppx[ip]);
                for (int ic = 0; ic < Lc; ic++) {
                    l.p[ip + (size_t)(ic + 1) * ntz] += M.rc[ic] * odx * R;
                    l.p[ip - (size_t)ic * ntz] -= M.rc[ic] * odx * R;
                }
            }
        for (int ix = Lc; ix <= ntx - Lc; ix++)
            for (int iz = Lc - 1; iz <= ntz - Lc - 1; iz++) {
                const size_t ip = (size_t)ix * ntz + iz;
                const T orho = (T)(1 / (0.5 * (M.rho[ip] + M.rho[ip + 1])));
                const T r = dt * orho * l.vz[ip];
                const T R = r + M.azh[iz] * (r + l.ppz[ip]);
                l.ppz[ip] = M.bzh[iz] * (r + l.ppz[ip]);
                for (int ic = 0; ic < Lc; ic++) {
                    l.p[ip + (ic + 1)] += M.rc[ic] * odz * R;
                    l.p[ip - ic] -= M.rc[ic] * odz * R;
                }
            }
        /* R^T and the gradient of this step */
        for (int r = 0; r < g->nrec; r++) l.p[(size_t)g->r_ix[r] * ntz + g->r_iz[r]] += (T)resid[(size_t)r * nt + k];
        const T *s = s0 + (size_t)k * ntp;
        for (size_t ip = 0; ip < ntp; ip++) grad[ip] += dt * s[ip] * l.p[ip];
    }
    FN(fld_free)(&l);
    free(s0);
    FN(mdl_free)(&M);
}

#undef FN
#undef ORC_CAT
#undef ORC_CAT_
