/*
 * oracle/swd_oracle.h -- CPU oracle for the single-GPU VSP RTM / PSF-decon hot path.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load this library, and only as the checker; the product (libswd)
 * never links or calls it.
 *
 * What it is: a plain-C restatement of the reference's loops, each function citing the
 * reference file:line it follows (paths relative to the reference project root).
 *   - host preparation (stencil coefficients, CPML profiles, Ricker wavelet, model
 *     padding, Gaussian smoothing, kz taper, well geometry) with the reference's own
 *     float/double arithmetic, so they can be compared bit for bit;
 *   - the propagation, imaging and deconvolution loops, compiled twice: once in float
 *     (the FP32 oracle, also the OpenMP CPU baseline) and once in double (the FP64
 *     oracle that image errors are quoted against).  Entry points end in _f32 / _f64.
 *
 * Pinning: the host preparation and the decon are checked against the reference's own
 * sources compiled here (oracle/Makefile -> oracle/_ref), the smoothing against the
 * reference's shipped kkdecon_acoustic/input/ini_vp.bin, the FFT against numpy.fft, and
 * forward/RTM against the reference's own CUDA build run on a B200 (tests/golden/).
 *
 * Grid convention (reference headrtm.h / acoustic_HLVSPRTMC.cpp:78-83): padded grid
 * ntx = nx + 2*pmlc, ntz = nz + 2*pmlc, pmlc = pml + Lc, cell ip = ix*ntz + iz (z fastest).
 */
#ifndef SWD_ORACLE_H
#define SWD_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- host preparation (reference arithmetic, exact) ---------------- */
void orc_cal_xishu(int Lc, float *rc);
void orc_cpml(int ntx, int ntz, int pmlc, float dx, float dz, float dt,
              float *a_x, float *a_x_half, float *a_z, float *a_z_half,
              float *b_x, float *b_x_half, float *b_z, float *b_z_half);
void orc_ricker2(int nt, float f0, float dt, float *rick);
void orc_pad_model(int nx, int nz, int pmlc, const float *v_in, float *v_pad);
void orc_smooth(int ntx, int ntz, int pmlc, int window, float *vp);
int orc_pow2_len(int n);
int orc_kz_taper(int nfftz, float dz, float *coef);
void orc_hilbert1d(int nt, const float *rick, float *hrick);
int orc_well_count(int nz, int pmlc, float dz, float shotdep, float offsetz);
void orc_well_geometry(int nx, int nz, int pmlc, float dz, float shotdep, float offsetz,
                       int *r_ix, int *r_iz);

/* ---------------- model descriptor shared by the loop restatements ---------------- */
typedef struct {
    int ntx, ntz, pmlc, Lc, nt;
    float dx, dz, dt;
    const float *rc;                       /* [Lc] */
    const float *vp, *rho;                 /* [ntx*ntz] */
    const float *a_x, *a_x_half, *a_z, *a_z_half;
    const float *b_x, *b_x_half, *b_z, *b_z_half;
} orc_model;

typedef struct {
    int s_ix, s_iz;
    int nrec;
    const int *r_ix, *r_iz;                /* [nrec], padded-grid cells */
} orc_geom;

/* number of boundary-strip values saved per time step: 2*Lc*nx + 2*Lc*(nz-2*Lc) */
int orc_strip_len(const orc_model *m);

#define ORC_DECL(T, S)                                                                        \
    /* forward propagation (acoustic_HLVSPRTMLc.cu:24-221,314-375;                        \
       forward/acoustic_hilbert_fftkz_HLForLc.cu:168-558,678-760) */                       \
    void orc_forward_##S(const orc_model *m, const orc_geom *g, const float *rick,           \
                         const float *hrick, T *seis, T *strips, T *final_state,            \
                         int ncol, const int *col_ix, T *cols);                             \
    /* kz up/down split of recorded columns (forward/...HLForLc.cu:52-137,761-777) */       \
    void orc_kzsep_##S(int ntz, int nfftz, int nt, int ncol, const T *cols,                 \
                       const float *coef, int nrec, const int *rec_col, const int *r_iz,    \
                       T *up, T *down);                                                     \
    /* -integral-integral preprocessing (acoustic_HLVSPRTMC.cpp:606-637) */                  \
    void orc_preprocess_##S(int nrec, int nt, float dt, const float *d, T *rms);            \
    /* backward: reconstruction + receiver back-propagation + imaging                       \
       (acoustic_HLVSPRTMLc.cu:434-817,1073-1148) */                                        \
    void orc_rtm_backward_##S(const orc_model *m, const orc_geom *g, const float *rick,     \
                              const T *rms, const T *strips, const T *final_state,          \
                              T *img, T *illum_s, T *illum_r,                               \
                              int thetan, int delt, float *cig /* nullable */);             \
    /* per-shot normalisation + -vp^2 Laplacian (acoustic_HLVSPRTMC.cpp:663-743) */          \
    void orc_rtm_post_##S(const orc_model *m, const T *img, const T *illum_s,               \
                          T *img_norm, T *fimage);                                          \
    /* Born modelling in kappa = rho*vp^2 and its exact adjoint (project operators) */      \
    void orc_born_##S(const orc_model *m, const orc_geom *g, const float *rick,              \
                      const float *dkappa, T *dseis);                                       \
    void orc_born_adjoint_##S(const orc_model *m, const orc_geom *g, const float *rick,     \
                              const float *resid, T *grad);

ORC_DECL(float, f32)
ORC_DECL(double, f64)

/* edge zeroing of the stacked image (acoustic_HLVSPRTMC.cpp:754-768) */
void orc_edge_zero(int nx, int nz, int Lc, float *img);

/* ---------------- windowed wavenumber PSF deconvolution ----------------
 * kkdecon_acoustic/kk_decon_interp_psf_minewindow.cpp:84-132,303-339,355-383,543-674.
 * fft_n0/fft_n1 <= 0 keep the reference's FFT size (fullw = filterwin + psfwin - 1);
 * positive values select a larger zero-padded FFT (project option, not in the reference).
 * Outputs are nx*nz (cropped from the expanded nxp*nzp grid as the reference writes them). */
typedef struct {
    int nx, nz;
    int psfwinx, psfwinz, filterwinx, filterwinz, snapwinx, snapwinz;
    float epsilon;
    int fft_n0, fft_n1;
    int psf_interp;   /* 1: bilinear interpolation of the lattice PSFs (project option) */
    /* project option, no reference counterpart (its reg_eps and itn are parsed, never used):
     * iters FISTA steps from the damped solution x0 on 1/2|s*x-m|^2 + mu/2|x|^2 + lambda|x|_1,
     * mu = reg_l2*max|S^|^2, step 1/(max|S^|^2 + mu), soft threshold reg_l1*max|x0| */
    int iters;
    float reg_l1, reg_l2;
} orc_decon_params;

int orc_decon_geometry(const orc_decon_params *p, int *out /* 16 ints, see swd_oracle.c */);
int orc_decon(const orc_decon_params *p, const float *migreal, const float *migpsf,
              float *mig_dec, float *mig_coef, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
