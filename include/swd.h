/*
 * swd.h -- C ABI of libswd, the B200 (sm_100a) engine for single-GPU VSP reverse-time
 * migration with scatter-point PSFs and windowed wavenumber PSF deconvolution.
 *
 * The reference programs (AFor, AVSPRTM, decon2d_mine) talk to their GPU code through
 * extern "C" functions taking POD structs (forward/headrtm.h, headrtm.h).  This header
 * replaces that seam with an opaque context and plain pointers; each entry point names
 * the reference interface it stands in for.
 *
 * Conventions
 *  - Grids are the reference's padded grids: ntx = nx + 2*pmlc, ntz = nz + 2*pmlc,
 *    pmlc = pml + Lc, cell (ix, iz) at ix*ntz + iz (z fastest), float32 little-endian.
 *  - Every pointer argument may be a host pointer or a device pointer on the context's
 *    device; the library detects which (cudaPointerGetAttributes).  Host results are
 *    complete when the call returns.
 *  - Every call returns an int status (SWD_OK = 0); swd_last_error() describes the last
 *    failure on a context.  A context is used by one host thread at a time and owns one
 *    CUDA stream (swd_set_stream() may substitute the caller's).  Time loops run as
 *    replayed CUDA graphs of 64 steps; on the legacy default stream (handle 0), which cannot
 *    be captured, they are launched step by step instead.
 *  - Seismograms are trace-major [r_n][nt]; images nx*nz unless stated otherwise.
 */
#ifndef SWD_H
#define SWD_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define SWD_OK 0
#define SWD_ERR_ARG 1        /* invalid argument or size */
#define SWD_ERR_CUDA 2       /* CUDA runtime error (message in swd_last_error) */
#define SWD_ERR_ALLOC 3      /* device or host allocation failed */
#define SWD_ERR_STATE 4      /* call made before the data it needs was set */
#define SWD_ERR_DEVICE 5     /* a kernel reported an error status */

/* strip storage precision for the source-wavefield reconstruction */
#define SWD_STRIP_F32 0
#define SWD_STRIP_F16 1      /* IEEE half with a per-(step, tile) scale */
#define SWD_STRIP_BF16 2     /* bfloat16 with a per-(step, tile) scale */
#define SWD_STRIP_I16 3      /* int16 fixed point of value / per-(step, tile) max |value| */

/* flags of swd_rtm_shot */
#define SWD_RTM_PREPROCESS 1u     /* apply rms = -int int d dt dt to the data first (reference default) */
#define SWD_RTM_ILLUM_RCV 2u      /* also accumulate the receiver illumination R = sum p_r^2 */
#define SWD_RTM_NO_STACK 4u       /* do not add this shot's filtered image to the stack */
#define SWD_RTM_CIG 8u            /* also accumulate angle-domain common-image gathers (swd_set_cig) */

typedef struct swd_ctx swd_ctx;

typedef struct {
    int nx, nz;          /* interior grid */
    int pml, Lc;         /* CPML cells and half stencil length; pmlc = pml + Lc */
    float dx, dz, dt;
    int nt_max;          /* longest record the context will run */
    int device;          /* CUDA device ordinal */
} swd_grid;

/* One shot: source cell and receiver cells, padded-grid coordinates.
 * Replaces struct Source (headrtm.h:8-13, forward/headrtm.h:12-17), whose receivers are
 * the depth list r_iz[] recorded at the two edge wells (acoustic_HLVSPRTMLc.cu:180-197). */
typedef struct {
    int s_ix, s_iz;
    int nt;              /* record length of this shot (<= nt_max) */
    int r_n;
    const int *r_ix;     /* [r_n] */
    const int *r_iz;     /* [r_n] */
} swd_shot;

/* ---- context ------------------------------------------------------------------------
 * Replaces getdevice/variables_malloc/variables_free (headrtm.h:5-6,176-186;
 * acoustic_HLVSPRTMLc.cu:1613-1845; forward/acoustic_hilbert_fftkz_HLForLc.cu:1425-1692). */
int swd_version(void);
int swd_device_count(int *n);
int swd_create(swd_ctx **out, const swd_grid *grid);
int swd_destroy(swd_ctx *ctx);
const char *swd_last_error(const swd_ctx *ctx);
int swd_set_stream(swd_ctx *ctx, void *cuda_stream);
int swd_synchronize(swd_ctx *ctx);
/* bytes of device memory the context holds right now */
size_t swd_device_bytes(const swd_ctx *ctx);

/* ---- model and operator setup (the H2D block of fdtd_2d_GPU_forward,
 *      acoustic_HLVSPRTMLc.cu:274-304) ------------------------------------------------ */
int swd_set_stencil(swd_ctx *ctx, const float *rc);                 /* rc[Lc], cal_xishu */
int swd_set_cpml(swd_ctx *ctx, const float *a_x, const float *a_x_half,
                 const float *a_z, const float *a_z_half,
                 const float *b_x, const float *b_x_half,
                 const float *b_z, const float *b_z_half);
int swd_set_model(swd_ctx *ctx, const float *vp, const float *rho);   /* padded ntx*ntz */
int swd_set_strip_precision(swd_ctx *ctx, int strip_precision);       /* SWD_STRIP_* */
/* Source wavefield of the RTM backward pass (no reference counterpart; the reference
 * reconstructs it from boundary strips, acoustic_HLVSPRTMLc.cu:434-620).  store = 0 (default):
 * reconstruct, as the reference does.  store = 1: the forward pass stores dp/dt of every step on
 * the interior at `prec` (SWD_STRIP_*, 16-bit codes with one scale per step and 128x8-cell
 * block; nt * nx * nz * 2 bytes at 16 bits) and the backward pass propagates only the receiver
 * wavefield, moving ~40% fewer bytes per step; the image differs from the reconstructed one by
 * the storage rounding (and not at all in exact arithmetic). */
int swd_set_source_storage(swd_ctx *ctx, int store, int prec);
/* kernel path: SWD_PATH_PLAIN (default) runs four cells of a column per thread with 128-bit
 * loads and two launches per time step (the velocity and pressure halves, like the
 * reference's vx/vz/p kernels); SWD_PATH_FUSED (Lc <= 6) runs one launch per time step on
 * shared-memory tiles with the velocity halo recomputed. */
#define SWD_PATH_PLAIN 0
#define SWD_PATH_FUSED 1
int swd_set_kernel_path(swd_ctx *ctx, int path);

/* ---- forward modelling --------------------------------------------------------------
 * Replaces fdtd_2d_GPU_forward of AFor (forward/headrtm.h:159-171,
 * forward/acoustic_hilbert_fftkz_HLForLc.cu:576-863) and, with hrick = kz_coef = NULL, the
 * inv_flag=0 call of fdtd_2d_GPU_forward in AVSPRTM (headrtm.h:129-141).
 *   seis      [r_n][nt]  pressure at the receivers (required)
 *   hrick     Hilbert-transformed wavelet; with kz_coef it propagates the twin wavefield
 *   kz_coef   [nfftz] kz taper; nfftz = 2^ceil(log2(ntz)) as the reference computes it
 *   seis_up / seis_down  [r_n][nt] kz-separated traces, scaled by nfftz like the
 *             reference's unnormalised inverse cuFFT (both NULL unless hrick and kz_coef). */
int swd_forward(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *hrick,
                const float *kz_coef, float *seis, float *seis_up, float *seis_down);

/* ---- scatter (PSF) data as an exact scattered field ------------------------------------
 * Replaces the scatter mode's two forward runs and their difference
 * (forward/acoustic_hilbert_fftkz_HLForC.cpp:620-795: background and perturbed records,
 * scatter data = perturbed - background, :733-794).  The difference of two FP32 records of
 * nearly equal size loses the digits the scatter points carry (about 1e-3 relative error of the
 * difference for the reference's 1e-3 * vp density scatterers); here the difference field
 * u(m1) - u(m) itself is propagated in FP32 beside the background field, in the perturbed model
 * with the exact secondary sources (coefficient differences formed in double), so its error
 * is relative to the scatter data, not to the record.
 * swd_set_scatter_model: the perturbed model (padded ntx*ntz, like swd_set_model, which must
 * come first; setting a new background clears it); NULL, NULL clears it.
 * swd_forward_scatter: arguments as swd_forward; seis receives the scatter record and, with
 * hrick and kz_coef, seis_up / seis_down its kz-separated traces (a second pass propagates the
 * Hilbert wavelet's fields). */
int swd_set_scatter_model(swd_ctx *ctx, const float *vp1, const float *rho1);
int swd_forward_scatter(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *hrick,
                        const float *kz_coef, float *seis, float *seis_up, float *seis_down);

/* ---- RTM of one shot ---------------------------------------------------------------
 * Replaces the fdtd_2d_GPU_forward(inv_flag=1) + fdtd_2d_GPU_backward pair and the per-shot
 * host steps of AVSPRTM (acoustic_HLVSPRTMC.cpp:576-745; acoustic_HLVSPRTMLc.cu:239-432,
 * 946-1215).  The final forward wavefield stays in HBM (no disk round trip).
 *   data      [r_n][nt] receiver data (the up-going file in the reference flow)
 *   syn       [r_n][nt] synthetic data of the forward pass (nullable)
 *   image_pp  nx*nz  I/(S + 1e-3 max S) as written to image_pp%d / image_psf%d (nullable)
 *   image_src nx*nz  S (image_sources%d) (nullable)
 *   fimage    nx*nz  -vp^2 Laplacian of image_pp, fimage_pp%d (nullable)
 * Unless SWD_RTM_NO_STACK, fimage is added to the context's FP64 stack. */
int swd_rtm_shot(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *data,
                 unsigned flags, float *syn, float *image_pp, float *image_src, float *fimage);
/* The same RTM in two calls, like the reference's fdtd_2d_GPU_forward(inv_flag=1) /
 * fdtd_2d_GPU_backward pair (acoustic_HLVSPRTMLc.cu:239-432, 946-1215): swd_rtm_forward runs
 * the forward pass (syn nullable) and keeps its final wavefield and boundary strips in the
 * context instead of a disk file; swd_rtm_backward then migrates `data` for the same shot
 * (same source cell, nt and r_n).  Any other propagation call in between discards the kept
 * pass, and swd_rtm_backward then returns SWD_ERR_STATE. */
int swd_rtm_forward(swd_ctx *ctx, const swd_shot *shot, const float *rick, float *syn);
int swd_rtm_backward(swd_ctx *ctx, const swd_shot *shot, const float *data, unsigned flags,
                     float *image_pp, float *image_src, float *fimage);
/* Angle-domain common-image gathers of the reference's Poynting-vector kernel
 * (sum_image_GPU_kernel_imageCIG, acoustic_HLVSPRTMLc.cu:819-905, declared and allocated by the
 * reference but never launched): with SWD_RTM_CIG, every backward step adds p_s*p_r into
 * 1-degree reflection-angle bins 2 .. thetan-1 of each interior cell, the angle taken from the
 * source and receiver Poynting vectors averaged over delt steps (the reference host uses
 * thetan = 10, delt = 1).  Plain kernel path and reconstructed source only.  swd_rtm_cig copies
 * the last shot's gathers, nx*nz*thetan floats with the angle fastest. */
int swd_set_cig(swd_ctx *ctx, int thetan, int delt);
int swd_rtm_cig(swd_ctx *ctx, float *cig);
/* raw accumulators of the last shot on the padded grid: I, S (and R if accumulated), FP64 */
int swd_rtm_raw(swd_ctx *ctx, double *image, double *illum_src, double *illum_rcv);
/* the stacked image nx*nz, optionally with the reference's edge zeroing
 * (acoustic_HLVSPRTMC.cpp:750-768); reset clears it */
int swd_stack_get(swd_ctx *ctx, int edge_zero, float *migration);
int swd_stack_reset(swd_ctx *ctx);

/* ---- batched RTM: many shots of uneven nt and aperture, stacked ---------------------
 * Replaces the per-rank shot loop of AVSPRTM (acoustic_HLVSPRTMC.cpp:546-748) on one GPU.
 * Shots are sorted by nt and run B at a time in batched launches (one launch per half step
 * for the whole batch, time loops as CUDA graphs); each shot's -vp^2-filtered image is added
 * to the FP64 stack exactly as swd_rtm_shot adds it.  B = swd_set_option(SWD_OPT_BATCH), or
 * chosen by timing probes of B = 1, 2, 4, 8 on the first call (SWD_OPT_BATCH_TUNED reads the
 * choice).  flags: SWD_RTM_PREPROCESS only (the batch always stacks).  The context's current
 * strip precision applies.  Every shot is validated before any device work: a bad shot returns
 * SWD_ERR_ARG and leaves the stack unchanged. */
int swd_rtm_batch(swd_ctx *ctx, int nshots, const swd_shot *shots, const float *const *ricks,
                  const float *const *data, unsigned flags);

/* ---- engine options (no reference counterpart) ---------------------------------------
 * SWD_OPT_GRAPHS  1 (default): time loops replay captured CUDA graphs of 64 steps;
 *                 0: every kernel is launched from the host (the plain engine)
 * SWD_OPT_BATCH   shots per batched launch in swd_rtm_batch, 0 (default) = autotune
 * SWD_OPT_BATCH_TUNED  (read only) the autotuner's batch size, 0 before the first batch
 * SWD_OPT_IMAGE_BLOCKS 1 (default): the imaging condition sums each 64-step block of
 *                 backward steps in FP32 and adds the block sums into the FP64 accumulators
 *                 (16 instead of 32 bytes per cell and step; relative change of the images
 *                 about 1e-7); 0: every step adds into FP64 */
#define SWD_OPT_GRAPHS 1
#define SWD_OPT_BATCH 2
#define SWD_OPT_BATCH_TUNED 3
#define SWD_OPT_IMAGE_BLOCKS 4
/* SWD_OPT_BWD_BY_KIND 1 (default): each RTM backward step runs the two wavefields' velocity
 *                 phases in one launch and their pressure phases plus the imaging in the other
 *                 (dp/dt stays in registers; 20 bytes less per interior cell and step; the same
 *                 images bit for bit); 0: the reference's pairing (source p with receiver v,
 *                 source v with receiver p).  Angle gathers always use the reference's pairing. */
#define SWD_OPT_BWD_BY_KIND 5
/* SWD_OPT_TMA 1: the velocity launches of the single-wavefield forward pass and of the backward
 *                 pass paired by kind read the pressure through tiles that the Tensor Memory
 *                 Accelerator copies into shared memory (persistent CTAs, two stages; the same
 *                 images bit for bit); 0 (default): per-thread loads, which measure faster */
#define SWD_OPT_TMA 6
/* SWD_OPT_PDL 1: the RTM step kernels are programmatic dependent launches (the next launch's
 *                 blocks are placed while this one's last blocks run; each waits for its
 *                 predecessor before touching memory; the same images bit for bit); 0 (default):
 *                 plain stream order, which measures the same with CUDA graphs */
#define SWD_OPT_PDL 7
/* SWD_OPT_STAGED 1: the pressure launch of the single-wavefield forward pass (RTM forward and
 *                 plain modelling, no Born, checkpoint or stored-source mode) stages every
 *                 stencil operand of its tiles (vx and vz with their halos, p, the material
 *                 coefficient) through the Tensor Memory Accelerator into a three-stage
 *                 shared-memory ring walked by persistent CTAs, so the bytes in flight are bounded
 *                 by shared memory rather than registers (the same images bit for bit);
 *                 0 (default): per-thread loads */
#define SWD_OPT_STAGED 8
/* SWD_OPT_AUTOTUNE 1: the RTM passes choose their step-kernel variants themselves.  The forward
 *                 pass of one wavefield tries, on successive passes, the four combinations of
 *                 per-thread or TMA-staged velocity launch and per-thread or fully staged pressure
 *                 launch, and (stencil order 4) the pressure kernel's register bound at 4 and 6
 *                 blocks per SM instead of 5 and the velocity kernel's at 6; the backward pass
 *                 tries the by-kind pairing with per-thread or TMA-staged velocities, the
 *                 reference's pairing, and (order 4) the pressure-and-imaging kernel at 4 and 6
 *                 blocks per SM and the velocity kernel at 6.  Without the tuning the velocity
 *                 kernels take the 6-block bound when the pass's working set exceeds the L2.  Each try is timed with CUDA events over
 *                 its graph replays (captures excluded) and the fastest per step is kept for the
 *                 context.  Every variant gives the same images bit for bit, so only the speed of
 *                 the first few shots depends on the order.  Setting the option restarts the tuning;
 *                 while it is on it overrides SWD_OPT_TMA, SWD_OPT_STAGED and SWD_OPT_BWD_BY_KIND
 *                 for those passes.  0 (default): the options as set.
 * SWD_OPT_TUNED_FWD / SWD_OPT_TUNED_BWD (read only): the chosen variant (forward: 1 TMA velocity
 *                 + 2 staged pressure, 8 / 16 pressure kernel at 4 / 6 blocks per SM, 32 velocity
 *                 kernel at 6; backward: 1 TMA velocity, 4 reference pairing, 8 / 16 at 4 / 6
 *                 blocks per SM, 32 velocity kernel at 6), -1 while still trying or when the tuning
 *                 is off. */
#define SWD_OPT_AUTOTUNE 9
#define SWD_OPT_TUNED_FWD 10
#define SWD_OPT_TUNED_BWD 11
/* SWD_OPT_LEAN 1 (default): blocks of the step kernels that lie inside the CPML-free, strip-free
 *                 box (found from the arrays of swd_set_cpml) take a path without the update
 *                 guards, CPML branches and strip code; 0: every block takes the general path.  The
 *                 same results bit for bit. */
#define SWD_OPT_LEAN 12
int swd_set_option(swd_ctx *ctx, int option, int value);
int swd_get_option(swd_ctx *ctx, int option, int *value);

/* ---- Born modelling and its exact adjoint (LSRTM / velocity gradients) --------------
 * No reference counterpart: the reference only migrates.  The Born operator linearises the
 * forward modelling of swd_forward in the bulk modulus kappa = rho*vp^2: the scattered field
 * propagates beside the background and receives dt*dkappa*S0 after each pressure update (S0
 * the background's p-update sum), and its pressure is recorded at the receivers.
 * swd_born_adjoint applies the exact transpose of that discrete operator, CPML included,
 * so <dseis_star, L dkappa> = <L^T dseis_star, dkappa> to rounding:
 *   grad[c] = sum_k dt * S0^k[c] * lambda_p^k[c],  lambda the adjoint state.
 * The adjoint needs S0 at every step in reverse order.  swd_set_checkpointing selects how:
 *   every == 0: the background pass stores S0 for all nt steps (FP32, nt*ntx*ntz floats);
 *   every  > 0: the background state (p, vx, vz and 4 CPML arrays) is stored every `every`
 *               steps at `prec` (SWD_STRIP_F32 / F16 / BF16 / I16, 16-bit with one scale per
 *               snapshot, array and 128x8-cell block) and each segment is recomputed
 *               before its adjoint steps.  Default: every = 50, BF16.
 * swd_born optionally leaves the background checkpoints of its pass in `ckpt` (device
 * memory of at least swd_checkpoint_bytes bytes, caller-owned, its size in ckpt_bytes; a
 * smaller buffer is rejected with SWD_ERR_ARG); swd_born_adjoint given the same `ckpt` for
 * the same shot skips its own background pass.  With ckpt = NULL (or every == 0)
 * swd_born_adjoint runs the background pass itself.
 *   dkappa  ntx*ntz padded grid (model layout), perturbation of rho*vp^2
 *   dseis   [r_n][nt] Born data;  resid [r_n][nt] adjoint source
 *   grad    ntx*ntz padded grid, FP64, d<resid, L dkappa>/d dkappa (overwritten) */
int swd_set_checkpointing(swd_ctx *ctx, int every, int prec);
int swd_checkpoint_bytes(swd_ctx *ctx, int nt, size_t *bytes);
int swd_born(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *dkappa, float *dseis,
             void *ckpt, size_t ckpt_bytes);
int swd_born_adjoint(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *resid,
                     double *grad, const void *ckpt, size_t ckpt_bytes);

/* ---- helpers that run on the GPU ----------------------------------------------------
 * swd_hilbert replaces hilbert_transform1d (forward/headrtm.h:228-229,
 * forward/acoustic_hilbert_fftkz_HLForLc.cu:1257-1324).
 * swd_smooth replaces ini_model_mine (acoustic_HLVSPRTMC.cpp:1473-1569): in place on a
 * padded ntx*ntz model, same double accumulation order.
 * swd_preprocess applies the reference's -int int dt dt to [r_n][nt] traces
 * (acoustic_HLVSPRTMC.cpp:606-637). */
int swd_hilbert(swd_ctx *ctx, int nt, const float *rick, float *hrick);
int swd_smooth(swd_ctx *ctx, int ntx, int ntz, int pmlc, int window, float *vp);
int swd_preprocess(swd_ctx *ctx, int r_n, int nt, float dt, const float *d, float *rms);

/* ---- windowed wavenumber PSF deconvolution -----------------------------------------
 * Replaces the window loop of decon2d_mine
 * (kkdecon_acoustic/kk_decon_interp_psf_minewindow.cpp:84-132,303-383,543-674).
 * fft_nx/fft_nz = 0 keep the reference's FFT size filterwin+psfwin-1; larger values select
 * a zero-padded FFT (project option).  Outputs are nx*nz like the reference's files. */
typedef struct {
    int nx, nz;
    int psfwinx, psfwinz, filterwinx, filterwinz, snapwinx, snapwinz;
    float epsilon;
    int fft_nx, fft_nz;
    /* 0: the nearest lattice PSF (the reference's rule, :586-598); 1: bilinear interpolation
     * of the four lattice PSFs around the window centre, within the same clamped lattice range
     * (project option: the reference declares but does not implement it, headpsf.h:166-167) */
    int psf_interp;
    /* 0: the window's transform buffer in shared memory when it fits (FX*FZ*8 bytes up to about
     * 200 KB, e.g. 158 x 158), otherwise in a global-memory workspace with each transform pass
     * staged through shared memory (same arithmetic, same bits); 1: always the workspace */
    int workspace;
    /* Iterative regularised deconvolution (project option: the reference parses reg_eps and its
     * parameter file lists an L2 coefficient and an iteration count, kkdecon_acoustic/
     * parameter.txt:35-40, but never uses them).  iters > 0 refines each window's damped
     * spectral solution x0 with iters FISTA steps on
     *   1/2 |psf * x - patch|^2 + mu/2 |x|^2 + lambda |x|_1,  mu = reg_l2 * max|PSF^|^2,
     * step 1/(max|PSF^|^2 + mu), soft threshold reg_l1 * max|x0| per step (both the patch and
     * the PSF L1-normalised as in the direct path).  iters = 0: the reference's direct division. */
    int iters;
    float reg_l1, reg_l2;
} swd_decon_params;
int swd_decon_geometry(const swd_decon_params *p, int *windows, int *fft_nx, int *fft_nz);
int swd_decon(swd_ctx *ctx, const swd_decon_params *p, const float *migreal,
              const float *migpsf, float *mig_dec, float *mig_coef);

/* ---- instrumentation (no reference counterpart; the reference only prints clock()) ---
 * swd_profile(ctx, every): bracket each kernel launch of every `every`-th time step with
 * CUDA events on the context stream (0 disables).  swd_profile_read fills, per kernel id
 * (0 forward-v, 1 forward-p, 2 backward-1, 3 backward-2 of the plain path; 4 forward step,
 * 5 backward step of the fused path; 6 / 7 whole forward / backward time steps, i.e. a pass
 * divided by its steps; 8 / 9 the two adjoint kernels of swd_born_adjoint and 10 its whole
 * adjoint time step), the summed milliseconds and the
 * number of timed launches, and clears them.  swd_launch_count is the number of kernels the
 * context has launched since it was created. */
#define SWD_NKERNELS 11
int swd_profile(swd_ctx *ctx, int every);
int swd_profile_read(swd_ctx *ctx, double *ms, long long *launches);
long long swd_launch_count(const swd_ctx *ctx);

/* ---- deconvolution without allocation ------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory while
 * they run: plug-in hosts that own the whole device memory pool and hand their plug-ins only
 * the buffers they pass in, and latency-bound services that reserve memory up front because
 * cudaFree synchronises the whole device and would stall their other streams.
 * Same algorithm and kernels as swd_decon, but all scratch (the per-window result slots, the
 * output taper and, for the workspace or iterative variants, the per-CTA workspaces) lives in
 * one static device array of SWD_DECON_STATIC_SCRATCH_FLOATS floats (16 MiB) that every GPU
 * which loads libswd holds until the process exits; those variants run on as many CTAs as
 * have a workspace that fits.  The call
 * allocates nothing: migreal/migpsf (nx*nz) and mig_dec/mig_coef (nx*nz) must be device
 * memory on the current device, already allocated by the caller.  Work is enqueued on
 * `cuda_stream` (NULL = the default stream); results are ready when that stream reaches it.
 * Returns SWD_ERR_CAPACITY when windows*outwinx*outwinz + outwinx*outwinz floats (plus the
 * transform tables, a few thousand floats) exceed the array
 * (or leaves no room for one CTA workspace when one is needed),
 * SWD_ERR_ARG for invalid geometry or for pointers that are not device memory of the current
 * device (host memory, or another GPU's memory, which the kernels could not dereference),
 * SWD_ERR_CUDA for a failed launch or query.  Each call looks up the array's device address
 * on the current device (cudaGetSymbolAddress, which allocates nothing); the first lookup on a
 * device loads the library's kernels there, so make the first call on each device before any
 * stream capture.  Every call reuses the same array and leaves its contents behind; each
 * call writes every scratch word it reads, so nothing needs clearing, but calls that overlap
 * on the GPU (other streams or host threads) race on the shared array. */
#define SWD_ERR_CAPACITY 6
#define SWD_DECON_STATIC_SCRATCH_FLOATS (4u << 20)
int swd_decon_noalloc(const swd_decon_params *p, const float *migreal, const float *migpsf,
                      float *mig_dec, float *mig_coef, void *cuda_stream);

/* ---- host preparation (the reference's host functions, restated) ------------------- */
/* cal_xishu, acoustic_HLVSPRTMC.cpp:1858-1878 */
void swd_prep_xishu(int Lc, float *rc);
/* get_absorbing_parameters, acoustic_HLVSPRTMC.cpp:891-1129 (pml argument = pmlc) */
void swd_prep_cpml(int ntx, int ntz, int pmlc, float dx, float dz, float dt,
                   float *a_x, float *a_x_half, float *a_z, float *a_z_half,
                   float *b_x, float *b_x_half, float *b_z, float *b_z_half);
/* ricker_wave flag 2 with t0 = 1/f0, acoustic_HLVSPRTMC.cpp:1249-1299 */
void swd_prep_ricker(int nt, float f0, float dt, float *rick);
/* get_acc_model edge replication, acoustic_HLVSPRTMC.cpp:1136-1196 */
void swd_prep_pad(int nx, int nz, int pmlc, const float *v_in, float *v_pad);
/* 2^ceil(log2 n) exactly as the reference evaluates it (forward/...HLForC.cpp:299-300) */
int swd_prep_pow2(int n);
/* kz taper, forward/...HLForC.cpp:354-377; returns layerz or -1 if the reference aborts */
int swd_prep_kz_taper(int nfftz, float dz, float *coef);
/* two-edge-well receiver depths, acoustic_HLVSPRTMC.cpp:153-200 + acoustic_HLVSPRTMLc.cu:180-197;
 * returns r_n; r_ix/r_iz may be NULL to query the count */
int swd_prep_wells(int nx, int nz, int pmlc, float dz, float shotdep, float offsetz,
                   int *r_ix, int *r_iz);

#ifdef __cplusplus
}
#endif
#endif
