// swd.cu -- libswd: C ABI, context, and orchestration of the sm_100a kernels.
//
// One context = one padded grid on one device with one stream.  It owns every device
// buffer (model, CPML profiles, wavefields, strips, images, stack); nothing crosses the
// host boundary inside a shot except the per-step wavelet sample, which is a kernel
// argument.  The final forward wavefield stays in HBM for the backward pass (the
// reference writes it to disk, acoustic_HLVSPRTMLc.cu:403-415 / :994-1004).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <initializer_list>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include "../../include/swd.h"
#include "prop.cuh"
#include "prop_fused.cuh"
#include "prop_tma.cuh"
#include "born.cuh"
#include "fft.cuh"
#include "decon.cuh"

using namespace swd;

// ------------------------------------------------------------------------------------
// small helpers
// ------------------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;   // allocation base (what cudaFree takes)
    size_t n = 0;        // bytes allocated
    size_t off = 0;      // byte offset of element 0 (guard band of grid arrays)
};

struct swd_ctx {
    int dev = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    swd_grid grid{};
    int ntx = 0, ntz = 0, ldz = 0, pmlc = 0, Lc = 0, nx = 0, nz = 0;
    float rc[MAXLC] = {0};
    bool have_rc = false, have_cpml = false, have_model = false;
    int strip_prec = SWD_STRIP_F32;
    std::string err;
    std::vector<DevBuf *> bufs;
    // model / operator; mat = the update coefficients cbx, cbz, ck (struct Mat)
    DevBuf vp, rho, cpml[8], mat[4];
    // perturbed model of the exact scattered field (swd_set_scatter_model): its coefficients
    // and the coefficient differences dcbx, dcbz, dck against the background
    DevBuf vp1, rho1, mat1[4], dmat[3];
    bool have_scatter = false;
    // wavefields: w[0], w[1] (7 arrays each), dp/dt
    DevBuf wave[2][7], dpdt;
    // second copies of p, vx, vz, phi_p_x, phi_p_z for the fused (double-buffered) path
    DevBuf wave2[2][5];
    int path = SWD_PATH_PLAIN;
    // acquisition
    DevBuf wcol, wmap, seis, seis2, rdata, colbuf, kzcoef, tw;
    // strips
    DevBuf strips, strip_scale;
    // imaging
    DevBuf I, S, R, stack, reduce;
    bool have_R = false, have_shot = false;
    DevBuf stage_in, stage_out;
    // Born modelling and its adjoint: perturbation, gradient, background p-update sums,
    // context-owned checkpoints, adjoint scratch (Qx, Qz, Rx, Rz), adjoint source, aliases
    DevBuf dk, gk, s0, ckpt, adj[4], rbuf, alias;
    int ckpt_every = 50, ckpt_prec = SWD_STRIP_BF16;
    // batched RTM (swd_rtm_batch): every per-shot grid array is one allocation of per-shot slices
    struct BatchBufs {
        DevBuf w[2][7], dpdt, I, S, Ip, Sp, strips, scale, rdata, wcol, wmap, desc, wav, reduce;
    } bat;
    // the RTM forward pass whose final wavefield and strips are kept for swd_rtm_backward;
    // every other pass that reuses those buffers clears it
    struct KeptShotState {
        bool valid;
        int s_ix, s_iz, nt, r_n, path;
        bool stored;     // the forward pass stored dp/dt (no reconstruction needed)
    };
    KeptShotState kept{false, 0, 0, 0, 0, 0, false};
    // stored-source RTM: the forward pass keeps dp/dt of every step (swd_set_source_storage)
    int src_store = 0, src_prec = SWD_STRIP_I16;
    DevBuf dpst, dpsc;
    // angle-domain common-image gathers (SWD_RTM_CIG)
    int cig_thetan = 0, cig_delt = 1;
    bool have_cig = false;
    DevBuf cig, cigring;
    // deconvolution scratch kept between swd_decon calls: inputs, taper, window slots,
    // outputs, staged workspaces
    DevBuf dcn[6];
    DevBuf Ipart, Spart, Rpart;   // FP32 block sums of the imaging condition
    int batch_opt = 0;      // shots per batched launch; 0 = autotune on first use
    int batch_tuned = 0;    // the autotuner's choice (0 = not tuned yet)
    // chunked CUDA-graph execution of the time loops
    DevBuf ctrl, wav;
    struct StepGraph {
        cudaGraphExec_t exec = nullptr, probe = nullptr;
        std::vector<char> key;
        std::vector<cudaEvent_t> ev;   // probe events: (start, end) per kernel of the probed step
    } gfwd, gbwd, gseg, gadj, gbf, gbb;
    int use_graphs = 1;
    int image_blocks = 1;   // SWD_OPT_IMAGE_BLOCKS
    int bwd_by_kind = 1;    // SWD_OPT_BWD_BY_KIND
    int use_tma = 0;        // SWD_OPT_TMA
    int use_pdl = 0;        // SWD_OPT_PDL
    int use_staged = 0;     // SWD_OPT_STAGED
    // SWD_OPT_AUTOTUNE: the step-kernel variants of a pass (all give the same bits) are tried on
    // successive passes, each timed over its graph replays, and the fastest is kept
    struct PassTune {
        int cand[8] = {0};
        double ms[8] = {0};
        int ncand = 0, next = 0, choice = -1;
    };
    int autotune = 0;
    PassTune tfwd, tbwd;
    size_t l2_bytes = 0;    // the device's L2 size, for the default register bounds
    int lean[4] = {0, 0, 0, 0};   // lean box of the step kernels (Geo::lx0 ...), from the CPML arrays
    int use_lean = 1;             // SWD_OPT_LEAN
    // instrumentation
    int prof_every = 0;
    double prof_ms[SWD_NKERNELS] = {0};
    long long prof_n[SWD_NKERNELS] = {0};
    long long launches = 0;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pending;
    std::vector<int> prof_count;
    std::vector<cudaEvent_t> ev_pool;
    swd_ctx()
    {
        DevBuf *all[] = {&vp, &rho, &dpdt, &wcol, &wmap, &seis, &seis2, &rdata, &colbuf, &kzcoef, &tw,
                         &strips, &strip_scale, &I, &S, &R, &stack, &reduce, &stage_in, &stage_out, &ctrl, &wav,
                         &dk, &gk, &s0, &ckpt, &rbuf, &alias, &dpst, &dpsc, &cig, &cigring, &Ipart, &Spart, &Rpart};
        for (DevBuf *b : all) bufs.push_back(b);
        for (auto &b : adj) bufs.push_back(&b);
        for (auto &b : dcn) bufs.push_back(&b);
        DevBuf *ball[] = {&bat.dpdt, &bat.I, &bat.S, &bat.Ip, &bat.Sp, &bat.strips, &bat.scale, &bat.rdata, &bat.wcol, &bat.wmap,
                          &bat.desc, &bat.wav, &bat.reduce};
        for (DevBuf *b : ball) bufs.push_back(b);
        for (auto &w : bat.w)
            for (auto &b : w) bufs.push_back(&b);
        for (auto &b : cpml) bufs.push_back(&b);
        for (auto &b : mat) bufs.push_back(&b);
        for (auto &b : mat1) bufs.push_back(&b);
        for (auto &b : dmat) bufs.push_back(&b);
        bufs.push_back(&vp1);
        bufs.push_back(&rho1);
        for (auto &w : wave)
            for (auto &b : w) bufs.push_back(&b);
        for (auto &w : wave2)
            for (auto &b : w) bufs.push_back(&b);
    }
};

static int fail(swd_ctx *c, int code, const char *fmt, ...)
{
    char msg[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof msg, fmt, ap);
    va_end(ap);
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(ctx, SWD_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),  \
                        __FILE__, __LINE__);                                               \
    } while (0)

#define CKR(expr)                          \
    do {                                   \
        int r_ = (expr);                   \
        if (r_ != SWD_OK) return r_;       \
    } while (0)

static int ensure(swd_ctx *ctx, DevBuf &b, size_t bytes)
{
    b.off = 0;
    if (b.n >= bytes && b.p) return SWD_OK;
    if (b.p) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(b.p);
        b.p = nullptr;
        b.n = 0;
    }
    if (bytes == 0) return SWD_OK;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return fail(ctx, SWD_ERR_ALLOC, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    b.n = bytes;
    return SWD_OK;
}

static bool is_device_ptr(const void *p)
{
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Whether a kernel running on device dev may dereference p: managed memory, or device memory
// allocated on dev.  Device memory of another GPU is not (it would need peer access); copies
// (cudaMemcpyAsync) still reach it, so the copy paths use is_device_ptr.
static bool is_device_ptr_on(const void *p, int dev)
{
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeManaged || (at.type == cudaMemoryTypeDevice && at.device == dev);
}

// copy n elements of host-or-device src into device buffer dst
static int to_dev(swd_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    CK(cudaMemcpyAsync(dst, src, bytes, is_device_ptr(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       ctx->stream));
    return SWD_OK;
}

static int from_dev(swd_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    CK(cudaMemcpyAsync(dst, src, bytes, is_device_ptr(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       ctx->stream));
    return SWD_OK;
}

// host copy of a small array that may live on the device
template <typename T>
static int host_copy(swd_ctx *ctx, std::vector<T> &out, const T *src, size_t n)
{
    out.resize(n);
    if (n == 0) return SWD_OK;
    if (is_device_ptr(src)) {
        CK(cudaMemcpyAsync(out.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    } else {
        memcpy(out.data(), src, n * sizeof(T));
    }
    return SWD_OK;
}

// padded-grid array (ntx x ntz, host layout) -> device layout with leading dimension ldz
static int grid_to_dev(swd_ctx *ctx, float *dst, const float *src)
{
    CK(cudaMemcpy2DAsync(dst, ctx->ldz * sizeof(float), src, ctx->ntz * sizeof(float), ctx->ntz * sizeof(float),
                         ctx->ntx, is_device_ptr(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                         ctx->stream));
    return SWD_OK;
}

static inline float *F(DevBuf &b) { return (float *)((char *)b.p + b.off); }
static inline double *D(DevBuf &b) { return (double *)((char *)b.p + b.off); }

// A grid-shaped array: ntx*ldz elements plus GUARD elements on both sides, zero-filled, so
// the four-cell kernels can read the vector chunks next to the grid edges.
static int ensure_grid(swd_ctx *ctx, DevBuf &b, size_t elem, size_t extra_cols = 0)
{
    const size_t n = ((size_t)(ctx->ntx + extra_cols) * ctx->ldz + 2 * GUARD) * elem;
    const bool fresh = !(b.p && b.n >= n);
    CKR(ensure(ctx, b, n));
    b.off = GUARD * elem;
    if (fresh) CK(cudaMemsetAsync(b.p, 0, b.n, ctx->stream));
    return SWD_OK;
}
static inline int *I32(DevBuf &b) { return (int *)b.p; }

static Geo make_geo(const swd_ctx *c)
{
    Geo g;
    g.ntx = c->ntx; g.ntz = c->ntz; g.ldz = c->ldz; g.pmlc = c->pmlc; g.Lc = c->Lc;
    g.odx = (float)(1.0 / (double)c->grid.dx);
    g.odz = (float)(1.0 / (double)c->grid.dz);
    g.dt = c->grid.dt;
    for (int i = 0; i < MAXLC; i++) {
        g.rc[i] = c->rc[i];
        g.cx[i] = g.rc[i] * g.odx;
        g.cz[i] = g.rc[i] * g.odz;
        g.ncx[i] = g.rc[i] * -g.odx;
        g.ncz[i] = g.rc[i] * -g.odz;
    }
    // an empty box (every block on the general path) when SWD_OPT_LEAN is 0
    g.lx0 = c->use_lean ? c->lean[0] : 0; g.lx1 = c->use_lean ? c->lean[1] : 0;
    g.lz0 = c->use_lean ? c->lean[2] : 0; g.lz1 = c->use_lean ? c->lean[3] : 0;
    return g;
}

static Cpml make_cpml(swd_ctx *c)
{
    Cpml p;
    p.ax = F(c->cpml[0]); p.axh = F(c->cpml[1]); p.az = F(c->cpml[2]); p.azh = F(c->cpml[3]);
    p.bx = F(c->cpml[4]); p.bxh = F(c->cpml[5]); p.bz = F(c->cpml[6]); p.bzh = F(c->cpml[7]);
    return p;
}

static Mat make_mat(swd_ctx *c)
{
    Mat m;
    m.cbx = F(c->mat[0]); m.cbz = F(c->mat[1]); m.ck = F(c->mat[2]); m.kap = F(c->mat[3]);
    return m;
}

static Mat make_mat1(swd_ctx *c)
{
    Mat m;
    m.cbx = F(c->mat1[0]); m.cbz = F(c->mat1[1]); m.ck = F(c->mat1[2]); m.kap = F(c->mat1[3]);
    return m;
}

static Wave make_wave(swd_ctx *c, int k)
{
    Wave w;
    w.p = F(c->wave[k][0]); w.vx = F(c->wave[k][1]); w.vz = F(c->wave[k][2]);
    w.ppx = F(c->wave[k][3]); w.ppz = F(c->wave[k][4]); w.pvx = F(c->wave[k][5]); w.pvz = F(c->wave[k][6]);
    return w;
}

// ---- per-kernel event timing on a subsample of steps --------------------------------
static cudaEvent_t ev_get(swd_ctx *c)
{
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

struct ProfScope {   // records a (start, end) event pair around a span of work when active
    swd_ctx *c;
    int k;
    bool on;
    int count;
    cudaEvent_t a{}, b{};
    ProfScope(swd_ctx *c_, int k_, bool on_, int count_ = 1) : c(c_), k(k_), on(on_), count(count_)
    {
        if (on) { a = ev_get(c); b = ev_get(c); cudaEventRecord(a, c->stream); }
    }
    ~ProfScope()
    {
        if (on) {
            cudaEventRecord(b, c->stream);
            c->prof_pending.push_back({k, {a, b}});
            c->prof_count.push_back(count);
        }
    }
};

static void prof_collect(swd_ctx *c)
{
    if (c->prof_pending.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (size_t i = 0; i < c->prof_pending.size(); i++) {
        auto &p = c->prof_pending[i];
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess) {
            c->prof_ms[p.first] += ms;
            c->prof_n[p.first] += c->prof_count[i];
        }
        c->ev_pool.push_back(p.second.first);
        c->ev_pool.push_back(p.second.second);
    }
    c->prof_pending.clear();
    c->prof_count.clear();
    cudaGetLastError();
}

static size_t grid_bytes(const swd_ctx *c) { return (size_t)c->ntx * c->ldz * sizeof(float); }

static int zero_wave(swd_ctx *ctx, int k)
{
    for (int i = 0; i < 7; i++) {
        CKR(ensure_grid(ctx, ctx->wave[k][i], sizeof(float)));
        CK(cudaMemsetAsync(ctx->wave[k][i].p, 0, ctx->wave[k][i].n, ctx->stream));
    }
    return SWD_OK;
}

static dim3 grid_blocks(const swd_ctx *c) { return dim3((c->ntz + 127) / 128, (c->ntx + 7) / 8); }

// ---- fused path: 32 x 32 tiles, double-buffered fields --------------------------------
constexpr int FTX = 32, FTZ = 32;
static bool fused(const swd_ctx *c) { return c->path == SWD_PATH_FUSED && c->Lc <= 6; }
static dim3 fused_blocks(const swd_ctx *c) { return dim3((c->ntz + FTZ - 1) / FTZ, (c->ntx + FTX - 1) / FTX); }

static int zero_wave2(swd_ctx *ctx, int k)
{
    for (int i = 0; i < 5; i++) {
        CKR(ensure_grid(ctx, ctx->wave2[k][i], sizeof(float)));
        CK(cudaMemsetAsync(ctx->wave2[k][i].p, 0, ctx->wave2[k][i].n, ctx->stream));
    }
    return SWD_OK;
}

// copy `par` of field k: par 0 = wave[k][0..4], par 1 = wave2[k][0..4]
static float *fcopy(swd_ctx *c, int k, int par, int i) { return par ? F(c->wave2[k][i]) : F(c->wave[k][i]); }

static Field2 make_field2(swd_ctx *c, int k, int in_par)
{
    Field2 f;
    const int o = 1 - in_par;
    f.p = fcopy(c, k, in_par, 0); f.vx = fcopy(c, k, in_par, 1); f.vz = fcopy(c, k, in_par, 2);
    f.ppx = fcopy(c, k, in_par, 3); f.ppz = fcopy(c, k, in_par, 4);
    f.po = fcopy(c, k, o, 0); f.vxo = fcopy(c, k, o, 1); f.vzo = fcopy(c, k, o, 2);
    f.ppxo = fcopy(c, k, o, 3); f.ppzo = fcopy(c, k, o, 4);
    f.pvx = F(c->wave[k][5]); f.pvz = F(c->wave[k][6]);
    return f;
}

// ------------------------------------------------------------------------------------
// acquisition: receivers grouped by well column
// ------------------------------------------------------------------------------------
struct ShotPlan {
    int nwells = 0;
    std::vector<int> wcol;              // [ntx]
    std::vector<int> wmap;              // [nwells][ldz]
    std::vector<std::pair<int, int>> alias;  // (dst trace, src trace) for duplicate cells
    std::vector<int> well_x;
};

// validation and the host-side well maps of one shot (no device work)
static int plan_shot_host(swd_ctx *ctx, const swd_shot *s, ShotPlan &P)
{
    if (!s) return fail(ctx, SWD_ERR_ARG, "shot is NULL");
    if (s->nt < 2 || s->nt > ctx->grid.nt_max) return fail(ctx, SWD_ERR_ARG, "shot nt=%d outside [2, nt_max=%d]", s->nt, ctx->grid.nt_max);
    if (s->r_n < 1 || !s->r_ix || !s->r_iz) return fail(ctx, SWD_ERR_ARG, "shot needs r_n >= 1 receivers");
    if (s->s_ix < 0 || s->s_ix >= ctx->ntx || s->s_iz < 0 || s->s_iz >= ctx->ntz)
        return fail(ctx, SWD_ERR_ARG, "source cell (%d,%d) outside the %dx%d grid", s->s_ix, s->s_iz, ctx->ntx, ctx->ntz);
    std::vector<int> rx, rz;
    CKR(host_copy(ctx, rx, s->r_ix, s->r_n));
    CKR(host_copy(ctx, rz, s->r_iz, s->r_n));
    P.wcol.assign(ctx->ntx, -1);
    P.nwells = 0;
    for (int r = 0; r < s->r_n; r++) {
        if (rx[r] < 0 || rx[r] >= ctx->ntx || rz[r] < 0 || rz[r] >= ctx->ntz)
            return fail(ctx, SWD_ERR_ARG, "receiver %d cell (%d,%d) outside the grid", r, rx[r], rz[r]);
        if (P.wcol[rx[r]] < 0) { P.wcol[rx[r]] = P.nwells++; P.well_x.push_back(rx[r]); }
    }
    P.wmap.assign((size_t)P.nwells * ctx->ldz, -1);
    for (int r = 0; r < s->r_n; r++) {
        int &slot = P.wmap[(size_t)P.wcol[rx[r]] * ctx->ldz + rz[r]];
        // injection keeps the last trace for a cell (the reference loop order); recorded
        // traces of the other duplicates are copied from it afterwards
        if (slot >= 0) P.alias.push_back({slot, r});
        slot = r;
    }
    for (auto &a : P.alias) {   // make every alias point at the surviving trace
        int keep = P.wmap[(size_t)P.wcol[rx[a.first]] * ctx->ldz + rz[a.first]];
        a.second = keep;
    }
    return SWD_OK;
}

static int plan_shot(swd_ctx *ctx, const swd_shot *s, ShotPlan &P)
{
    CKR(plan_shot_host(ctx, s, P));
    CKR(ensure(ctx, ctx->wcol, sizeof(int) * ctx->ntx));
    CKR(ensure(ctx, ctx->wmap, sizeof(int) * P.wmap.size()));
    CK(cudaMemcpyAsync(ctx->wcol.p, P.wcol.data(), sizeof(int) * ctx->ntx, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->wmap.p, P.wmap.data(), sizeof(int) * P.wmap.size(), cudaMemcpyHostToDevice, ctx->stream));
    // pageable H2D copies above complete before returning, so the vectors may go away
    return SWD_OK;
}

static int copy_aliases(swd_ctx *ctx, const ShotPlan &P, float *dev_seis, int nt)
{
    for (auto &a : P.alias)
        if (a.first != a.second)
            CK(cudaMemcpyAsync(dev_seis + (size_t)a.first * nt, dev_seis + (size_t)a.second * nt, sizeof(float) * nt,
                               cudaMemcpyDeviceToDevice, ctx->stream));
    return SWD_OK;
}

// ------------------------------------------------------------------------------------
// kernels: data preprocessing, kz split, Hilbert, imaging post, smoothing, reductions
// ------------------------------------------------------------------------------------
// rms = -sum(sum(d*dt)*dt), one thread per trace, float ops in the reference's order
// without contraction (acoustic_HLVSPRTMC.cpp:606-637).
__global__ void k_preprocess(const float *__restrict__ d, float *__restrict__ out, int r_n, int nt, float dt)
{
    const int tr = blockIdx.x * blockDim.x + threadIdx.x;
    if (tr >= r_n) return;
    const float *src = d + (size_t)tr * nt;
    float *dst = out + (size_t)tr * nt;
    float t = 0.f;
    for (int it = 0; it < nt; it++) { t = __fadd_rn(t, __fmul_rn(src[it], dt)); dst[it] = t; }
    float u = 0.f;
    for (int it = 0; it < nt; it++) { u = __fadd_rn(u, __fmul_rn(dst[it], dt)); dst[it] = -u; }
}

// kz up/down split of the recorded well columns: forward FFT of (p + i*p_twin) along z,
// up = bins [0, N/2] x taper, down = bins (N/2, N) x taper, inverse FFTs, real part at the
// receiver depths (forward/acoustic_hilbert_fftkz_HLForLc.cu:52-137,761-777).
__global__ void __launch_bounds__(256) k_kzsep(const float2 *__restrict__ colbuf, const float *__restrict__ coef,
                                               const float2 *__restrict__ tw, const int *__restrict__ wmap,
                                               float *up, float *down, int nt, int ntz, int ldz, int N, int logN)
{
    extern __shared__ float2 sm[];
    float2 *su = sm, *sd = sm + N;
    const int c = blockIdx.y, it = blockIdx.x;
    const float2 *src = colbuf + ((size_t)c * nt + it) * ldz;
    for (int j = threadIdx.x; j < N; j += blockDim.x) su[j] = j < ntz ? src[j] : make_float2(0.f, 0.f);
    __syncthreads();
    block_fft_dif(su, N, tw);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        const int k = bitrev(j, logN);
        const float cf = __ldg(coef + k);
        const float2 v = make_float2(su[j].x * cf, su[j].y * cf);
        if (k <= N / 2) { su[j] = v; sd[j] = make_float2(0.f, 0.f); }
        else { sd[j] = v; su[j] = make_float2(0.f, 0.f); }
    }
    __syncthreads();
    block_ifft_dit(su, N, tw);
    block_ifft_dit(sd, N, tw);
    const int *m = wmap + (size_t)c * ldz;
    for (int z = threadIdx.x; z < ntz; z += blockDim.x) {
        const int tr = __ldg(m + z);
        if (tr >= 0) {
            up[(size_t)tr * nt + it] = su[z].x;
            down[(size_t)tr * nt + it] = sd[z].x;
        }
    }
}

// Hilbert transform of the wavelet on NZ = 2^ceil(log2 nt) points: -i on bins [1, NZ/2),
// +i on [NZ/2, NZ), bin 0 zeroed, inverse / NZ (forward/...HLForLc.cu:1257-1324).
__global__ void __launch_bounds__(256) k_hilbert(const float *__restrict__ rick, float *hr, const float2 *__restrict__ tw,
                                                  int nt, int N, int logN)
{
    extern __shared__ float2 sm[];
    for (int j = threadIdx.x; j < N; j += blockDim.x) sm[j] = make_float2(j < nt ? rick[j] : 0.f, 0.f);
    __syncthreads();
    block_fft_dif(sm, N, tw);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        const int k = bitrev(j, logN);
        const float2 f = sm[j];
        if (k == 0) sm[j] = make_float2(0.f, 0.f);
        else if (k < N / 2) sm[j] = make_float2(f.y, -f.x);
        else sm[j] = make_float2(-f.y, f.x);
    }
    __syncthreads();
    block_ifft_dit(sm, N, tw);
    for (int j = threadIdx.x; j < nt; j += blockDim.x) hr[j] = sm[j].x / (float)N;
}

// max of a non-negative double array (bit patterns of non-negative doubles order like
// the values, so an integer atomicMax is exact)
__global__ void k_max_nonneg(const double *__restrict__ a, size_t n, unsigned long long *out)
{
    double m = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(a[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// Per-shot post (acoustic_HLVSPRTMC.cpp:663-743): In = I/(S + 1e-3*max S) on the padded
// grid, -vp^2 * (5-point Laplacian of In) on the interior, stacked in FP64.
__global__ void k_rtm_post(const double *__restrict__ I, const double *__restrict__ S, const float *__restrict__ vp,
                           const unsigned long long *__restrict__ smax, int ntx, int ntz, int ldz, int pmlc,
                           float dx, float dz, float *img_pp, float *img_src, float *fimage, double *stack)
{
    const int nz = ntz - 2 * pmlc, nx = ntx - 2 * pmlc;
    const int iz = blockIdx.x * 32 + threadIdx.x, ixi = blockIdx.y * 8 + threadIdx.y;
    if (iz >= nz || ixi >= nx) return;
    const double rem = 1.0e-3 * __longlong_as_double((long long)*smax);
    const int x = ixi + pmlc, z = iz + pmlc;
    auto In = [&](int xx, int zz) -> float {
        const size_t q = (size_t)xx * ldz + zz;
        return (float)(I[q] / (S[q] + rem));
    };
    const size_t ip = (size_t)x * ldz + z;
    const float c = In(x, z);
    const double lap = (In(x + 1, z) - 2.0 * c + In(x - 1, z)) / (double)(dx * dx) +
                       (In(x, z + 1) - 2.0 * c + In(x, z - 1)) / (double)(dz * dz);
    const double v = (double)vp[ip];
    const float f = (float)(-lap * v * v);
    const size_t o = (size_t)ixi * nz + iz;
    if (img_pp) img_pp[o] = c;
    if (img_src) img_src[o] = (float)S[ip];
    if (fimage) fimage[o] = f;
    if (stack) stack[o] += (double)f;
}

// stacked image -> float, reference edge zeroing (acoustic_HLVSPRTMC.cpp:754-768)
__global__ void k_stack_out(const double *__restrict__ st, float *out, int nx, int nz, int Lc, int edge)
{
    const size_t n = (size_t)nx * nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i / nz), iz = (int)(i % nz);
        float v = (float)st[i];
        if (edge && (ix <= 3 || ix >= nx - Lc || iz < 7 || iz >= nz - Lc)) v = 0.f;
        out[i] = v;
    }
}

// Gaussian smoothing of ini_model_mine (acoustic_HLVSPRTMC.cpp:1514-1556): double
// accumulation in the reference's loop order with unfused multiply and add, clamped
// indices, rows iz < pml+8 unchanged.  Coefficients come from the host.
__global__ void k_smooth(const float *__restrict__ vin, float *vout, const double *__restrict__ coef, int ntx, int ntz,
                         int pml, int w)
{
    const int iz = blockIdx.x * 32 + threadIdx.x + pml, ix = blockIdx.y * 8 + threadIdx.y + pml;
    if (iz > ntz - pml - 1 || ix > ntx - pml - 1) return;
    const int wx = 2 * w + 1;
    double s = 0.0;
    for (int izw = iz - w; izw <= iz + w; izw++) {
        const int iz1 = izw < 0 ? 0 : (izw > ntz - 1 ? ntz - 1 : izw);
        for (int ixw = ix - w; ixw <= ix + w; ixw++) {
            const int ix1 = ixw < 0 ? 0 : (ixw > ntx - 1 ? ntx - 1 : ixw);
            s = __dadd_rn(s, __dmul_rn((double)vin[(size_t)ix1 * ntz + iz1], coef[(izw - iz + w) * wx + (ixw - ix + w)]));
        }
    }
    const size_t ip = (size_t)ix * ntz + iz;
    vout[ip] = iz < pml + 8 ? vin[ip] : (float)s;
}

// Update coefficients of struct Mat on the padded grid (same operations and order as the
// per-cell expressions of the reference kernels): cbx = dt*rcp(0.5*(rho[x]+rho[x+1])),
// cbz = dt*rcp(0.5*(rho[z]+rho[z+1])), ck = ((dt*rho)*vp)*vp, kap = (rho*vp)*vp.  Neighbours past the grid read
// the zeroed padding; coefficients whose denominator is zero are stored as 0 (the updates
// never use those cells).
__global__ void k_material(const float *__restrict__ vp, const float *__restrict__ rho, float dt, int ntx, int ntz,
                           int ldz, float *cbx, float *cbz, float *ck, float *kap)
{
    const size_t n = (size_t)ntx * ldz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % ldz);
        float bx = 0.f, bz = 0.f, kc = 0.f, ka = 0.f;
        if (z < ntz) {
            const float r0 = rho[i], r1 = rho[i + ldz], r2 = rho[i + 1], v = vp[i];
            const float sx = 0.5f * (r0 + r1), sz = 0.5f * (r0 + r2);
            if (sx != 0.f) bx = dt * __frcp_rn(sx);
            if (sz != 0.f) bz = dt * __frcp_rn(sz);
            kc = dt * r0 * v * v;
            ka = r0 * v * v;
        }
        cbx[i] = bx;
        cbz[i] = bz;
        ck[i] = kc;
        kap[i] = ka;
    }
}

// Differences of the update coefficients of a perturbed model (vp1, rho1) and the background
// (vp0, rho0), formed in double from the float models and rounded once, so the secondary
// sources of the exact scattered field carry the FP64 coefficient differences rather than the
// difference of two rounded coefficients (which would lose the digits the perturbation holds).
__global__ void k_material_delta(const float *__restrict__ vp0, const float *__restrict__ rho0,
                                 const float *__restrict__ vp1, const float *__restrict__ rho1, float dt, int ntx,
                                 int ntz, int ldz, float *dcbx, float *dcbz, float *dck)
{
    const size_t n = (size_t)ntx * ldz;
    const double t = (double)dt;
    auto b = [&](double r0, double r1) { const double s = 0.5 * (r0 + r1); return s != 0.0 ? t / s : 0.0; };
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % ldz);
        float bx = 0.f, bz = 0.f, kc = 0.f;
        if (z < ntz) {
            const double v0 = vp0[i], v1 = vp1[i], r0 = rho0[i], r1 = rho1[i];
            bx = (float)(b(r1, rho1[i + ldz]) - b(r0, rho0[i + ldz]));
            bz = (float)(b(r1, rho1[i + 1]) - b(r0, rho0[i + 1]));
            kc = (float)(t * r1 * v1 * v1 - t * r0 * v0 * v0);
        }
        dcbx[i] = bx;
        dcbz[i] = bz;
        dck[i] = kc;
    }
}

// model_in_pml (acoustic_HLVSPRTMC.cpp:1428-1468): x-edges for interior rows, then z-edges
__global__ void k_pml_x(float *v, int ntx, int ntz, int pml)
{
    const int iz = blockIdx.x * blockDim.x + threadIdx.x + pml;
    if (iz > ntz - pml - 1) return;
    for (int ix = 0; ix <= pml - 1; ix++) v[(size_t)ix * ntz + iz] = v[(size_t)pml * ntz + iz];
    for (int ix = ntx - pml; ix < ntx; ix++) v[(size_t)ix * ntz + iz] = v[(size_t)(ntx - pml - 1) * ntz + iz];
}
__global__ void k_pml_z(float *v, int ntx, int ntz, int pml)
{
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    if (ix >= ntx) return;
    for (int iz = 0; iz <= pml - 1; iz++) v[(size_t)ix * ntz + iz] = v[(size_t)ix * ntz + pml];
    for (int iz = ntz - pml; iz < ntz; iz++) v[(size_t)ix * ntz + iz] = v[(size_t)ix * ntz + (ntz - pml - 1)];
}

// ------------------------------------------------------------------------------------
// launch dispatch on the stencil half-length
// ------------------------------------------------------------------------------------
// the checkpointing and Born variants are separate instantiations, so the plain modelling
// and RTM kernels keep their register budget
// Launch of an RTM step kernel (block 32 x 8, no dynamic shared memory); with pdl, as a
// programmatic dependent launch (the step kernels open with pdl_begin)
template <typename... P, typename... A>
static void launch_step(void (*k)(P...), dim3 grid, cudaStream_t s, bool pdl, A &&...args)
{
    if (!pdl) {
        k<<<grid, dim3(32, 8), 0, s>>>(std::forward<A>(args)...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(32, 8);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

template <int LC>
static void launch_fwd_v(const FwdArgs &a, int nw, dim3 grid, cudaStream_t s, bool pdl = false, int mb = 0)
{
    const bool ck = a.ck.every > 0;
    // register-bound variant of the plain single-wavefield kernel (stencil order 4)
    if constexpr (LC == 4) {
        if (nw == 1 && !ck && mb == 6) return launch_step(k_fwd_v<4, 1, false, false, false, 6>, grid, s, pdl, a);
    }
    if (nw == 2 && a.dck) {
        launch_step(k_fwd_v<LC, 2, false, false, true>, grid, s, pdl, a);
    } else if (nw == 2) {
        if (ck) launch_step(k_fwd_v<LC, 2, true>, grid, s, pdl, a);
        else launch_step(k_fwd_v<LC, 2, false>, grid, s, pdl, a);
    } else {
        if (ck) launch_step(k_fwd_v<LC, 1, true>, grid, s, pdl, a);
        else launch_step(k_fwd_v<LC, 1, false>, grid, s, pdl, a);
    }
}

template <int LC>
static void launch_fwd_p(const FwdArgs &a, int nw, dim3 grid, cudaStream_t s, bool pdl = false, int mb = 0)
{
    const bool born = a.s0_out || a.dkappa;
    // register-bound variants of the plain single-wavefield kernel (stencil order 4 only)
    if constexpr (LC == 4) {
        if (nw == 1 && !a.ds.buf && !born && mb == 4) return launch_step(k_fwd_p<4, 1, FP_PLAIN, false, 4>, grid, s, pdl, a);
        if (nw == 1 && !a.ds.buf && !born && mb == 6) return launch_step(k_fwd_p<4, 1, FP_PLAIN, false, 6>, grid, s, pdl, a);
    }
    if (nw == 2 && a.dck) {
        launch_step(k_fwd_p<LC, 2, FP_SCAT>, grid, s, pdl, a);
    } else if (nw == 2) {
        if (born) launch_step(k_fwd_p<LC, 2, FP_BORN>, grid, s, pdl, a);
        else launch_step(k_fwd_p<LC, 2, FP_PLAIN>, grid, s, pdl, a);
    } else {
        if (a.ds.buf) launch_step(k_fwd_p<LC, 1, FP_STORE>, grid, s, pdl, a);
        else if (born) launch_step(k_fwd_p<LC, 1, FP_BORN>, grid, s, pdl, a);
        else launch_step(k_fwd_p<LC, 1, FP_PLAIN>, grid, s, pdl, a);
    }
}

template <int LC>
static void launch_bwd_1(const BwdArgs &a, dim3 grid, cudaStream_t s, bool pdl = false) { launch_step(k_bwd_1<LC>, grid, s, pdl, a); }

template <int LC>
static void launch_bwd_2(const BwdArgs &a, dim3 grid, cudaStream_t s, bool pdl = false) { launch_step(k_bwd_2<LC>, grid, s, pdl, a); }

template <int LC>
static void launch_bwd_v(const BwdArgs &a, dim3 grid, cudaStream_t s, bool pdl = false, int mb = 0)
{
    if constexpr (LC == 4) {   // register-bound variant (stencil order 4)
        if (mb == 6) return launch_step(k_bwd_v<4, false, 6>, grid, s, pdl, a);
    }
    launch_step(k_bwd_v<LC>, grid, s, pdl, a);
}

template <int LC>
static void launch_bwd_2_cig(const BwdArgs &a, const CigArgs &c, dim3 grid, cudaStream_t s, bool pdl = false)
{
    launch_step(k_bwd_2_cig<LC>, grid, s, pdl, a, c);
}

// ---- TMA-staged velocity kernels (prop_tma.cuh) -----------------------------------------
typedef CUresult (*TmapEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// the driver's tensor-map encoder, looked up once through the runtime (no libcuda link)
static TmapEncodeFn tmap_encoder()
{
    static const TmapEncodeFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return (TmapEncodeFn)p;
    }();
    return fn;
}

template <int LC>
static void tma_box(int *rows, int *cols)
{
    *rows = VTile<LC>::PR;
    *cols = VTile<LC>::PC;
}

// tensor map of a padded grid array (ntx columns of ldz floats) with a box of rows x cols
// (tma_box of the context's stencil order)
static bool make_pmap(const swd_ctx *ctx, CUtensorMap *m, const float *base, int rows, int cols)
{
    TmapEncodeFn enc = tmap_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)ctx->ldz, (cuuint64_t)ctx->ntx};
    const cuuint64_t strides[1] = {(cuuint64_t)ctx->ldz * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)rows, (cuuint32_t)cols};
    const cuuint32_t estride[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)base, dims, strides, box, estride,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// launch shape of a TMA velocity kernel with nbox boxes per stage: persistent CTAs, as many as
// are resident (nblk = 0 when the kernel cannot be used)
struct TmaShape {
    int nblk = 0;
    size_t smem = 0;
};

template <int LC>
static void tma_prepare(int dev, int nbox, TmaShape *t)
{
    t->nblk = 0;
    t->smem = vtile_smem<LC>(nbox);
    const void *fn = nbox == 1 ? (const void *)k_fwd_v_tma<LC> : (const void *)k_bwd_v_tma<LC>;
    int nsm = 0, occ = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t->smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, t->smem) != cudaSuccess || occ < 1) {
        cudaGetLastError();
        return;
    }
    t->nblk = nsm * occ;
}

template <int LC>
static void launch_fwd_v_tma(const FwdArgs &a, const CUtensorMap &m, int *err, const TmaShape &t, cudaStream_t s)
{
    k_fwd_v_tma<LC><<<t.nblk, dim3(32, 8), t.smem, s>>>(a, m, err);
}

template <int LC>
static void launch_bwd_v_tma(const BwdArgs &a, const CUtensorMap &mr, const CUtensorMap &ms, int *err, const TmaShape &t,
                             cudaStream_t s)
{
    k_bwd_v_tma<LC><<<t.nblk, dim3(32, 8), t.smem, s>>>(a, mr, ms, err);
}

// launch shape of the fully staged forward pressure kernel (nblk = 0: unusable here)
template <int LC>
static void staged_p_prepare(int dev, TmaShape *t)
{
    t->nblk = 0;
    t->smem = fwd_p_stage_smem<LC>();
    const void *fn = (const void *)k_fwd_p_staged<LC>;
    int nsm = 0, occ = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t->smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 32 * (ST_CONS + 1), t->smem) != cudaSuccess ||
        occ < 1) {
        cudaGetLastError();
        return;
    }
    t->nblk = nsm * occ;
}

// tensor maps of the staged forward pressure kernel: vx (TZ rows x VXC columns), vz (VZR x TX),
// p and ck (TZ x TX)
template <int LC>
static void staged_p_maps(const swd_ctx *ctx, const FwdArgs &a, CUtensorMap *m, bool *ok)
{
    using S = FwdPStage<LC>;
    *ok = make_pmap(ctx, &m[0], a.w[0].vx, ST_TZ, S::VXC) && make_pmap(ctx, &m[1], a.w[0].vz, S::VZR, ST_TX) &&
          make_pmap(ctx, &m[2], a.w[0].p, ST_TZ, ST_TX) && make_pmap(ctx, &m[3], a.m.ck, ST_TZ, ST_TX);
}

template <int LC>
static void launch_fwd_p_staged(const FwdArgs &a, const CUtensorMap *m, int *err, const TmaShape &t, cudaStream_t s)
{
    k_fwd_p_staged<LC><<<t.nblk, dim3(32, ST_CONS + 1), t.smem, s>>>(a, m[0], m[1], m[2], m[3], err);
}

// error word of the TMA kernels (set when a wait on a copy gave up), after the step counter
static int *tma_err(swd_ctx *ctx) { return I32(ctx->ctrl) + 8; }

static int tma_check(swd_ctx *ctx)
{
    int h = 0;
    CK(cudaMemcpyAsync(&h, tma_err(ctx), sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h) return fail(ctx, SWD_ERR_CUDA, "a TMA-staged kernel gave up waiting for its tile");
    return SWD_OK;
}

template <int LC>
static void launch_bwd_p(const BwdArgs &a, dim3 grid, cudaStream_t s, bool pdl = false, int mb = 0)
{
    // register-bound variants (stencil order 4 only)
    if constexpr (LC == 4) {
        if (mb == 4) return launch_step(k_bwd_p<4, false, 4>, grid, s, pdl, a);
        if (mb == 6) return launch_step(k_bwd_p<4, false, 6>, grid, s, pdl, a);
    }
    launch_step(k_bwd_p<LC>, grid, s, pdl, a);
}

template <int LC>
static void launch_bwd_rcv_v(const BwdArgs &a, dim3 grid, cudaStream_t s, bool pdl = false) { launch_step(k_bwd_rcv_v<LC>, grid, s, pdl, a); }

template <int LC>
static void launch_bwd_rcv_p(const BwdArgs &a, dim3 grid, cudaStream_t s, bool pdl = false) { launch_step(k_bwd_rcv_p<LC>, grid, s, pdl, a); }

template <int LC>
static void launch_fwd_fused(const FStepArgs &a, int nw, cudaStream_t s)
{
    const dim3 grid((a.g.ntz + FTZ - 1) / FTZ, (a.g.ntx + FTX - 1) / FTX);
    if (nw == 2) k_fwd_step<LC, 2, FTX, FTZ><<<grid, 256, 0, s>>>(a);
    else k_fwd_step<LC, 1, FTX, FTZ><<<grid, 256, 0, s>>>(a);
}

template <int LC>
static void launch_bwd_fused(const BStepArgs &a, cudaStream_t s)
{
    const dim3 grid((a.g.ntz + FTZ - 1) / FTZ, (a.g.ntx + FTX - 1) / FTX);
    k_bwd_step<LC, FTX, FTZ><<<grid, 256, 0, s>>>(a);
}

#define LC_DISPATCH6(LCV, FN, ...)                               \
    switch (LCV) {                                               \
        case 1: FN<1>(__VA_ARGS__); break;                       \
        case 2: FN<2>(__VA_ARGS__); break;                       \
        case 3: FN<3>(__VA_ARGS__); break;                       \
        case 4: FN<4>(__VA_ARGS__); break;                       \
        case 5: FN<5>(__VA_ARGS__); break;                       \
        default: FN<6>(__VA_ARGS__); break;                      \
    }

#define LC_DISPATCH(LCV, FN, ...)                                \
    switch (LCV) {                                               \
        case 1: FN<1>(__VA_ARGS__); break;                       \
        case 2: FN<2>(__VA_ARGS__); break;                       \
        case 3: FN<3>(__VA_ARGS__); break;                       \
        case 4: FN<4>(__VA_ARGS__); break;                       \
        case 5: FN<5>(__VA_ARGS__); break;                       \
        case 6: FN<6>(__VA_ARGS__); break;                       \
        case 7: FN<7>(__VA_ARGS__); break;                       \
        default: FN<8>(__VA_ARGS__); break;                      \
    }

// twiddle table exp(-2 pi i j / N), j < N/2, built in double on the host
static int make_twiddles(swd_ctx *ctx, DevBuf &buf, int N)
{
    std::vector<float2> h(N / 2);
    for (int j = 0; j < N / 2; j++) {
        const double a = -2.0 * M_PI * (double)j / (double)N;
        h[j] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    CKR(ensure(ctx, buf, sizeof(float2) * h.size()));
    CK(cudaMemcpyAsync(buf.p, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SWD_OK;
}

static int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}

// ------------------------------------------------------------------------------------
// forward pass shared by swd_forward and swd_rtm_shot
// ------------------------------------------------------------------------------------
struct FwdJob {
    const swd_shot *shot;
    std::vector<float> rick, hrick;
    bool twin = false, save_strips = false;
    float *seis_dev = nullptr;
    float2 *colbuf = nullptr;
    // Born: field 1 is the scattered field (no wavelet, secondary source dt*dkappa*S0)
    const float *dkappa = nullptr;
    float *s0 = nullptr;     // background p-update sums, slot it % s0_mod
    int s0_mod = 1;
    Ckpt ck{};               // background checkpoints (ck.every == 0: none)
    DpStore ds{};            // stored source dp/dt (ds.buf == nullptr: none)
    // exact scattered field: field 1 = u(perturbed model) - u(background), no wavelet of its
    // own; colcomp: the colbuf component it records (-1: the twin pair)
    bool scat = false;
    int colcomp = -1;
};

// device copies of the shot's wavelet(s): wav[0..nt) = rick, wav[nt..2nt) = Hilbert twin
static int upload_wavelets(swd_ctx *ctx, const FwdJob &J, int nt)
{
    CKR(ensure(ctx, ctx->wav, sizeof(float) * 2 * (size_t)ctx->grid.nt_max));
    CK(cudaMemcpyAsync(F(ctx->wav), J.rick.data(), sizeof(float) * nt, cudaMemcpyHostToDevice, ctx->stream));
    if (J.twin && (J.dkappa || J.scat)) CK(cudaMemsetAsync(F(ctx->wav) + nt, 0, sizeof(float) * nt, ctx->stream));
    else if (J.twin) CK(cudaMemcpyAsync(F(ctx->wav) + nt, J.hrick.data(), sizeof(float) * nt, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));   // the host vectors may go away after this
    return SWD_OK;
}

static int strip_len(const swd_ctx *c) { return 2 * c->Lc * c->nx + 2 * c->Lc * (c->nz - 2 * c->Lc); }


// ------------------------------------------------------------------------------------
// Chunked graph execution of a time loop.  The step kernels read their time index from a
// device counter (it = *counter + itoff), so one captured graph of K steps followed by a
// one-thread counter advance serves every chunk; it is replayed nsteps/K times and the
// remaining steps are launched directly.  The graph is re-captured only when the step
// arguments (pointers, geometry, shot) change.  When profiling is on, each chunk is replayed
// from a probe copy whose first step is bracketed by event nodes, read after the chunk.
// ------------------------------------------------------------------------------------
constexpr int GRAPH_K = 64;

__global__ void k_advance(int *counter, int d) { *counter += d; }

static void graph_free(swd_ctx::StepGraph &G)
{
    if (G.exec) cudaGraphExecDestroy(G.exec);
    if (G.probe) cudaGraphExecDestroy(G.probe);
    for (cudaEvent_t e : G.ev) cudaEventDestroy(e);
    G = swd_ctx::StepGraph();
}

// variant of the next pass of a tuner: the chosen one, else the next one to try
// Whether a pass that touches `arrays` full-grid float arrays per step streams them from HBM
// (its working set exceeds L2).  Such passes run the register-bound velocity kernels by default
// (6 blocks of 256 per SM): with the data in HBM the extra resident warps keep more bytes in
// flight, while an L2-resident pass is faster with the unbounded kernels.  Same bits either way.
static bool streams_hbm(const swd_ctx *ctx, int arrays)
{
    return (size_t)ctx->ntx * ctx->ldz * sizeof(float) * arrays > ctx->l2_bytes;
}

static int tune_pick(const swd_ctx::PassTune &T) { return T.choice >= 0 ? T.cand[T.choice] : T.cand[T.next]; }

static void tune_record(swd_ctx::PassTune &T, double ms_per_step)
{
    if (T.choice >= 0) return;
    T.ms[T.next++] = ms_per_step;
    if (T.next < T.ncand) return;
    int best = 0;
    for (int i = 1; i < T.ncand; i++)
        if (T.ms[i] < T.ms[best]) best = i;
    T.choice = best;
}

static void tune_reset(swd_ctx::PassTune &T, std::initializer_list<int> cands)
{
    T = swd_ctx::PassTune();
    for (int c : cands) T.cand[T.ncand++] = c;
}

template <class Launch>
static int capture_chunk(swd_ctx *ctx, cudaGraphExec_t *out, int dir, int *counter, Launch launch, cudaEvent_t *ev,
                         int klen)
{
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < klen; k++) launch(k, k == klen / 2 ? ev : nullptr);
    k_advance<<<1, 1, 0, ctx->stream>>>(counter, dir * klen);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (e != cudaSuccess) return fail(ctx, SWD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, SWD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return SWD_OK;
}

// Launch(k, ev): enqueue step k (itoff = dir*k) on ctx->stream; when ev != nullptr record
// ev[2j] / ev[2j+1] around its j-th kernel.  nk kernels per step with profiling ids kid[].
// Chunks hold klen steps (the key of the captured graph includes it).
// pass_ms: when given, the pass's replays (captures excluded) are timed with events and the
// milliseconds returned there (the stream is synchronised for it).
template <class Launch>
static int run_steps(swd_ctx *ctx, swd_ctx::StepGraph &G, const void *key, size_t keylen, int start, int dir,
                     int nsteps, int nk, const int *kid, Launch launch, int klen = GRAPH_K, int pass_id = -1,
                     float *pass_ms = nullptr)
{
    CKR(ensure(ctx, ctx->ctrl, 64));
    int *counter = I32(ctx->ctrl);
    CK(cudaMemcpyAsync(counter, &start, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    // the legacy default stream (handle 0) cannot be captured: launch directly there
    const int nchunks = (ctx->use_graphs && ctx->stream != nullptr) ? nsteps / klen : 0;
    const int rem = nsteps - nchunks * klen;
    const bool prof = ctx->prof_every > 0;
    if (nchunks > 0) {
        std::vector<char> k2((const char *)key, (const char *)key + keylen);
        k2.insert(k2.end(), (const char *)&klen, (const char *)&klen + sizeof klen);
        const bool same = G.exec && G.key == k2;
        if (!same) {
            graph_free(G);
            G.key = k2;
            CKR(capture_chunk(ctx, &G.exec, dir, counter, launch, nullptr, klen));
        }
        if (prof && !G.probe) {
            G.ev.resize(2 * nk);
            for (auto &e : G.ev) CK(cudaEventCreate(&e));
            CKR(capture_chunk(ctx, &G.probe, dir, counter, launch, G.ev.data(), klen));
        }
    }
    const int pc = prof && nchunks > 0 ? nchunks / 2 : -1;   // the chunk that carries the probe events
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (pass_ms) {
        t0 = ev_get(ctx);
        t1 = ev_get(ctx);
        if (!t0 || !t1) return fail(ctx, SWD_ERR_CUDA, "no timing events");
        CK(cudaEventRecord(t0, ctx->stream));
    }
    {
        // whole-pass time per step (profiling ids 6 forward, 7 backward)
        ProfScope pass(ctx, pass_id >= 0 ? pass_id : (dir > 0 ? 6 : 7), prof, nsteps);
        for (int c = 0; c < nchunks; c++) {
            CK(cudaGraphLaunch(c == pc ? G.probe : G.exec, ctx->stream));
            ctx->launches += (long long)nk * klen;
        }
        for (int k = 0; k < rem; k++) {
            launch(k, nullptr);
            ctx->launches += nk;
        }
    }
    CK(cudaGetLastError());
    if (pass_ms) {
        CK(cudaEventRecord(t1, ctx->stream));
        CK(cudaEventSynchronize(t1));
        CK(cudaEventElapsedTime(pass_ms, t0, t1));
    }
    if (pc >= 0) {
        // the probe step sits mid-chunk between busy neighbours; read it once the pass drained
        CK(cudaStreamSynchronize(ctx->stream));
        for (int j = 0; j < nk; j++) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, G.ev[2 * j], G.ev[2 * j + 1]) == cudaSuccess) {
                ctx->prof_ms[kid[j]] += ms;
                ctx->prof_n[kid[j]] += 1;
            }
        }
    }
    return SWD_OK;
}

static int run_forward_fused(swd_ctx *ctx, FwdJob &J, ShotPlan &P);

static int run_forward(swd_ctx *ctx, FwdJob &J, ShotPlan &P)
{
    ctx->kept.valid = false;   // wave[0], strips and the wavelet buffer are overwritten
    // Born fields, S0 output and checkpoints exist on the plain kernels only
    if (fused(ctx) && !J.dkappa && !J.s0 && !J.ck.every && !J.ds.buf && !J.scat) return run_forward_fused(ctx, J, P);
    const swd_shot *s = J.shot;
    const int nt = s->nt;
    CKR(zero_wave(ctx, 0));
    if (J.twin) CKR(zero_wave(ctx, 1));
    FwdArgs a;
    memset(&a, 0, sizeof a);
    a.g = make_geo(ctx);
    a.c = make_cpml(ctx);
    a.vp = F(ctx->vp);
    a.rho = F(ctx->rho);
    a.m = make_mat(ctx);
    a.w[0] = make_wave(ctx, 0);
    a.w[1] = J.twin ? make_wave(ctx, 1) : make_wave(ctx, 0);
    a.sx = s->s_ix;
    a.sz = s->s_iz;
    a.nt = nt;
    a.wells.wcol = I32(ctx->wcol);
    a.wells.wmap = I32(ctx->wmap);
    a.seis = J.seis_dev;
    a.colmap = J.colbuf ? I32(ctx->wcol) : nullptr;
    a.colbuf = J.colbuf;
    a.s0_out = J.s0;
    a.s0_stride = (long long)ctx->ntx * ctx->ldz;
    a.s0_mod = J.s0_mod;
    a.dkappa = J.dkappa;
    a.ck = J.ck;
    a.ds = J.ds;
    a.colcomp = J.colcomp;
    if (J.scat) {
        a.m1 = make_mat1(ctx);
        a.dcbx = F(ctx->dmat[0]);
        a.dcbz = F(ctx->dmat[1]);
        a.dck = F(ctx->dmat[2]);
    }
    const dim3 grid = grid_blocks(ctx);
    if (J.save_strips) {
        const int slen = strip_len(ctx);
        const int nscale = grid.x * grid.y;
        const size_t esz = ctx->strip_prec == SWD_STRIP_F32 ? 4 : 2;
        CKR(ensure(ctx, ctx->strips, esz * (size_t)slen * nt));
        a.strips.buf = ctx->strips.p;
        a.strips.slen = slen;
        a.strips.prec = ctx->strip_prec;
        a.strips.nscale = nscale;
        if (ctx->strip_prec != SWD_STRIP_F32) {
            CKR(ensure(ctx, ctx->strip_scale, sizeof(float) * (size_t)nscale * nt));
            a.strips.scale = F(ctx->strip_scale);
        }
    }
    CKR(upload_wavelets(ctx, J, nt));
    CKR(ensure(ctx, ctx->ctrl, 64));
    a.itp = I32(ctx->ctrl);
    a.wav0 = F(ctx->wav);
    a.wav1 = J.twin ? F(ctx->wav) + nt : F(ctx->wav);
    const int nw = J.twin ? 2 : 1;
    // one wavefield without checkpoints: the velocity kernel with TMA-staged pressure
    // the plain single-wavefield forward (RTM forward, modelling without a twin): variants of the
    // velocity and pressure launches, chosen by the tuner when SWD_OPT_AUTOTUNE is on
    const bool plain1 = nw == 1 && !a.ck.every && !a.ds.buf && !a.s0_out && !a.dkappa && !a.dck;
    const bool tune = ctx->autotune && plain1;
    // variant bits: 1 TMA velocity launch, 2 staged pressure launch, 8 / 16 pressure kernel at 4 / 6
    // blocks per SM, 32 velocity kernel at 6 blocks per SM (p, vx, vz and three coefficients a step;
    // the stored-source forward also streams its dp/dt store out every step)
    const int fv = tune ? tune_pick(ctx->tfwd)
                        : ((ctx->use_tma ? 1 : 0) | (ctx->use_staged ? 2 : 0) |
                           (streams_hbm(ctx, 6) || a.ds.buf ? 32 : 0));
    int use_tma = (fv & 1) && nw == 1 && !a.ck.every;
    CUtensorMap pmap;
    TmaShape tsh;
    if (use_tma) {
        int rows = 0, cols = 0;
        LC_DISPATCH(ctx->Lc, tma_box, &rows, &cols);
        LC_DISPATCH(ctx->Lc, tma_prepare, ctx->dev, 1, &tsh);
        use_tma = tsh.nblk > 0 && make_pmap(ctx, &pmap, a.w[0].p, rows, cols);
        if (use_tma) CK(cudaMemsetAsync(tma_err(ctx), 0, sizeof(int), ctx->stream));
    }
    // one plain wavefield: the pressure kernel with every stencil operand staged by TMA
    int use_staged = (fv & 2) && plain1;
    const int fmb = plain1 ? ((fv & 8) ? 4 : (fv & 16) ? 6 : 0) : 0;   // register-bound variants
    const int vmb = nw == 1 && !a.ck.every && (fv & 32) ? 6 : 0;
    CUtensorMap smap[4];
    TmaShape ssh;
    if (use_staged) {
        bool ok = false;
        LC_DISPATCH(ctx->Lc, staged_p_prepare, ctx->dev, &ssh);
        if (ssh.nblk > 0) LC_DISPATCH(ctx->Lc, staged_p_maps, ctx, a, smap, &ok);
        use_staged = ok;
        if (use_staged) CK(cudaMemsetAsync(tma_err(ctx), 0, sizeof(int), ctx->stream));
    }
    auto launch = [&](int k, cudaEvent_t *ev) {
        FwdArgs b = a;
        b.itoff = k;
        if (ev) cudaEventRecordWithFlags(ev[0], ctx->stream, cudaEventRecordExternal);
        if (use_tma) {
            LC_DISPATCH(ctx->Lc, launch_fwd_v_tma, b, pmap, tma_err(ctx), tsh, ctx->stream);
        } else {
            LC_DISPATCH(ctx->Lc, launch_fwd_v, b, nw, grid, ctx->stream, ctx->use_pdl, vmb);
        }
        if (ev) { cudaEventRecordWithFlags(ev[1], ctx->stream, cudaEventRecordExternal); cudaEventRecordWithFlags(ev[2], ctx->stream, cudaEventRecordExternal); }
        if (use_staged) {
            LC_DISPATCH(ctx->Lc, launch_fwd_p_staged, b, smap, tma_err(ctx), ssh, ctx->stream);
        } else {
            LC_DISPATCH(ctx->Lc, launch_fwd_p, b, nw, grid, ctx->stream, ctx->use_pdl, fmb);
        }
        if (ev) cudaEventRecordWithFlags(ev[3], ctx->stream, cudaEventRecordExternal);
    };
    const int kid[2] = {0, 1};
    a.itoff = 0;
    // the TMA choices are part of the captured graph's identity
    std::vector<char> key((const char *)&a, (const char *)&a + sizeof a);
    key.insert(key.end(), (const char *)&use_tma, (const char *)&use_tma + sizeof use_tma);
    key.insert(key.end(), (const char *)&use_staged, (const char *)&use_staged + sizeof use_staged);
    key.insert(key.end(), (const char *)&fmb, (const char *)&fmb + sizeof fmb);
    key.insert(key.end(), (const char *)&vmb, (const char *)&vmb + sizeof vmb);
    key.insert(key.end(), (const char *)&ctx->use_pdl, (const char *)&ctx->use_pdl + sizeof ctx->use_pdl);
    float pass_ms = 0.f;
    const bool timing = tune && ctx->tfwd.choice < 0;
    CKR(run_steps(ctx, ctx->gfwd, key.data(), key.size(), 0, +1, nt, 2, kid, launch, GRAPH_K, -1,
                  timing ? &pass_ms : nullptr));
    if (use_tma || use_staged) CKR(tma_check(ctx));
    if (timing) tune_record(ctx->tfwd, pass_ms / nt);
    return SWD_OK;
}

// Fused forward: step it reads copy it%2 and writes copy (it+1)%2 of every double-buffered
// array; the final state ends in copy nt%2.
static int run_forward_fused(swd_ctx *ctx, FwdJob &J, ShotPlan &P)
{
    const swd_shot *s = J.shot;
    const int nt = s->nt;
    const int nw = J.twin ? 2 : 1;
    for (int k = 0; k < nw; k++) {
        CKR(zero_wave(ctx, k));
        CKR(zero_wave2(ctx, k));
    }
    FStepArgs a;
    memset(&a, 0, sizeof a);
    a.g = make_geo(ctx);
    a.c = make_cpml(ctx);
    a.vp = F(ctx->vp);
    a.rho = F(ctx->rho);
    a.sx = s->s_ix;
    a.sz = s->s_iz;
    a.nt = nt;
    a.wells.wcol = I32(ctx->wcol);
    a.wells.wmap = I32(ctx->wmap);
    a.seis = J.seis_dev;
    a.colmap = J.colbuf ? I32(ctx->wcol) : nullptr;
    a.colbuf = J.colbuf;
    const dim3 grid = fused_blocks(ctx);
    if (J.save_strips) {
        const int slen = strip_len(ctx);
        const int nscale = grid.x * grid.y;
        const size_t esz = ctx->strip_prec == SWD_STRIP_F32 ? 4 : 2;
        CKR(ensure(ctx, ctx->strips, esz * (size_t)slen * nt));
        a.strips.buf = ctx->strips.p;
        a.strips.slen = slen;
        a.strips.prec = ctx->strip_prec;
        a.strips.nscale = nscale;
        if (ctx->strip_prec != SWD_STRIP_F32) {
            CKR(ensure(ctx, ctx->strip_scale, sizeof(float) * (size_t)nscale * nt));
            a.strips.scale = F(ctx->strip_scale);
        }
    }
    CKR(upload_wavelets(ctx, J, nt));
    CKR(ensure(ctx, ctx->ctrl, 64));
    a.itp = I32(ctx->ctrl);
    a.wav0 = F(ctx->wav);
    a.wav1 = J.twin ? F(ctx->wav) + nt : F(ctx->wav);
    a.w[0] = make_field2(ctx, 0, 0);
    a.w[1] = nw == 2 ? make_field2(ctx, 1, 0) : a.w[0];
    auto launch = [&](int k, cudaEvent_t *ev) {
        // chunks start at even steps, so step k of a chunk reads copy k%2
        FStepArgs b = a;
        b.itoff = k;
        b.w[0] = make_field2(ctx, 0, k & 1);
        b.w[1] = nw == 2 ? make_field2(ctx, 1, k & 1) : b.w[0];
        if (ev) cudaEventRecordWithFlags(ev[0], ctx->stream, cudaEventRecordExternal);
        LC_DISPATCH6(ctx->Lc, launch_fwd_fused, b, nw, ctx->stream);
        if (ev) cudaEventRecordWithFlags(ev[1], ctx->stream, cudaEventRecordExternal);
    };
    const int kid[1] = {4};
    a.itoff = 0;
    return run_steps(ctx, ctx->gfwd, &a, sizeof a, 0, +1, nt, 1, kid, launch);
}

static int check_ready(swd_ctx *ctx)
{
    if (!ctx) return SWD_ERR_ARG;
    if (!ctx->have_rc) return fail(ctx, SWD_ERR_STATE, "stencil coefficients not set (swd_set_stencil)");
    if (!ctx->have_cpml) return fail(ctx, SWD_ERR_STATE, "CPML profiles not set (swd_set_cpml)");
    if (!ctx->have_model) return fail(ctx, SWD_ERR_STATE, "model not set (swd_set_model)");
    CK(cudaSetDevice(ctx->dev));
    return SWD_OK;
}


// ------------------------------------------------------------------------------------
// decon geometry (kk_decon_interp_psf_minewindow.cpp:84-132)
// ------------------------------------------------------------------------------------
static int decon_geo(const swd_decon_params *p, DeconGeo &g)
{
    if (!p || p->nx < 1 || p->nz < 1) return SWD_ERR_ARG;
    if (p->psfwinx % 2 == 0 || p->psfwinz % 2 == 0 || p->filterwinx % 2 == 0 || p->filterwinz % 2 == 0) return SWD_ERR_ARG;
    if (p->psfwinx < 1 || p->psfwinz < 1 || p->snapwinx < 2 || p->snapwinz < 2) return SWD_ERR_ARG;
    memset(&g, 0, sizeof g);
    g.nx = p->nx; g.nz = p->nz;
    g.psfwinx = p->psfwinx; g.psfwinz = p->psfwinz; g.filterwinx = p->filterwinx; g.filterwinz = p->filterwinz;
    g.snapwinx = p->snapwinx; g.snapwinz = p->snapwinz; g.epsilon = p->epsilon;
    if (p->psf_interp != 0 && p->psf_interp != 1) return SWD_ERR_ARG;
    g.psf_interp = p->psf_interp;
    g.halfpsfwx = p->psfwinx / 2; g.halfpsfwz = p->psfwinz / 2;
    g.halfltwx = p->filterwinx / 2; g.halfltwz = p->filterwinz / 2;
    g.nzwpsf = (int)ceil(1.0 * p->nz / p->psfwinz);
    g.nxwpsf = (int)ceil(1.0 * p->nx / p->psfwinx);
    const int fullwx = p->filterwinx + p->psfwinx - 1, fullwz = p->filterwinz + p->psfwinz - 1;
    if (p->fft_nx > 0 && p->fft_nz > 0) {
        if (p->fft_nx < fullwx || p->fft_nz < fullwz) return SWD_ERR_ARG;
        g.FX = p->fft_nx; g.FZ = p->fft_nz; g.n0 = g.FX; g.n1 = g.FZ;
    } else {
        g.FX = fullwx; g.FZ = fullwz; g.n0 = fullwz; g.n1 = fullwx;
    }
    g.midpx = g.FX / 2; g.midpz = g.FZ / 2;
    g.ocx = g.midpx - g.halfpsfwx; g.ocz = g.midpz - g.halfpsfwz;
    g.outwinx = 2 * (p->psfwinx / 10) + 2 * p->snapwinx + 1;
    g.outwinz = 2 * (p->psfwinz / 10) + 2 * p->snapwinz + 1;
    g.halfoutwx = g.outwinx / 2; g.halfoutwz = g.outwinz / 2;
    g.stepwinx = g.outwinx - p->snapwinx; g.stepwinz = g.outwinz - p->snapwinz;
    g.stepnumx = (int)ceil(1.0 * (p->nx + fullwx) / g.stepwinx) + 1;
    g.stepnumz = (int)ceil(1.0 * (p->nz + fullwz) / g.stepwinz) + 1;
    g.totalnum = g.stepnumx * g.stepnumz;
    g.nxp = g.stepnumx * g.stepwinx; g.nzp = g.stepnumz * g.stepwinz;
    if (p->filterwinx < p->psfwinx || p->filterwinz < p->psfwinz) return SWD_ERR_ARG;
    if (p->filterwinx < g.outwinx || p->filterwinz < g.outwinz) return SWD_ERR_ARG;
    if (g.n0 > 512 || g.n1 > 512) return SWD_ERR_ARG;
    if (p->workspace != 0 && p->workspace != 1) return SWD_ERR_ARG;
    // the buffer and the transform tables in shared memory when they fit in 220 KB (of the
    // 227 KB a CTA may have), else the buffer in a global workspace
    g.staged = p->workspace == 1 || ((size_t)g.FX * g.FZ + decon_tab_len(g)) * 8 > 220 * 1024;
    if (p->iters < 0 || p->iters > 100000 || !(p->reg_l1 >= 0.0f) || !(p->reg_l2 >= 0.0f)) return SWD_ERR_ARG;
    g.iters = p->iters;
    g.reg_l1 = p->reg_l1;
    g.reg_l2 = p->reg_l2;
    // the PSF lattice must hold at least 7 cells per axis so the clamp range [3, n-4] exists
    if (g.nxwpsf < 7 || g.nzwpsf < 7) return SWD_ERR_ARG;
    return SWD_OK;
}

// Launch shape of the persistent window kernel (staged transforms or the iterative option): a
// 96 KB shared chunk when staged, else the buffer in shared memory; as many CTAs as are
// resident at once, each owning decon_ws_floats(g) floats of workspace.
static bool decon_persistent(const DeconGeo &g) { return g.staged || g.iters > 0; }
static size_t decon_staged_cap(const DeconGeo &g) { return std::max<size_t>(12288, std::max(g.n0, g.n1)); }
static size_t decon_ws_smem(const DeconGeo &g)
{
    return sizeof(float2) * (decon_tab_len(g) + (g.staged ? decon_staged_cap(g) : (size_t)g.FX * g.FZ));
}
static const void *decon_ws_kernel(const DeconGeo &g)
{
    return g.staged ? (const void *)k_decon_window_ws<true> : (const void *)k_decon_window_ws<false>;
}
// CTAs of the persistent window kernel, or -1 when a CUDA query fails (the error is cleared).
static int decon_ws_blocks(const DeconGeo &g, int dev)
{
    int nsm = 0, occ = 0;
    const size_t sm = decon_ws_smem(g);
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(decon_ws_kernel(g), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, decon_ws_kernel(g), 512, sm) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return std::max(1, std::min(g.totalnum, nsm * std::max(occ, 1)));
}

// Window kernel of g: the transform tables are built into tabs (decon_tab_len(g) float2),
// then one CTA per window in shared memory, or nblk persistent CTAs over the workspace ws
// (staged transforms or iterations).  Two launches (three when n1 != n0).
static cudaError_t launch_decon_windows(const DeconGeo &g, const float *mig, const float *psf, float *winout,
                                        float *ws, int nblk, float2 *tabs, cudaStream_t st)
{
    k_wfft_tables<<<(int)((wfft_table_len(g.n0) + 63) / 64), 64, 0, st>>>(tabs, g.n0);
    if (g.n1 != g.n0) k_wfft_tables<<<(int)((wfft_table_len(g.n1) + 63) / 64), 64, 0, st>>>(tabs + wfft_table_len(g.n0), g.n1);
    if (decon_persistent(g)) {
        const size_t sm = decon_ws_smem(g);
        cudaError_t e = cudaFuncSetAttribute(decon_ws_kernel(g), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        if (g.staged) k_decon_window_ws<true><<<nblk, 512, sm, st>>>(g, mig, psf, winout, ws, (int)decon_staged_cap(g), tabs);
        else k_decon_window_ws<false><<<nblk, 512, sm, st>>>(g, mig, psf, winout, ws, 0, tabs);
    } else {
        const size_t sm = sizeof(float2) * ((size_t)g.FX * g.FZ + decon_tab_len(g));
        cudaError_t e = cudaFuncSetAttribute(k_decon_window, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        // two CTAs of 256 threads per SM where two windows' buffers fit in shared memory (one CTA's
        // barriers then overlap the other's transforms), else one CTA of 512; a window's result
        // does not depend on the block size (one warp per transform, order-free maximum)
        const int nthr = 2 * (sm + 1024) <= 227 * 1024 ? 256 : 512;
        k_decon_window<<<g.totalnum, nthr, sm, st>>>(g, mig, psf, winout, tabs);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Static scratch of swd_decon_noalloc: the per-window result slots and the output taper of
// one deconvolution, so that entry point never allocates.  Every device that loads this
// library holds the 16 MiB array until the process exits; all calls share it.
// ------------------------------------------------------------------------------------
static __device__ __align__(256) float g_decon_scratch[SWD_DECON_STATIC_SCRATCH_FLOATS];

// Hann-edged output taper on the device (same expression as the host taper of swd_decon,
// kk_decon_interp_psf_minewindow.cpp:355-383), written into the static scratch.
__global__ void k_decon_taper(float *coefr, int outwinx, int outwinz, int snapwinx, int snapwinz)
{
    const double PI = 3.1415926;
    const int n = outwinx * outwinz;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int ix = j / outwinz, iz = j % outwinz;
        float cx, cz;
        if (ix <= snapwinx - 1) cx = 0.5000 - 0.5 * cos(PI * ix / (snapwinx - 1));
        else if (ix >= outwinx - snapwinx) cx = 0.5000 + 0.5 * cos(PI * (ix - outwinx + snapwinx) / (snapwinx - 1));
        else cx = 1.0;
        if (iz <= snapwinz - 1) cz = 0.5000 - 0.5 * cos(PI * iz / (snapwinz - 1));
        else if (iz >= outwinz - snapwinz) cz = 0.5000 + 0.5 * cos(PI * (iz - outwinz + snapwinz) / (snapwinz - 1));
        else cz = 1.0;
        coefr[j] = cx * cz;
    }
}

// ------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------
extern "C" {

int swd_version(void) { return 10000; }

int swd_device_count(int *n)
{
    if (!n) return SWD_ERR_ARG;
    cudaError_t e = cudaGetDeviceCount(n);
    if (e != cudaSuccess) { *n = 0; return SWD_ERR_CUDA; }
    return SWD_OK;
}

int swd_create(swd_ctx **out, const swd_grid *g)
{
    if (!out || !g) return SWD_ERR_ARG;
    *out = nullptr;
    if (g->nx < 1 || g->nz < 1 || g->pml < 0 || g->Lc < 1 || g->Lc > MAXLC || g->nt_max < 2 || !(g->dx > 0) ||
        !(g->dz > 0) || !(g->dt > 0))
        return SWD_ERR_ARG;
    if (g->nx < 2 * g->Lc + 1 || g->nz < 2 * g->Lc + 1) return SWD_ERR_ARG;
    swd_ctx *ctx = new swd_ctx();
    ctx->grid = *g;
    ctx->dev = g->device;
    ctx->Lc = g->Lc;
    ctx->pmlc = g->pml + g->Lc;
    ctx->nx = g->nx;
    ctx->nz = g->nz;
    ctx->ntx = g->nx + 2 * ctx->pmlc;
    ctx->ntz = g->nz + 2 * ctx->pmlc;
    ctx->ldz = (ctx->ntz + 31) / 32 * 32;
    cudaError_t e = cudaSetDevice(ctx->dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    // the L2 size only picks default register bounds (same bits either way): a failed query
    // leaves 0, which counts every pass as streaming from HBM
    int l2 = 0;
    if (e == cudaSuccess && cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ctx->dev) != cudaSuccess) {
        cudaGetLastError();
        l2 = 0;
    }
    ctx->l2_bytes = (size_t)l2;
    if (e != cudaSuccess) {
        delete ctx;
        return SWD_ERR_CUDA;
    }
    *out = ctx;
    return SWD_OK;
}

int swd_destroy(swd_ctx *ctx)
{
    if (!ctx) return SWD_OK;
    cudaSetDevice(ctx->dev);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (DevBuf *b : ctx->bufs)
        if (b->p) cudaFree(b->p);
    prof_collect(ctx);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    graph_free(ctx->gfwd);
    graph_free(ctx->gbwd);
    graph_free(ctx->gseg);
    graph_free(ctx->gadj);
    graph_free(ctx->gbf);
    graph_free(ctx->gbb);
    if (ctx->stream && ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SWD_OK;
}

const char *swd_last_error(const swd_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int swd_set_stream(swd_ctx *ctx, void *stream)
{
    if (!ctx) return SWD_ERR_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (ctx->own_stream && ctx->stream) {
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaStreamDestroy(ctx->stream));
    }
    ctx->stream = (cudaStream_t)stream;
    ctx->own_stream = false;
    return SWD_OK;
}

int swd_synchronize(swd_ctx *ctx)
{
    if (!ctx) return SWD_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    return SWD_OK;
}

size_t swd_device_bytes(const swd_ctx *ctx)
{
    size_t n = 0;
    if (ctx)
        for (const DevBuf *b : ctx->bufs) n += b->n;
    return n;
}

int swd_profile(swd_ctx *ctx, int every)
{
    if (!ctx || every < 0) return SWD_ERR_ARG;
    ctx->prof_every = every;
    return SWD_OK;
}

int swd_profile_read(swd_ctx *ctx, double *ms, long long *launches)
{
    if (!ctx) return SWD_ERR_ARG;
    prof_collect(ctx);
    for (int k = 0; k < SWD_NKERNELS; k++) {
        if (ms) ms[k] = ctx->prof_ms[k];
        if (launches) launches[k] = ctx->prof_n[k];
        ctx->prof_ms[k] = 0.0;
        ctx->prof_n[k] = 0;
    }
    return SWD_OK;
}

long long swd_launch_count(const swd_ctx *ctx) { return ctx ? ctx->launches : 0; }

int swd_set_stencil(swd_ctx *ctx, const float *rc)
{
    if (!ctx || !rc) return fail(ctx, SWD_ERR_ARG, "rc is NULL");
    std::vector<float> h;
    CKR(host_copy(ctx, h, rc, ctx->Lc));
    for (int i = 0; i < MAXLC; i++) ctx->rc[i] = i < ctx->Lc ? h[i] : 0.f;
    ctx->have_rc = true;
    return SWD_OK;
}

int swd_set_cpml(swd_ctx *ctx, const float *a_x, const float *a_x_half, const float *a_z, const float *a_z_half,
                 const float *b_x, const float *b_x_half, const float *b_z, const float *b_z_half)
{
    if (!ctx) return SWD_ERR_ARG;
    const float *src[8] = {a_x, a_x_half, a_z, a_z_half, b_x, b_x_half, b_z, b_z_half};
    CK(cudaSetDevice(ctx->dev));
    for (int i = 0; i < 8; i++) {
        if (!src[i]) return fail(ctx, SWD_ERR_ARG, "CPML array %d is NULL", i);
        const bool xaxis = (i % 4) < 2;
        const int n = xaxis ? ctx->ntx : ctx->ntz;
        const size_t cap = (size_t)(xaxis ? ctx->ntx : ctx->ldz) + 2 * GUARD;
        CKR(ensure(ctx, ctx->cpml[i], sizeof(float) * cap));
        ctx->cpml[i].off = GUARD * sizeof(float);
        CK(cudaMemsetAsync(ctx->cpml[i].p, 0, ctx->cpml[i].n, ctx->stream));
        CKR(to_dev(ctx, F(ctx->cpml[i]), src[i], sizeof(float) * n));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->have_cpml = true;
    // lean box: inside the strip band's inner edge (pmlc + Lc from every side), shrunk to the
    // columns / rows where both a coefficients (integer and half grid) are zero; empty when a
    // nonzero coefficient remains inside
    auto span = [&](const float *a, const float *ah, int n, int *s) {
        int lo = ctx->pmlc + ctx->Lc, hi = n - ctx->pmlc - ctx->Lc;
        while (lo < hi && (a[lo] != 0.f || ah[lo] != 0.f)) lo++;
        while (hi > lo && (a[hi - 1] != 0.f || ah[hi - 1] != 0.f)) hi--;
        bool clean = true;
        for (int i = lo; i < hi; i++) clean = clean && a[i] == 0.f && ah[i] == 0.f;
        s[0] = clean ? lo : 0;
        s[1] = clean ? hi : 0;
    };
    span(a_x, a_x_half, ctx->ntx, ctx->lean);
    span(a_z, a_z_half, ctx->ntz, ctx->lean + 2);
    return SWD_OK;
}

int swd_set_model(swd_ctx *ctx, const float *vp, const float *rho)
{
    if (!ctx || !vp || !rho) return fail(ctx, SWD_ERR_ARG, "vp/rho is NULL");
    CK(cudaSetDevice(ctx->dev));
    // one extra column of padding so the half-node buoyancy reads at x+1 of the last cells
    // stay inside the allocation; guard bands for the vector chunk reads
    CKR(ensure_grid(ctx, ctx->vp, sizeof(float), 1));
    CKR(ensure_grid(ctx, ctx->rho, sizeof(float), 1));
    CK(cudaMemsetAsync(ctx->vp.p, 0, ctx->vp.n, ctx->stream));
    CK(cudaMemsetAsync(ctx->rho.p, 0, ctx->rho.n, ctx->stream));
    CKR(grid_to_dev(ctx, F(ctx->vp), vp));
    CKR(grid_to_dev(ctx, F(ctx->rho), rho));
    for (auto &b : ctx->mat) CKR(ensure_grid(ctx, b, sizeof(float)));
    k_material<<<592, 256, 0, ctx->stream>>>(F(ctx->vp), F(ctx->rho), ctx->grid.dt, ctx->ntx, ctx->ntz, ctx->ldz,
                                             F(ctx->mat[0]), F(ctx->mat[1]), F(ctx->mat[2]), F(ctx->mat[3]));
    ctx->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->have_model = true;
    ctx->have_scatter = false;   // its coefficient differences were formed against the old model
    return SWD_OK;
}

int swd_set_kernel_path(swd_ctx *ctx, int path)
{
    if (!ctx) return SWD_ERR_ARG;
    if (path != SWD_PATH_PLAIN && path != SWD_PATH_FUSED) return fail(ctx, SWD_ERR_ARG, "unknown kernel path %d", path);
    ctx->path = path;
    return SWD_OK;
}

int swd_set_cig(swd_ctx *ctx, int thetan, int delt)
{
    if (!ctx) return SWD_ERR_ARG;
    if (thetan < 3 || thetan > 180 || delt < 1 || delt > 64)
        return fail(ctx, SWD_ERR_ARG, "swd_set_cig: thetan %d outside [3, 180] or delt %d outside [1, 64]", thetan, delt);
    ctx->cig_thetan = thetan;
    ctx->cig_delt = delt;
    return SWD_OK;
}

int swd_rtm_cig(swd_ctx *ctx, float *cig)
{
    if (!ctx || !cig) return SWD_ERR_ARG;
    if (!ctx->have_cig) return fail(ctx, SWD_ERR_STATE, "the last RTM shot accumulated no angle gathers");
    CK(cudaSetDevice(ctx->dev));
    const int th = ctx->cig_thetan;
    // interior cells of each column are contiguous in the [x*ldz + z][thetan] layout
    CK(cudaMemcpy2DAsync(cig, sizeof(float) * (size_t)ctx->nz * th,
                         F(ctx->cig) + ((size_t)ctx->pmlc * ctx->ldz + ctx->pmlc) * th, sizeof(float) * (size_t)ctx->ldz * th,
                         sizeof(float) * (size_t)ctx->nz * th, ctx->nx,
                         is_device_ptr(cig) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SWD_OK;
}

int swd_set_source_storage(swd_ctx *ctx, int store, int prec)
{
    if (!ctx) return SWD_ERR_ARG;
    if (store != 0 && store != 1) return fail(ctx, SWD_ERR_ARG, "source storage mode %d is not 0 or 1", store);
    if (prec < SWD_STRIP_F32 || prec > SWD_STRIP_I16) return fail(ctx, SWD_ERR_ARG, "unknown precision %d", prec);
    ctx->src_store = store;
    ctx->src_prec = prec;
    ctx->kept.valid = false;
    return SWD_OK;
}

int swd_set_strip_precision(swd_ctx *ctx, int prec)
{
    if (!ctx) return SWD_ERR_ARG;
    if (prec < SWD_STRIP_F32 || prec > SWD_STRIP_I16) return fail(ctx, SWD_ERR_ARG, "unknown strip precision %d", prec);
    ctx->strip_prec = prec;
    return SWD_OK;
}

int swd_forward(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *hrick, const float *kz_coef,
                float *seis, float *seis_up, float *seis_down)
{
    CKR(check_ready(ctx));
    if (!rick || !seis) return fail(ctx, SWD_ERR_ARG, "rick and seis are required");
    const bool twin = hrick != nullptr && kz_coef != nullptr;
    if ((seis_up || seis_down) && !twin) return fail(ctx, SWD_ERR_ARG, "seis_up/seis_down need hrick and kz_coef");
    ShotPlan P;
    CKR(plan_shot(ctx, shot, P));
    const int nt = shot->nt, r_n = shot->r_n;
    FwdJob J;
    J.shot = shot;
    CKR(host_copy(ctx, J.rick, rick, nt));
    if (twin) CKR(host_copy(ctx, J.hrick, hrick, nt));
    J.twin = twin;
    CKR(ensure(ctx, ctx->seis, sizeof(float) * (size_t)r_n * nt));
    CK(cudaMemsetAsync(ctx->seis.p, 0, sizeof(float) * (size_t)r_n * nt, ctx->stream));
    J.seis_dev = F(ctx->seis);
    const int N = swd_prep_pow2(ctx->ntz);
    if (twin) {
        CKR(ensure(ctx, ctx->colbuf, sizeof(float2) * (size_t)P.nwells * nt * ctx->ldz));
        J.colbuf = (float2 *)ctx->colbuf.p;
    }
    CKR(run_forward(ctx, J, P));
    CKR(copy_aliases(ctx, P, F(ctx->seis), nt));
    CKR(from_dev(ctx, seis, ctx->seis.p, sizeof(float) * (size_t)r_n * nt));
    if (twin) {
        CKR(ensure(ctx, ctx->kzcoef, sizeof(float) * N));
        CKR(to_dev(ctx, ctx->kzcoef.p, kz_coef, sizeof(float) * N));
        CKR(make_twiddles(ctx, ctx->tw, N));
        CKR(ensure(ctx, ctx->seis2, sizeof(float) * 2 * (size_t)r_n * nt));
        float *up = F(ctx->seis2), *dn = up + (size_t)r_n * nt;
        CK(cudaMemsetAsync(up, 0, sizeof(float) * 2 * (size_t)r_n * nt, ctx->stream));
        const size_t sm = 2 * sizeof(float2) * N;
        CK(cudaFuncSetAttribute(k_kzsep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_kzsep<<<dim3(nt, P.nwells), 256, sm, ctx->stream>>>((const float2 *)ctx->colbuf.p, F(ctx->kzcoef),
                                                               (const float2 *)ctx->tw.p, I32(ctx->wmap), up, dn, nt,
                                                               ctx->ntz, ctx->ldz, N, ilog2(N));
        ctx->launches++;
        CK(cudaGetLastError());
        CKR(copy_aliases(ctx, P, up, nt));
        CKR(copy_aliases(ctx, P, dn, nt));
        if (seis_up) CKR(from_dev(ctx, seis_up, up, sizeof(float) * (size_t)r_n * nt));
        if (seis_down) CKR(from_dev(ctx, seis_down, dn, sizeof(float) * (size_t)r_n * nt));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    return SWD_OK;
}

int swd_set_scatter_model(swd_ctx *ctx, const float *vp1, const float *rho1)
{
    if (!ctx) return SWD_ERR_ARG;
    if (!vp1 && !rho1) {
        ctx->have_scatter = false;
        return SWD_OK;
    }
    if (!vp1 || !rho1) return fail(ctx, SWD_ERR_ARG, "vp1 and rho1 are both required");
    if (!ctx->have_model) return fail(ctx, SWD_ERR_STATE, "set the background model first");
    CK(cudaSetDevice(ctx->dev));
    CKR(ensure_grid(ctx, ctx->vp1, sizeof(float), 1));
    CKR(ensure_grid(ctx, ctx->rho1, sizeof(float), 1));
    CK(cudaMemsetAsync(ctx->vp1.p, 0, ctx->vp1.n, ctx->stream));
    CK(cudaMemsetAsync(ctx->rho1.p, 0, ctx->rho1.n, ctx->stream));
    CKR(grid_to_dev(ctx, F(ctx->vp1), vp1));
    CKR(grid_to_dev(ctx, F(ctx->rho1), rho1));
    for (auto &b : ctx->mat1) CKR(ensure_grid(ctx, b, sizeof(float)));
    for (auto &b : ctx->dmat) CKR(ensure_grid(ctx, b, sizeof(float)));
    k_material<<<592, 256, 0, ctx->stream>>>(F(ctx->vp1), F(ctx->rho1), ctx->grid.dt, ctx->ntx, ctx->ntz, ctx->ldz,
                                             F(ctx->mat1[0]), F(ctx->mat1[1]), F(ctx->mat1[2]), F(ctx->mat1[3]));
    k_material_delta<<<592, 256, 0, ctx->stream>>>(F(ctx->vp), F(ctx->rho), F(ctx->vp1), F(ctx->rho1), ctx->grid.dt,
                                                   ctx->ntx, ctx->ntz, ctx->ldz, F(ctx->dmat[0]), F(ctx->dmat[1]),
                                                   F(ctx->dmat[2]));
    ctx->launches += 2;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->have_scatter = true;
    return SWD_OK;
}

int swd_forward_scatter(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *hrick,
                        const float *kz_coef, float *seis, float *seis_up, float *seis_down)
{
    CKR(check_ready(ctx));
    if (!ctx->have_scatter) return fail(ctx, SWD_ERR_STATE, "no perturbed model (swd_set_scatter_model)");
    if (!rick || !seis) return fail(ctx, SWD_ERR_ARG, "rick and seis are required");
    const bool split = hrick != nullptr && kz_coef != nullptr;
    if ((seis_up || seis_down) && !split) return fail(ctx, SWD_ERR_ARG, "seis_up/seis_down need hrick and kz_coef");
    ShotPlan P;
    CKR(plan_shot(ctx, shot, P));
    const int nt = shot->nt, r_n = shot->r_n;
    const size_t nrec = (size_t)r_n * nt;
    CKR(ensure(ctx, ctx->seis, sizeof(float) * nrec));
    CK(cudaMemsetAsync(ctx->seis.p, 0, sizeof(float) * nrec, ctx->stream));
    if (split) {
        CKR(ensure(ctx, ctx->colbuf, sizeof(float2) * (size_t)P.nwells * nt * ctx->ldz));
        CKR(ensure(ctx, ctx->seis2, sizeof(float) * 2 * nrec));
    }
    // pass 0: the wavelet's background and scattered fields (scattered record; column .x);
    // pass 1, for the up/down split: the Hilbert wavelet's (column .y; its record is dropped)
    for (int pass = 0; pass < (split ? 2 : 1); pass++) {
        FwdJob J;
        J.shot = shot;
        CKR(host_copy(ctx, J.rick, pass == 0 ? rick : hrick, nt));
        J.twin = true;
        J.scat = true;
        J.colcomp = split ? pass : -1;
        J.seis_dev = pass == 0 ? F(ctx->seis) : F(ctx->seis2);
        J.colbuf = split ? (float2 *)ctx->colbuf.p : nullptr;
        CKR(run_forward(ctx, J, P));
    }
    CKR(copy_aliases(ctx, P, F(ctx->seis), nt));
    CKR(from_dev(ctx, seis, ctx->seis.p, sizeof(float) * nrec));
    if (split) {
        const int N = swd_prep_pow2(ctx->ntz);
        CKR(ensure(ctx, ctx->kzcoef, sizeof(float) * N));
        CKR(to_dev(ctx, ctx->kzcoef.p, kz_coef, sizeof(float) * N));
        CKR(make_twiddles(ctx, ctx->tw, N));
        float *up = F(ctx->seis2), *dn = up + nrec;
        CK(cudaMemsetAsync(up, 0, sizeof(float) * 2 * nrec, ctx->stream));
        const size_t sm = 2 * sizeof(float2) * N;
        CK(cudaFuncSetAttribute(k_kzsep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_kzsep<<<dim3(nt, P.nwells), 256, sm, ctx->stream>>>((const float2 *)ctx->colbuf.p, F(ctx->kzcoef),
                                                               (const float2 *)ctx->tw.p, I32(ctx->wmap), up, dn, nt,
                                                               ctx->ntz, ctx->ldz, N, ilog2(N));
        ctx->launches++;
        CK(cudaGetLastError());
        CKR(copy_aliases(ctx, P, up, nt));
        CKR(copy_aliases(ctx, P, dn, nt));
        if (seis_up) CKR(from_dev(ctx, seis_up, up, sizeof(float) * nrec));
        if (seis_down) CKR(from_dev(ctx, seis_down, dn, sizeof(float) * nrec));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    return SWD_OK;
}

// Layout and buffers of the stored dp/dt of an nt-step shot (interior columns, interior rows
// rounded out to 4-cell chunks, one step after another).
static int dp_store_layout(swd_ctx *ctx, int nt, DpStore *ds)
{
    memset(ds, 0, sizeof *ds);
    const dim3 grid = grid_blocks(ctx);
    const int zlo = ctx->pmlc & ~3, zhi = (ctx->ntz - ctx->pmlc + 3) & ~3;
    ds->zlo = zlo;
    ds->ldr = zhi - zlo;
    ds->step = (long long)ctx->nx * ds->ldr;
    ds->prec = ctx->src_prec;
    ds->nwarps = grid.x * grid.y * 8;   // (32, 8) blocks of cell4
    const size_t esz = ctx->src_prec == SWD_STRIP_F32 ? 4 : 2;
    CKR(ensure(ctx, ctx->dpst, esz * (size_t)ds->step * nt));
    ds->buf = ctx->dpst.p;
    if (ctx->src_prec != SWD_STRIP_F32) {
        CKR(ensure(ctx, ctx->dpsc, sizeof(float) * (size_t)ds->nwarps * nt));
        ds->scale = F(ctx->dpsc);
    }
    return SWD_OK;
}

// RTM forward pass: boundary strips saved (or dp/dt stored), the final state stays in wave[0]
// (and in the second copies for the fused path) for rtm_backward_part; the shot is remembered.
static int rtm_forward_part(swd_ctx *ctx, const swd_shot *shot, const float *rick, float *syn)
{
    ShotPlan P;
    CKR(plan_shot(ctx, shot, P));
    const int nt = shot->nt, r_n = shot->r_n;
    const size_t ntr = (size_t)r_n * nt;
    FwdJob J;
    J.shot = shot;
    CKR(host_copy(ctx, J.rick, rick, nt));
    const bool stored = ctx->src_store != 0;
    J.save_strips = !stored;
    if (stored) CKR(dp_store_layout(ctx, nt, &J.ds));
    // the synthetic record is formed only when the caller asks for it (the backward pass uses
    // the observed data)
    if (syn) {
        CKR(ensure(ctx, ctx->seis, sizeof(float) * ntr));
        CK(cudaMemsetAsync(ctx->seis.p, 0, sizeof(float) * ntr, ctx->stream));
        J.seis_dev = F(ctx->seis);
    }
    CKR(run_forward(ctx, J, P));
    if (syn) {
        CKR(copy_aliases(ctx, P, F(ctx->seis), nt));
        CKR(from_dev(ctx, syn, ctx->seis.p, sizeof(float) * ntr));
    }
    ctx->kept = swd_ctx::KeptShotState{true, shot->s_ix, shot->s_iz, shot->nt, shot->r_n, ctx->path, stored};
    return SWD_OK;
}

// RTM backward pass of the shot whose forward pass is kept: receiver data (-int int dt dt),
// source reconstruction + receiver back-propagation + FP64 imaging, per-shot post and stack.
static int rtm_backward_part(swd_ctx *ctx, const swd_shot *shot, const float *data, unsigned flags, float *image_pp,
                             float *image_src, float *fimage)
{
    const swd_ctx::KeptShotState &k = ctx->kept;
    if (!shot) return fail(ctx, SWD_ERR_ARG, "shot is NULL");
    if (!k.valid || k.s_ix != shot->s_ix || k.s_iz != shot->s_iz || k.nt != shot->nt || k.r_n != shot->r_n ||
        k.path != ctx->path)
        return fail(ctx, SWD_ERR_STATE, "the backward pass needs the forward pass of the same shot just before it");
    const bool stored = k.stored;
    ctx->kept.valid = false;   // the reconstruction runs the kept wavefield back to time 0
    ShotPlan P;
    CKR(plan_shot(ctx, shot, P));
    const int nt = shot->nt, r_n = shot->r_n;
    const size_t ntr = (size_t)r_n * nt;
    // 2. receiver data, -int int dt dt
    CKR(ensure(ctx, ctx->rdata, sizeof(float) * 2 * ntr));
    float *raw = F(ctx->rdata), *rms = raw + ntr;
    CKR(to_dev(ctx, raw, data, sizeof(float) * ntr));
    if (flags & SWD_RTM_PREPROCESS) {
        k_preprocess<<<(r_n + 127) / 128, 128, 0, ctx->stream>>>(raw, rms, r_n, nt, ctx->grid.dt);
        ctx->launches++;
        CK(cudaGetLastError());
    } else {
        CK(cudaMemcpyAsync(rms, raw, sizeof(float) * ntr, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    // 3. backward: reconstruction (or the stored dp/dt) + receiver back-propagation + FP64 imaging
    const bool fz = fused(ctx) && !stored;
    const bool want_cig = (flags & SWD_RTM_CIG) != 0;
    ctx->have_cig = false;
    if (want_cig) {
        if (ctx->cig_thetan <= 0) return fail(ctx, SWD_ERR_STATE, "SWD_RTM_CIG needs swd_set_cig first");
        if (fz || stored) return fail(ctx, SWD_ERR_ARG, "angle gathers need the plain kernel path and the reconstructed source");
        const size_t fsz = (size_t)ctx->ntx * ctx->ldz;
        CKR(ensure(ctx, ctx->cig, sizeof(float) * fsz * ctx->cig_thetan));
        CKR(ensure(ctx, ctx->cigring, sizeof(float) * fsz * 2 * ctx->cig_delt));
        CK(cudaMemsetAsync(ctx->cig.p, 0, sizeof(float) * fsz * ctx->cig_thetan, ctx->stream));
        CK(cudaMemsetAsync(ctx->cigring.p, 0, sizeof(float) * fsz * 2 * ctx->cig_delt, ctx->stream));
    }
    CKR(zero_wave(ctx, 1));
    if (fz) {
        CKR(zero_wave2(ctx, 1));
        // both copies of the source wavefield start from the final forward state (copy nt%2)
        const int fpar = nt & 1;
        for (int i = 0; i < 3; i++)
            CK(cudaMemcpyAsync(fcopy(ctx, 0, 1 - fpar, i), fcopy(ctx, 0, fpar, i), grid_bytes(ctx),
                               cudaMemcpyDeviceToDevice, ctx->stream));
    }
    const size_t gb = (size_t)ctx->ntx * ctx->ldz;
    CKR(ensure_grid(ctx, ctx->dpdt, sizeof(float)));
    CK(cudaMemsetAsync(ctx->dpdt.p, 0, ctx->dpdt.n, ctx->stream));
    CKR(ensure_grid(ctx, ctx->I, sizeof(double)));
    CKR(ensure_grid(ctx, ctx->S, sizeof(double)));
    CK(cudaMemsetAsync(ctx->I.p, 0, ctx->I.n, ctx->stream));
    CK(cudaMemsetAsync(ctx->S.p, 0, ctx->S.n, ctx->stream));
    ctx->have_R = (flags & SWD_RTM_ILLUM_RCV) != 0;
    if (ctx->have_R) {
        CKR(ensure_grid(ctx, ctx->R, sizeof(double)));
        CK(cudaMemsetAsync(ctx->R.p, 0, ctx->R.n, ctx->stream));
    }
    const bool blocks = ctx->image_blocks && !fz;
    if (blocks) {
        DevBuf *pb[3] = {&ctx->Ipart, &ctx->Spart, &ctx->Rpart};
        for (int i = 0; i < (ctx->have_R ? 3 : 2); i++) {
            CKR(ensure_grid(ctx, *pb[i], sizeof(float)));
            CK(cudaMemsetAsync(pb[i]->p, 0, pb[i]->n, ctx->stream));
        }
    }
    BwdArgs b;
    memset(&b, 0, sizeof b);
    b.g = make_geo(ctx);
    b.c = make_cpml(ctx);
    b.vp = F(ctx->vp);
    b.rho = F(ctx->rho);
    b.m = make_mat(ctx);
    b.s = make_wave(ctx, 0);
    b.r = make_wave(ctx, 1);
    b.dpdt = F(ctx->dpdt);
    b.sx = shot->s_ix;
    b.sz = shot->s_iz;
    b.nt = nt;
    b.strips.buf = ctx->strips.p;
    b.strips.scale = F(ctx->strip_scale);
    b.strips.slen = strip_len(ctx);
    b.strips.prec = ctx->strip_prec;
    b.strips.nscale = grid_blocks(ctx).x * grid_blocks(ctx).y;
    b.wells.wcol = I32(ctx->wcol);
    b.wells.wmap = I32(ctx->wmap);
    b.rdata = rms;
    b.I = D(ctx->I);
    b.S = D(ctx->S);
    b.R = ctx->have_R ? D(ctx->R) : nullptr;
    b.Ip = blocks ? F(ctx->Ipart) : nullptr;
    b.Sp = blocks ? F(ctx->Spart) : nullptr;
    b.Rp = blocks && ctx->have_R ? F(ctx->Rpart) : nullptr;
    const dim3 grid = grid_blocks(ctx);
    CKR(ensure(ctx, ctx->ctrl, 64));
    if (fz) {
        BStepArgs f;
        memset(&f, 0, sizeof f);
        f.g = b.g; f.c = b.c; f.vp = b.vp; f.rho = b.rho;
        f.sx = b.sx; f.sz = b.sz; f.nt = nt;
        f.strips = b.strips;
        f.strips.nscale = fused_blocks(ctx).x * fused_blocks(ctx).y;
        f.wells = b.wells; f.rdata = b.rdata; f.I = b.I; f.S = b.S; f.R = b.R;
        f.itp = I32(ctx->ctrl);
        f.wavsub = F(ctx->wav);
        const int fpar = nt & 1;
        // step j of the backward loop (it = nt-2-j) reads source copy (fpar + j)%2 and receiver
        // copy j%2; chunks start at even j, so the pattern depends on k = j % GRAPH_K only
        f.r = make_field2(ctx, 1, 0);
        auto launch = [&](int k, cudaEvent_t *ev) {
            BStepArgs q = f;
            q.itoff = -k;
            const int spar = (fpar + k) & 1;
            q.r = make_field2(ctx, 1, k & 1);
            q.ps = fcopy(ctx, 0, spar, 0); q.vxs = fcopy(ctx, 0, spar, 1); q.vzs = fcopy(ctx, 0, spar, 2);
            q.pso = fcopy(ctx, 0, 1 - spar, 0); q.vxso = fcopy(ctx, 0, 1 - spar, 1); q.vzso = fcopy(ctx, 0, 1 - spar, 2);
            if (ev) cudaEventRecordWithFlags(ev[0], ctx->stream, cudaEventRecordExternal);
            LC_DISPATCH6(ctx->Lc, launch_bwd_fused, q, ctx->stream);
            if (ev) cudaEventRecordWithFlags(ev[1], ctx->stream, cudaEventRecordExternal);
        };
        const int kid[1] = {5};
        f.itoff = 0;
        CKR(run_steps(ctx, ctx->gbwd, &f, sizeof f, nt - 2, -1, nt - 1, 1, kid, launch));
    } else if (stored) {
        // receiver wavefield only; the imaging reads the dp/dt stored by the forward pass
        b.itp = I32(ctx->ctrl);
        CKR(dp_store_layout(ctx, nt, &b.ds));
        auto launch = [&](int k, cudaEvent_t *ev) {
            BwdArgs q = b;
            q.itoff = -k;
            if (ev) cudaEventRecordWithFlags(ev[0], ctx->stream, cudaEventRecordExternal);
            LC_DISPATCH(ctx->Lc, launch_bwd_rcv_v, q, grid, ctx->stream, ctx->use_pdl);
            if (ev) { cudaEventRecordWithFlags(ev[1], ctx->stream, cudaEventRecordExternal); cudaEventRecordWithFlags(ev[2], ctx->stream, cudaEventRecordExternal); }
            LC_DISPATCH(ctx->Lc, launch_bwd_rcv_p, q, grid, ctx->stream, ctx->use_pdl);
            if (ev) cudaEventRecordWithFlags(ev[3], ctx->stream, cudaEventRecordExternal);
        };
        const int kid[2] = {2, 3};
        b.itoff = 0;
        std::vector<char> key((const char *)&b, (const char *)&b + sizeof b);
        key.insert(key.end(), (const char *)&ctx->use_pdl, (const char *)&ctx->use_pdl + sizeof ctx->use_pdl);
        CKR(run_steps(ctx, ctx->gbwd, key.data(), key.size(), nt - 2, -1, nt - 1, 2, kid, launch));
    } else {
        b.itp = I32(ctx->ctrl);
        b.wavsub = F(ctx->wav);
        CigArgs cg;
        memset(&cg, 0, sizeof cg);
        if (want_cig) {
            cg.g = b.g; cg.s = b.s; cg.r = b.r; cg.itp = b.itp; cg.nt = nt;
            cg.thetan = ctx->cig_thetan; cg.delt = ctx->cig_delt;
            cg.ring = F(ctx->cigring); cg.cig = F(ctx->cig);
        }
        // phases paired by kind (k_bwd_v + k_bwd_p) unless the angle gathers need the source
        // velocities of every step (k_bwd_1 + k_bwd_2, the reference's pairing)
        // the variants (by-kind pairing with plain or TMA velocities, the reference's pairing)
        // chosen by the tuner when SWD_OPT_AUTOTUNE is on
        const bool tune = ctx->autotune && !want_cig;
        // variant bits: 1 TMA velocity launch, 4 the reference's pairing, 8 / 16 pressure kernel at
        // 4 / 6 blocks per SM, 32 velocity kernel at 6 blocks per SM (two wavefields, four
        // coefficients and the imaging sums: about twelve arrays a step)
        const int bv = tune ? tune_pick(ctx->tbwd)
                            : ((ctx->use_tma ? 1 : 0) | (ctx->bwd_by_kind ? 0 : 4) | (streams_hbm(ctx, 12) ? 32 : 0));
        const int by_kind = !(bv & 4) && !want_cig;
        // velocities of both wavefields with TMA-staged pressures
        int use_tma = by_kind && (bv & 1);
        const int bmb = by_kind ? ((bv & 8) ? 4 : (bv & 16) ? 6 : 0) : 0;   // register-bound variants
        const int bvmb = by_kind && (bv & 32) ? 6 : 0;
        CUtensorMap pmap_r, pmap_s;
        TmaShape tsh;
        if (use_tma) {
            int rows = 0, cols = 0;
            LC_DISPATCH(ctx->Lc, tma_box, &rows, &cols);
            LC_DISPATCH(ctx->Lc, tma_prepare, ctx->dev, 2, &tsh);
            use_tma = tsh.nblk > 0 && make_pmap(ctx, &pmap_r, b.r.p, rows, cols) && make_pmap(ctx, &pmap_s, b.s.p, rows, cols);
            if (use_tma) CK(cudaMemsetAsync(tma_err(ctx), 0, sizeof(int), ctx->stream));
        }
        auto launch = [&](int k, cudaEvent_t *ev) {
            BwdArgs q = b;
            q.itoff = -k;
            if (ev) cudaEventRecordWithFlags(ev[0], ctx->stream, cudaEventRecordExternal);
            if (by_kind && use_tma) {
                LC_DISPATCH(ctx->Lc, launch_bwd_v_tma, q, pmap_r, pmap_s, tma_err(ctx), tsh, ctx->stream);
            } else if (by_kind) {
                LC_DISPATCH(ctx->Lc, launch_bwd_v, q, grid, ctx->stream, ctx->use_pdl, bvmb);
            } else {
                LC_DISPATCH(ctx->Lc, launch_bwd_1, q, grid, ctx->stream, ctx->use_pdl);
            }
            if (ev) { cudaEventRecordWithFlags(ev[1], ctx->stream, cudaEventRecordExternal); cudaEventRecordWithFlags(ev[2], ctx->stream, cudaEventRecordExternal); }
            if (by_kind) {
                LC_DISPATCH(ctx->Lc, launch_bwd_p, q, grid, ctx->stream, ctx->use_pdl, bmb);
            } else if (want_cig) {
                // the gathers fused into the imaging launch
                CigArgs cq = cg;
                cq.itoff = -k;
                LC_DISPATCH(ctx->Lc, launch_bwd_2_cig, q, cq, grid, ctx->stream, ctx->use_pdl);
            } else {
                LC_DISPATCH(ctx->Lc, launch_bwd_2, q, grid, ctx->stream, ctx->use_pdl);
            }
            if (ev) cudaEventRecordWithFlags(ev[3], ctx->stream, cudaEventRecordExternal);
        };
        const int kid[2] = {2, 3};
        b.itoff = 0;
        // the CIG switch and the pairing are part of the captured graph's identity
        std::vector<char> key((const char *)&b, (const char *)&b + sizeof b);
        key.insert(key.end(), (const char *)&cg, (const char *)&cg + sizeof cg);
        key.insert(key.end(), (const char *)&by_kind, (const char *)&by_kind + sizeof by_kind);
        key.insert(key.end(), (const char *)&use_tma, (const char *)&use_tma + sizeof use_tma);
        key.insert(key.end(), (const char *)&bmb, (const char *)&bmb + sizeof bmb);
        key.insert(key.end(), (const char *)&bvmb, (const char *)&bvmb + sizeof bvmb);
        key.insert(key.end(), (const char *)&ctx->use_pdl, (const char *)&ctx->use_pdl + sizeof ctx->use_pdl);
        float pass_ms = 0.f;
        const bool timing = tune && ctx->tbwd.choice < 0;
        CKR(run_steps(ctx, ctx->gbwd, key.data(), key.size(), nt - 2, -1, nt - 1, 2, kid, launch, GRAPH_K, -1,
                      timing ? &pass_ms : nullptr));
        if (use_tma) CKR(tma_check(ctx));
        if (timing) tune_record(ctx->tbwd, pass_ms / (nt - 1));
        ctx->have_cig = want_cig;
    }
    CK(cudaGetLastError());
    // 4. per-shot post and stack
    CKR(ensure(ctx, ctx->reduce, 64));
    CK(cudaMemsetAsync(ctx->reduce.p, 0, 8, ctx->stream));
    k_max_nonneg<<<592, 256, 0, ctx->stream>>>(D(ctx->S), gb, (unsigned long long *)ctx->reduce.p);
    ctx->launches += 2;   // with k_rtm_post below
    const size_t nimg = (size_t)ctx->nx * ctx->nz;
    if (!ctx->stack.p) {
        CKR(ensure(ctx, ctx->stack, sizeof(double) * nimg));
        CK(cudaMemsetAsync(ctx->stack.p, 0, sizeof(double) * nimg, ctx->stream));
    }
    CKR(ensure(ctx, ctx->stage_out, sizeof(float) * 3 * nimg));
    float *o_pp = F(ctx->stage_out), *o_src = o_pp + nimg, *o_f = o_src + nimg;
    k_rtm_post<<<dim3((ctx->nz + 31) / 32, (ctx->nx + 7) / 8), dim3(32, 8), 0, ctx->stream>>>(
        D(ctx->I), D(ctx->S), F(ctx->vp), (const unsigned long long *)ctx->reduce.p, ctx->ntx, ctx->ntz, ctx->ldz,
        ctx->pmlc, ctx->grid.dx, ctx->grid.dz, o_pp, o_src, o_f, (flags & SWD_RTM_NO_STACK) ? nullptr : D(ctx->stack));
    CK(cudaGetLastError());
    if (image_pp) CKR(from_dev(ctx, image_pp, o_pp, sizeof(float) * nimg));
    if (image_src) CKR(from_dev(ctx, image_src, o_src, sizeof(float) * nimg));
    if (fimage) CKR(from_dev(ctx, fimage, o_f, sizeof(float) * nimg));
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    ctx->have_shot = true;
    return SWD_OK;
}

int swd_rtm_shot(swd_ctx *ctx, const swd_shot *shot, const float *rick, const float *data, unsigned flags, float *syn,
                 float *image_pp, float *image_src, float *fimage)
{
    CKR(check_ready(ctx));
    if (!rick || !data) return fail(ctx, SWD_ERR_ARG, "rick and data are required");
    CKR(rtm_forward_part(ctx, shot, rick, syn));
    return rtm_backward_part(ctx, shot, data, flags, image_pp, image_src, fimage);
}

int swd_rtm_forward(swd_ctx *ctx, const swd_shot *shot, const float *rick, float *syn)
{
    CKR(check_ready(ctx));
    if (!rick) return fail(ctx, SWD_ERR_ARG, "rick is required");
    CKR(rtm_forward_part(ctx, shot, rick, syn));
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    return SWD_OK;
}

int swd_rtm_backward(swd_ctx *ctx, const swd_shot *shot, const float *data, unsigned flags, float *image_pp,
                     float *image_src, float *fimage)
{
    CKR(check_ready(ctx));
    if (!data) return fail(ctx, SWD_ERR_ARG, "data is required");
    return rtm_backward_part(ctx, shot, data, flags, image_pp, image_src, fimage);
}

int swd_rtm_raw(swd_ctx *ctx, double *image, double *illum_src, double *illum_rcv)
{
    if (!ctx) return SWD_ERR_ARG;
    if (!ctx->have_shot) return fail(ctx, SWD_ERR_STATE, "no RTM shot has run");
    if (illum_rcv && !ctx->have_R) return fail(ctx, SWD_ERR_STATE, "receiver illumination was not accumulated");
    CK(cudaSetDevice(ctx->dev));
    double *dst[3] = {image, illum_src, illum_rcv};
    DevBuf *src[3] = {&ctx->I, &ctx->S, &ctx->R};
    for (int k = 0; k < 3; k++) {
        if (!dst[k]) continue;
        CK(cudaMemcpy2DAsync(dst[k], ctx->ntz * sizeof(double), D(*src[k]), ctx->ldz * sizeof(double),
                             ctx->ntz * sizeof(double), ctx->ntx,
                             is_device_ptr(dst[k]) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return SWD_OK;
}

int swd_stack_get(swd_ctx *ctx, int edge_zero, float *migration)
{
    if (!ctx || !migration) return SWD_ERR_ARG;
    CK(cudaSetDevice(ctx->dev));
    const size_t nimg = (size_t)ctx->nx * ctx->nz;
    if (!ctx->stack.p) {
        CKR(ensure(ctx, ctx->stack, sizeof(double) * nimg));
        CK(cudaMemsetAsync(ctx->stack.p, 0, sizeof(double) * nimg, ctx->stream));
    }
    CKR(ensure(ctx, ctx->stage_in, sizeof(float) * nimg));
    k_stack_out<<<296, 256, 0, ctx->stream>>>(D(ctx->stack), F(ctx->stage_in), ctx->nx, ctx->nz, ctx->Lc, edge_zero);
    CK(cudaGetLastError());
    CKR(from_dev(ctx, migration, ctx->stage_in.p, sizeof(float) * nimg));
    CK(cudaStreamSynchronize(ctx->stream));
    return SWD_OK;
}

int swd_stack_reset(swd_ctx *ctx)
{
    if (!ctx) return SWD_ERR_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (ctx->stack.p) CK(cudaMemsetAsync(ctx->stack.p, 0, ctx->stack.n, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SWD_OK;
}

int swd_hilbert(swd_ctx *ctx, int nt, const float *rick, float *hrick)
{
    if (!ctx || !rick || !hrick || nt < 2) return fail(ctx, SWD_ERR_ARG, "bad hilbert arguments");
    CK(cudaSetDevice(ctx->dev));
    const int N = swd_prep_pow2(nt);
    if (N < 32 || N > 16384) return fail(ctx, SWD_ERR_ARG, "Hilbert length %d outside [32, 16384]", N);
    DevBuf tw, io;
    CKR(make_twiddles(ctx, tw, N));
    CKR(ensure(ctx, io, sizeof(float) * 2 * nt));
    CKR(to_dev(ctx, io.p, rick, sizeof(float) * nt));
    const size_t sm = sizeof(float2) * N;
    CK(cudaFuncSetAttribute(k_hilbert, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_hilbert<<<1, 256, sm, ctx->stream>>>(F(io), F(io) + nt, (const float2 *)tw.p, nt, N, ilog2(N));
    cudaError_t e = cudaGetLastError();
    int rc = SWD_OK;
    if (e != cudaSuccess) rc = fail(ctx, SWD_ERR_CUDA, "k_hilbert: %s", cudaGetErrorString(e));
    if (rc == SWD_OK) rc = from_dev(ctx, hrick, F(io) + nt, sizeof(float) * nt);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(tw.p);
    cudaFree(io.p);
    return rc;
}

int swd_smooth(swd_ctx *ctx, int ntx, int ntz, int pml, int window, float *vp)
{
    if (!ctx || !vp || ntx <= 2 * pml || ntz <= 2 * pml || window < 0 || window > 64)
        return fail(ctx, SWD_ERR_ARG, "bad smoothing arguments");
    CK(cudaSetDevice(ctx->dev));
    // normalised Gaussian of ini_model_mine (acoustic_HLVSPRTMC.cpp:1475-1501), built on the host
    const int wx = 2 * window + 1;
    const double PI = 3.1415926, sigma = window / 2.0;
    std::vector<double> coef(wx * wx);
    double sum = 0.0;
    for (int ix = 0; ix < wx; ix++)
        for (int iz = 0; iz < wx; iz++) {
            int ip = ix * wx + iz;
            coef[ip] = 1.0 / (2.0 * PI * sigma * sigma) *
                       exp(-((ix - window) * (ix - window) + (iz - window) * (iz - window)) / (2.0 * sigma * sigma));
            sum += coef[ip];
        }
    for (auto &c : coef) c /= sum;
    const size_t n = (size_t)ntx * ntz;
    DevBuf a, b, cf;
    int rc = ensure(ctx, a, sizeof(float) * n);
    if (rc == SWD_OK) rc = ensure(ctx, b, sizeof(float) * n);
    if (rc == SWD_OK) rc = ensure(ctx, cf, sizeof(double) * coef.size());
    if (rc == SWD_OK) rc = to_dev(ctx, a.p, vp, sizeof(float) * n);
    if (rc == SWD_OK) {
        cudaMemcpyAsync(cf.p, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync(b.p, a.p, sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream);
        k_smooth<<<dim3((ntz - 2 * pml + 31) / 32, (ntx - 2 * pml + 7) / 8), dim3(32, 8), 0, ctx->stream>>>(
            F(a), F(b), D(cf), ntx, ntz, pml, window);
        k_pml_x<<<(ntz + 127) / 128, 128, 0, ctx->stream>>>(F(b), ntx, ntz, pml);
        k_pml_z<<<(ntx + 127) / 128, 128, 0, ctx->stream>>>(F(b), ntx, ntz, pml);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(ctx, SWD_ERR_CUDA, "smoothing kernels: %s", cudaGetErrorString(e));
        else rc = from_dev(ctx, vp, b.p, sizeof(float) * n);
    }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(a.p);
    cudaFree(b.p);
    cudaFree(cf.p);
    return rc;
}

int swd_preprocess(swd_ctx *ctx, int r_n, int nt, float dt, const float *d, float *rms)
{
    if (!ctx || !d || !rms || r_n < 1 || nt < 1) return fail(ctx, SWD_ERR_ARG, "bad preprocess arguments");
    CK(cudaSetDevice(ctx->dev));
    const size_t n = (size_t)r_n * nt;
    CKR(ensure(ctx, ctx->stage_in, sizeof(float) * 2 * n));
    float *a = F(ctx->stage_in), *b = a + n;
    CKR(to_dev(ctx, a, d, sizeof(float) * n));
    k_preprocess<<<(r_n + 127) / 128, 128, 0, ctx->stream>>>(a, b, r_n, nt, dt);
    CK(cudaGetLastError());
    CKR(from_dev(ctx, rms, b, sizeof(float) * n));
    CK(cudaStreamSynchronize(ctx->stream));
    return SWD_OK;
}


int swd_decon_geometry(const swd_decon_params *p, int *windows, int *fft_nx, int *fft_nz)
{
    DeconGeo g;
    int rc = decon_geo(p, g);
    if (rc) return rc;
    if (windows) *windows = g.totalnum;
    if (fft_nx) *fft_nx = g.FX;
    if (fft_nz) *fft_nz = g.FZ;
    return SWD_OK;
}

int swd_decon(swd_ctx *ctx_in, const swd_decon_params *p, const float *migreal, const float *migpsf, float *mig_dec,
              float *mig_coef)
{
    // a NULL context runs on the current device with a temporary stream
    swd_ctx tmp;
    swd_ctx *ctx = ctx_in ? ctx_in : &tmp;
    if (!ctx_in) {
        cudaGetDevice(&tmp.dev);
        if (cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking) != cudaSuccess) return SWD_ERR_CUDA;
    }
    int rc = SWD_OK;
    do {
        DeconGeo g;
        if (!migreal || !migpsf || !mig_dec || !mig_coef) { rc = fail(ctx, SWD_ERR_ARG, "decon: NULL array"); break; }
        if (decon_geo(p, g) != SWD_OK) { rc = fail(ctx, SWD_ERR_ARG, "decon: invalid window geometry"); break; }
        if (cudaSetDevice(ctx->dev) != cudaSuccess) { rc = fail(ctx, SWD_ERR_CUDA, "cudaSetDevice"); break; }
        // Hann-edged output taper (:355-383), built on the host with the reference's arithmetic
        const double PI = 3.1415926;
        std::vector<float> coefr((size_t)g.outwinx * g.outwinz);
        for (int ix = 0; ix < g.outwinx; ix++)
            for (int iz = 0; iz < g.outwinz; iz++) {
                float cx, cz;
                if (ix <= p->snapwinx - 1) cx = 0.5000 - 0.5 * cos(PI * ix / (p->snapwinx - 1));
                else if (ix >= g.outwinx - p->snapwinx) cx = 0.5000 + 0.5 * cos(PI * (ix - g.outwinx + p->snapwinx) / (p->snapwinx - 1));
                else cx = 1.0;
                if (iz <= p->snapwinz - 1) cz = 0.5000 - 0.5 * cos(PI * iz / (p->snapwinz - 1));
                else if (iz >= g.outwinz - p->snapwinz) cz = 0.5000 + 0.5 * cos(PI * (iz - g.outwinz + p->snapwinz) / (p->snapwinz - 1));
                else cz = 1.0;
                coefr[(size_t)ix * g.outwinz + iz] = cx * cz;
            }
        // device arrays are read and written in place; host arrays go through the scratch
        const size_t np = (size_t)g.nx * g.nz, nout = coefr.size();
        // the kernels read and write only memory of this device; anything else (host memory,
        // another GPU's memory) goes through the context's scratch with copies
        const bool din = is_device_ptr_on(migreal, ctx->dev) && is_device_ptr_on(migpsf, ctx->dev);
        const bool dout = is_device_ptr_on(mig_dec, ctx->dev) && is_device_ptr_on(mig_coef, ctx->dev);
        DevBuf &bin = ctx->dcn[0], &bcoef = ctx->dcn[1], &bwin = ctx->dcn[2], &bout = ctx->dcn[3], &bws = ctx->dcn[4],
               &btab = ctx->dcn[5];
        const int nblk = decon_persistent(g) ? decon_ws_blocks(g, ctx->dev) : 0;
        if (decon_persistent(g) && nblk < 1) { rc = fail(ctx, SWD_ERR_CUDA, "decon: no launch shape for the window kernel"); break; }
        if (decon_persistent(g)) rc = ensure(ctx, bws, sizeof(float) * (size_t)nblk * decon_ws_floats(g));
        if (!rc && !din) rc = ensure(ctx, bin, sizeof(float) * 2 * np);
        if (!rc) rc = ensure(ctx, bcoef, sizeof(float) * nout);
        if (!rc) rc = ensure(ctx, bwin, sizeof(float) * nout * g.totalnum);
        if (!rc) rc = ensure(ctx, btab, sizeof(float2) * decon_tab_len(g));
        if (!rc && !dout) rc = ensure(ctx, bout, sizeof(float) * 2 * np);
        const float *im = din ? migreal : F(bin), *ps = din ? migpsf : F(bin) + np;
        float *od = dout ? mig_dec : F(bout), *oc = dout ? mig_coef : F(bout) + np;
        if (!rc && !din) rc = to_dev(ctx, bin.p, migreal, sizeof(float) * np);
        if (!rc && !din) rc = to_dev(ctx, F(bin) + np, migpsf, sizeof(float) * np);
        if (!rc && cudaMemcpyAsync(bcoef.p, coefr.data(), sizeof(float) * nout, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
            rc = fail(ctx, SWD_ERR_CUDA, "decon: coefficient upload");
        if (!rc) {
            cudaError_t e = launch_decon_windows(g, im, ps, F(bwin), F(bws), nblk, (float2 *)btab.p, ctx->stream);
            if (e == cudaSuccess) {
                k_decon_gather<<<592, 256, 0, ctx->stream>>>(g, F(bwin), F(bcoef), od, oc);
                e = cudaGetLastError();
            }
            if (e != cudaSuccess) rc = fail(ctx, SWD_ERR_CUDA, "decon kernels: %s", cudaGetErrorString(e));
            else ctx->launches += g.n1 != g.n0 ? 4 : 3;
        }
        if (!rc && !dout) rc = from_dev(ctx, mig_dec, od, sizeof(float) * np);
        if (!rc && !dout) rc = from_dev(ctx, mig_coef, oc, sizeof(float) * np);
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (!rc && e != cudaSuccess) rc = fail(ctx, SWD_ERR_CUDA, "decon: %s", cudaGetErrorString(e));
    } while (0);
    if (!ctx_in) {
        for (DevBuf &b : tmp.dcn) cudaFree(b.p);
        cudaStreamDestroy(tmp.stream);
    }
    return rc;
}

int swd_decon_noalloc(const swd_decon_params *p, const float *migreal, const float *migpsf, float *mig_dec,
                      float *mig_coef, void *cuda_stream)
{
    DeconGeo g;
    if (!p || decon_geo(p, g) != SWD_OK) return SWD_ERR_ARG;
    const size_t nout = (size_t)g.outwinx * g.outwinz;
    // scratch: taper, window slots, the transform tables (from a 256-byte aligned offset), then
    // (persistent kernel) the CTA workspaces from the next 256-byte aligned offset; that kernel
    // runs on as many CTAs as have a workspace that fits
    const size_t tabof = ((size_t)g.totalnum * nout + nout + 63) & ~(size_t)63;
    const size_t used = tabof + 2 * decon_tab_len(g), wsoff = (used + 63) & ~(size_t)63;
    if (used > SWD_DECON_STATIC_SCRATCH_FLOATS) return SWD_ERR_CAPACITY;
    // a launch error left over from the caller's own work is not this call's: clear it, so the
    // checks below see only this call's launches
    cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return SWD_ERR_CUDA;
    }
    // the kernels dereference the four arrays on this device: memory of another GPU would be an
    // illegal access without peer mappings, so it is refused here
    const void *ptrs[4] = {migreal, migpsf, mig_dec, mig_coef};
    for (const void *q : ptrs)
        if (!is_device_ptr_on(q, dev)) return SWD_ERR_ARG;
    // Device address of the static scratch on this device.  It is looked up on every call (the
    // lookup allocates nothing) rather than cached: a cache would have to be shared between host
    // threads and would go stale if the caller reset the device, which reloads the module.  The
    // first lookup on a device loads the module there, so the first call should come before any
    // stream capture.
    void *sa = nullptr;
    if (cudaGetSymbolAddress(&sa, g_decon_scratch) != cudaSuccess || !sa) {
        cudaGetLastError();
        return SWD_ERR_CUDA;
    }
    int nblk = 0;
    if (decon_persistent(g)) {
        const size_t per = decon_ws_floats(g);
        const size_t fit = wsoff < SWD_DECON_STATIC_SCRATCH_FLOATS ? (SWD_DECON_STATIC_SCRATCH_FLOATS - wsoff) / per : 0;
        const int occ = decon_ws_blocks(g, dev);
        if (occ < 0) return SWD_ERR_CUDA;
        nblk = (int)std::min<long long>(occ, (long long)fit);
        if (nblk < 1) return SWD_ERR_CAPACITY;
    }
    float *coefr = (float *)sa, *winout = coefr + nout;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    k_decon_taper<<<(int)((nout + 255) / 256), 256, 0, st>>>(coefr, g.outwinx, g.outwinz, p->snapwinx, p->snapwinz);
    if (cudaGetLastError() != cudaSuccess) return SWD_ERR_CUDA;
    if (launch_decon_windows(g, migreal, migpsf, winout, coefr + wsoff, nblk, (float2 *)(coefr + tabof), st) !=
        cudaSuccess)
        return SWD_ERR_CUDA;
    k_decon_gather<<<592, 256, 0, st>>>(g, winout, coefr, mig_dec, mig_coef);
    return cudaGetLastError() == cudaSuccess ? SWD_OK : SWD_ERR_CUDA;
}

}  // extern "C"

#include "born_host.inl"
#include "batch_host.inl"
