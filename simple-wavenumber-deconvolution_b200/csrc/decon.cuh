// decon.cuh -- windowed wavenumber-domain PSF deconvolution (decon2d_mine's window loop,
// kkdecon_acoustic/kk_decon_interp_psf_minewindow.cpp:543-674) as one CTA per window.
//
// Per window, in shared memory:
//   Z = M/|M|_1 + i*S/|S|_1 on an n0 x n1 buffer (M: filterwin^2 image patch centred at
//   the buffer midpoint, S: nearest psfwin^2 PSF at the buffer corner);
//   Z^ = DFT2(Z) once (the two real transforms packed into one complex one);
//   M^(k) = (Z^(k) + conj Z^(-k))/2,  S^(k) = (Z^(k) - conj Z^(-k))/(2i);
//   D(k) = M^ conj(S^) / (|S^|^2 + eps*max|S^|^2), numerator and quotient in FP64, the
//   damped denominator rounded through float as the reference does (:636,648);
//   d = IDFT2(D) (unnormalised); the outwin^2 centre, times the Hann-edged taper, is
//   written to a per-window slot.  A second kernel overlap-adds the slots in window order.
//
// Windows whose buffer does not fit in shared memory (or workspace = 1) keep it in a per-CTA
// global-memory workspace instead; each transform pass then copies a chunk of whole
// transforms into shared memory, transforms it there and writes it back (dft2_staged), with
// the same per-output arithmetic, so both variants give the same bits.
//
// Iterative option (iters > 0, no counterpart in the reference, which parses reg_eps and itn
// but never uses them): the damped solution x0 = IDFT2(D)/n of the window starts FISTA on
//   f(x) = 1/(2n) |S^ X^ - M^|^2 + mu/2 |x|^2 + lambda |x|_1,   mu = reg_l2 * max|S^|^2,
// step tau = 1/(max|S^|^2 + mu), soft threshold tau*lambda = reg_l1 * max|x0|; gradient
// IDFT2((|S^|^2 + mu) Y^ - M^ conj S^)/n, two 2D transforms per iteration; B = M^ conj S^,
// P = |S^|^2 and the iterates live in the global workspace.  The output is n*x, the scale of
// the direct path's unnormalised inverse transform.
//
// The buffer index is ixx*FZ + izz and the 2D transform is taken over (n0 rows x n1
// columns) of that linear buffer, which is how the reference plans it
// (fftw_plan_dft_2d(fullwz, fullwx) on an x-major buffer, :490-493).  Transforms are FP32
// FFTs, one warp per row or column (wfft.cuh): radix 2 for power-of-two lengths, Bluestein's
// chirp-z through a power-of-two FFT for every other length up to 512 (the reference's 101 is
// prime), with tables built in double by k_wfft_tables and copied into shared memory.
// The L1 norms are accumulated serially in the reference's order with the reference's
// float-through-double rounding, so the normalisation matches it exactly.
#pragma once
#include <cuda_runtime.h>
#include "fft.cuh"
#include "wfft.cuh"

namespace swd {

struct DeconGeo {
    int nx, nz;
    int psfwinx, psfwinz, filterwinx, filterwinz, snapwinx, snapwinz;
    int halfpsfwx, halfpsfwz, halfltwx, halfltwz, nxwpsf, nzwpsf;
    int FX, FZ, n0, n1, midpx, midpz, ocx, ocz;
    int outwinx, outwinz, halfoutwx, halfoutwz, stepwinx, stepwinz, stepnumx, stepnumz, totalnum, nxp, nzp;
    float epsilon;
    int psf_interp;   // 1: bilinear interpolation of the lattice PSFs (project option)
    int staged;       // 1: buffer in a global workspace, passes staged through shared memory
    int iters;        // FISTA iterations (0: the reference's direct division)
    float reg_l1, reg_l2;
};

// Per-CTA global scratch of the iterative option (n = FX*FZ elements each)
struct DeconIter {
    float2 *B;        // M^ conj S^
    float *P;         // |S^|^2
    float *X, *XP;    // current and previous iterate
};

// Bracketing lattice points of a window-centre coordinate for PSF interpolation: f0 =
// floor((c - h)/w) and f1 = f0 + 1 clamped to [3, n - 4] (the reference's lattice range), t the
// fractional position in [0, 1] (0 when they coincide).
__device__ __forceinline__ void psf_bracket(int c, int h, int w, int n, int &f0, int &f1, double &t)
{
    const double pos = (double)(c - h) / (double)w;
    int a = (int)floor(pos);
    a = a < 3 ? 3 : (a > n - 4 ? n - 4 : a);
    const int b = a + 1 > n - 4 ? n - 4 : a + 1;
    double u = pos - (double)a;
    u = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
    f0 = a;
    f1 = b;
    t = b == a ? 0.0 : u;
}

// expanded-image read (edge replication of :303-339): clamp to the last row/column
__device__ __forceinline__ float img_at(const float *__restrict__ im, int nx, int nz, int ix, int iz)
{
    ix = ix < nx ? ix : nx - 1;
    iz = iz < nz ? iz : nz - 1;
    return __ldg(im + (size_t)ix * nz + iz);
}

__device__ void dft2(float2 *s, const WfftPlan &P0, const WfftPlan &P1, int n0, int n1, int sign)
{
    fft_pass(s, P1, n0, 1, n1, sign);   // rows (length n1)
    fft_pass(s, P0, n1, n1, 1, sign);   // columns (length n0)
}

// dft2 on a buffer Zg in global memory: row transforms (length n1, contiguous) and then column
// transforms (length n0, stride n1) are copied cap elements at a time into the shared chunk,
// transformed by fft_pass and written back.  cap >= max(n0, n1).
__device__ void dft2_staged(float2 *Zg, float2 *chunk, int cap, const WfftPlan &P0, const WfftPlan &P1, int n0, int n1,
                            int sign)
{
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int R = cap / n1;
    for (int r0 = 0; r0 < n0; r0 += R) {
        const int nr = min(R, n0 - r0), m = nr * n1;
        float2 *src = Zg + (size_t)r0 * n1;
        for (int j = tid; j < m; j += nthr) chunk[j] = src[j];
        __syncthreads();
        fft_pass(chunk, P1, nr, 1, n1, sign);
        for (int j = tid; j < m; j += nthr) src[j] = chunk[j];
        __syncthreads();
    }
    const int Cc = cap / n0;
    for (int c0 = 0; c0 < n1; c0 += Cc) {
        const int nc = min(Cc, n1 - c0), m = n0 * nc;
        for (int j = tid; j < m; j += nthr) chunk[j] = Zg[(size_t)(j / nc) * n1 + c0 + j % nc];
        __syncthreads();
        fft_pass(chunk, P0, nc, nc, 1, sign);
        for (int j = tid; j < m; j += nthr) Zg[(size_t)(j / nc) * n1 + c0 + j % nc] = chunk[j];
        __syncthreads();
    }
}

// Floats2 of transform tables of a window geometry: lengths n0 and n1 (one copy when equal).
__host__ __device__ inline size_t decon_tab_len(const DeconGeo &g)
{
    return wfft_table_len(g.n0) + (g.n1 != g.n0 ? wfft_table_len(g.n1) : 0);
}

// Copies the transform tables (built by k_wfft_tables into tabs: length n0, then length n1
// unless equal) into shared memory at sm and returns the two plans over that copy.
__device__ __forceinline__ void decon_plans(const DeconGeo &g, const float2 *__restrict__ tabs, float2 *sm,
                                            WfftPlan &P0, WfftPlan &P1)
{
    const int n = (int)decon_tab_len(g);
    for (int j = threadIdx.x; j < n; j += blockDim.x) sm[j] = tabs[j];
    P0 = wfft_plan(g.n0, sm);
    P1 = g.n1 != g.n0 ? wfft_plan(g.n1, sm + wfft_table_len(g.n0)) : P0;
    __syncthreads();
}

// One window w on the buffer Z (shared memory, or global memory when STAGED with the shared
// chunk of cap elements); the twiddle tables are filled by the caller.
template <bool STAGED>
__device__ __forceinline__ void window_dft2(float2 *Z, float2 *chunk, int cap, const WfftPlan &P0, const WfftPlan &P1,
                                            const DeconGeo &g, int sign)
{
    if (STAGED) dft2_staged(Z, chunk, cap, P0, P1, g.n0, g.n1, sign);
    else dft2(Z, P0, P1, g.n0, g.n1, sign);
}

// FISTA refinement of the window solution held (unnormalised) in Z.x; leaves n*x in Z.x.
template <bool STAGED>
__device__ void decon_iterate(const DeconGeo &g, float2 *Z, const DeconIter &it, float fmax, const WfftPlan &P0,
                              const WfftPlan &P1, float2 *chunk, int cap)
{
    __shared__ unsigned s_xmax;
    const int n = g.FX * g.FZ, tid = threadIdx.x, nthr = blockDim.x;
    const float invn = 1.0f / (float)n, mu = g.reg_l2 * fmax, tau = 1.0f / (fmax + mu);
    if (tid == 0) s_xmax = 0u;
    __syncthreads();
    float am = 0.f;
    for (int j = tid; j < n; j += nthr) {
        const float x = Z[j].x * invn;
        it.X[j] = x;
        it.XP[j] = x;
        am = fmaxf(am, fabsf(x));
    }
    for (int o = 16; o > 0; o >>= 1) am = fmaxf(am, __shfl_xor_sync(0xffffffffu, am, o));
    if ((tid & 31) == 0) atomicMax(&s_xmax, __float_as_uint(am));
    __syncthreads();
    const float thr = g.reg_l1 * __uint_as_float(s_xmax);
    float t = 1.0f;
    for (int k = 0; k < g.iters; k++) {
        const float tn = 0.5f * (1.0f + sqrtf(1.0f + 4.0f * t * t)), beta = (t - 1.0f) / tn;
        t = tn;
        for (int j = tid; j < n; j += nthr) Z[j] = make_float2(it.X[j] + beta * (it.X[j] - it.XP[j]), 0.f);
        __syncthreads();
        window_dft2<STAGED>(Z, chunk, cap, P0, P1, g, -1);
        for (int j = tid; j < n; j += nthr) {
            const float2 y = Z[j], b = it.B[j];
            const float q = it.P[j] + mu;
            Z[j] = make_float2(q * y.x - b.x, q * y.y - b.y);
        }
        __syncthreads();
        window_dft2<STAGED>(Z, chunk, cap, P0, P1, g, +1);
        for (int j = tid; j < n; j += nthr) {
            const float x = it.X[j], y = x + beta * (x - it.XP[j]);
            const float v = y - tau * (Z[j].x * invn);
            it.XP[j] = x;
            it.X[j] = copysignf(fmaxf(fabsf(v) - thr, 0.f), v);
        }
        __syncthreads();
    }
    for (int j = tid; j < n; j += nthr) Z[j].x = it.X[j] * (float)n;
    __syncthreads();
}

// Sum of |Z[(ox + ixx)*FZ + oz + izz]| (component x, or y when Y) over ixx < nxw, izz < nzw,
// in that order, into a float: the reference's accumulation acc = (float)((double)acc + |v|).
// That is computed here as one correctly rounded float addition, which gives the same bits: the
// sum of two floats rounded to double and then to float equals the sum rounded to float once,
// because double carries more than twice float's precision plus two bits (53 >= 2*24 + 2; double
// rounding is innocuous for a single addition).  The chain of additions is serial; loads are
// issued eight at a time ahead of it.
template <bool Y>
__device__ float l1_serial(const float2 *Z, int FZ, int ox, int oz, int nxw, int nzw)
{
    float acc = 0.f;
    for (int ixx = 0; ixx < nxw; ixx++) {
        const float2 *row = Z + (size_t)(ox + ixx) * FZ + oz;
        int izz = 0;
        for (; izz + 8 <= nzw; izz += 8) {
            float v[8];
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] = Y ? row[izz + k].y : row[izz + k].x;
#pragma unroll
            for (int k = 0; k < 8; k++) acc = __fadd_rn(acc, fabsf(v[k]));
        }
        for (; izz < nzw; izz++) acc = __fadd_rn(acc, fabsf(Y ? row[izz].y : row[izz].x));
    }
    return acc;
}

template <bool STAGED>
__device__ void decon_window(const DeconGeo &g, const float *__restrict__ mig, const float *__restrict__ psf,
                             float *__restrict__ winout, int w, float2 *Z, const WfftPlan &P0, const WfftPlan &P1,
                             float2 *chunk, int cap, const DeconIter &itr)
{
    const int n = g.FX * g.FZ;
    __shared__ float s_ppmax, s_psfmax;
    __shared__ unsigned s_fmax;
    const int ix = g.stepwinx * (w / g.stepnumz), iz = g.stepwinz * (w % g.stepnumz);
    const int tid = threadIdx.x, nthr = blockDim.x;
    // nearest PSF on the lattice, indices clamped to [3, nwpsf-4] (:586-598)
    int ixf = (ix - g.halfpsfwx) / g.psfwinx, izf = (iz - g.halfpsfwz) / g.psfwinz;
    if (ixf <= 2) ixf = 3;
    if (ixf >= g.nxwpsf - 3) ixf = g.nxwpsf - 4;
    if (izf <= 2) izf = 3;
    if (izf >= g.nzwpsf - 3) izf = g.nzwpsf - 4;
    const int ixp = g.halfpsfwx + ixf * g.psfwinx, izp = g.halfpsfwz + izf * g.psfwinz;
    // PSF patch value: the nearest lattice PSF, or (psf_interp) the bilinear blend of the four
    // around the window centre, formed in double without contraction and rounded to float
    int fx0 = 0, fx1 = 0, fz0 = 0, fz1 = 0;
    double tx = 0.0, tz = 0.0;
    if (g.psf_interp) {
        psf_bracket(ix, g.halfpsfwx, g.psfwinx, g.nxwpsf, fx0, fx1, tx);
        psf_bracket(iz, g.halfpsfwz, g.psfwinz, g.nzwpsf, fz0, fz1, tz);
    }
    auto psf_val = [&](int ixx, int izz) -> float {
        if (!g.psf_interp) return img_at(psf, g.nx, g.nz, ixp + ixx - g.halfpsfwx, izp + izz - g.halfpsfwz);
        const int xa = fx0 * g.psfwinx + ixx, xb = fx1 * g.psfwinx + ixx;
        const int za = fz0 * g.psfwinz + izz, zb = fz1 * g.psfwinz + izz;
        const double a = img_at(psf, g.nx, g.nz, xa, za), b = img_at(psf, g.nx, g.nz, xb, za);
        const double c = img_at(psf, g.nx, g.nz, xa, zb), d = img_at(psf, g.nx, g.nz, xb, zb);
        const double s1 = __dadd_rn(__dmul_rn(1.0 - tx, a), __dmul_rn(tx, b));
        const double s2 = __dadd_rn(__dmul_rn(1.0 - tx, c), __dmul_rn(tx, d));
        return (float)__dadd_rn(__dmul_rn(1.0 - tz, s1), __dmul_rn(tz, s2));
    };

    for (int j = tid; j < n; j += nthr) Z[j] = make_float2(0.f, 0.f);
    if (tid == 64) s_fmax = 0u;
    __syncthreads();
    // raw image patch (centred) and PSF patch (corner) into the buffer
    for (int j = tid; j < g.filterwinx * g.filterwinz; j += nthr) {
        const int ixx = j / g.filterwinz, izz = j % g.filterwinz;
        const int iix = ix - g.halfltwx + ixx, iiz = iz - g.halfltwz + izz;
        if (iix >= 0 && iix < g.nxp && iiz >= 0 && iiz < g.nzp)
            Z[(g.midpx - g.halfltwx + ixx) * g.FZ + g.midpz - g.halfltwz + izz].x = img_at(mig, g.nx, g.nz, iix, iiz);
    }
    for (int j = tid; j < g.psfwinx * g.psfwinz; j += nthr) {
        const int ixx = j / g.psfwinz, izz = j % g.psfwinz;
        Z[ixx * g.FZ + izz].y = psf_val(ixx, izz);
    }
    __syncthreads();
    // L1 norms in the reference's order and rounding (:554-576, :618-620), from the buffer:
    // thread 0 sums the image patch, thread 32 the PSF (cells outside the expanded image are
    // zero there and add nothing)
    if (tid == 0) {
        float pp = l1_serial<false>(Z, g.FZ, g.midpx - g.halfltwx, g.midpz - g.halfltwz, g.filterwinx, g.filterwinz);
        if ((double)pp <= 1.0e-15) pp = 1.0e-10f;
        s_ppmax = pp;
    } else if (tid == 32) {
        s_psfmax = l1_serial<true>(Z, g.FZ, 0, 0, g.psfwinx, g.psfwinz);
    }
    __syncthreads();
    const double ppm = (double)s_ppmax, psm = (double)s_psfmax;
    for (int j = tid; j < g.filterwinx * g.filterwinz; j += nthr) {
        const int ixx = j / g.filterwinz, izz = j % g.filterwinz;
        float2 &z = Z[(g.midpx - g.halfltwx + ixx) * g.FZ + g.midpz - g.halfltwz + izz];
        z.x = (float)((double)z.x / ppm);
    }
    for (int j = tid; j < g.psfwinx * g.psfwinz; j += nthr) {
        const int ixx = j / g.psfwinz, izz = j % g.psfwinz;
        float2 &z = Z[ixx * g.FZ + izz];
        z.y = (float)((double)z.y / psm);
    }
    __syncthreads();
    window_dft2<STAGED>(Z, chunk, cap, P0, P1, g, -1);
    // |S^|^2 maximum over all bins (float compare of the double square, :625-633)
    float fm = 0.f;
    for (int j = tid; j < n; j += nthr) {
        const int r = j / g.n1, c = j % g.n1;
        const int jm = ((g.n0 - r) % g.n0) * g.n1 + (g.n1 - c) % g.n1;
        const float2 a = Z[j], b = Z[jm];
        const double sr = 0.5 * ((double)a.y + (double)b.y), si = -0.5 * ((double)a.x - (double)b.x);
        fm = fmaxf(fm, (float)(sr * sr + si * si));
    }
    for (int o = 16; o > 0; o >>= 1) fm = fmaxf(fm, __shfl_xor_sync(0xffffffffu, fm, o));
    if ((tid & 31) == 0) atomicMax(&s_fmax, __float_as_uint(fm));
    __syncthreads();
    float fft_max = __uint_as_float(s_fmax) * g.epsilon;
    if (fft_max == 0.0f) fft_max = 1.0e-15f;
    // D(k) and D(-k) from the pair (Z(k), Z(-k)); each pair handled once (j <= jm)
    for (int j = tid; j < n; j += nthr) {
        const int r = j / g.n1, c = j % g.n1;
        const int jm = ((g.n0 - r) % g.n0) * g.n1 + (g.n1 - c) % g.n1;
        if (j > jm) continue;
        const float2 a = Z[j], b = Z[jm];
        // bin k: M = ((a+b*)/2), S = ((a-b*)/2i); bin -k uses the conjugates
        const double mr = 0.5 * ((double)a.x + (double)b.x), mi = 0.5 * ((double)a.y - (double)b.y);
        const double sr = 0.5 * ((double)a.y + (double)b.y), si = -0.5 * ((double)a.x - (double)b.x);
        const float den = (float)((sr * sr + si * si) + (double)fft_max);
        const double dr = (mr * sr + mi * si) / (double)den;
        const double di = (-mr * si + mi * sr) / (double)den;
        Z[j] = make_float2((float)dr, (float)di);
        if (jm != j) Z[jm] = make_float2((float)dr, (float)-di);   // D(-k) = conj D(k)
        if (g.iters > 0) {
            const float2 b = make_float2((float)(mr * sr + mi * si), (float)(mi * sr - mr * si));
            const float pk = (float)(sr * sr + si * si);
            itr.B[j] = b;
            itr.P[j] = pk;
            itr.B[jm] = make_float2(b.x, -b.y);
            itr.P[jm] = pk;
        }
    }
    __syncthreads();
    window_dft2<STAGED>(Z, chunk, cap, P0, P1, g, +1);
    if (g.iters > 0 && __uint_as_float(s_fmax) > 0.0f)
        decon_iterate<STAGED>(g, Z, itr, __uint_as_float(s_fmax), P0, P1, chunk, cap);
    const int nout = g.outwinx * g.outwinz;
    float *o = winout + (size_t)w * nout;
    for (int j = tid; j < nout; j += nthr) {
        const int ixx = j / g.outwinz, izz = j % g.outwinz;
        const int ip = (g.ocx - g.halfoutwx + ixx) * g.FZ + g.ocz - g.halfoutwz + izz;
        o[j] = Z[ip].x;
    }
}

// One CTA per window, the whole buffer and the transform tables in shared memory.
__global__ void __launch_bounds__(512) k_decon_window(DeconGeo g, const float *__restrict__ mig,
                                                      const float *__restrict__ psf, float *__restrict__ winout,
                                                      const float2 *__restrict__ tabs)
{
    extern __shared__ float2 sm[];
    float2 *Z = sm;
    WfftPlan P0, P1;
    decon_plans(g, tabs, Z + (size_t)g.FX * g.FZ, P0, P1);
    decon_window<false>(g, mig, psf, winout, blockIdx.x, Z, P0, P1, nullptr, 0, DeconIter{});
}

// Floats of global workspace one persistent CTA of k_decon_window_ws needs: the staged
// transform buffer and the iterative option's B, P and iterates.
__host__ __device__ inline size_t decon_ws_floats(const DeconGeo &g)
{
    const size_t n = (size_t)g.FX * g.FZ;
    return ((g.staged ? 2 * n : 0) + (g.iters > 0 ? 5 * n : 0) + 63) & ~(size_t)63;   // 256-byte aligned slices
}

// Persistent CTAs working through windows blockIdx.x, blockIdx.x + gridDim.x, ..., each with
// decon_ws_floats(g) floats of the global workspace ws.  STAGED: the transform buffer is in
// that workspace and shared memory holds the twiddles and a chunk of cap elements for the
// staged passes; otherwise the buffer and the twiddles are in shared memory.
template <bool STAGED>
__global__ void __launch_bounds__(512) k_decon_window_ws(DeconGeo g, const float *__restrict__ mig,
                                                         const float *__restrict__ psf, float *__restrict__ winout,
                                                         float *__restrict__ ws, int cap, const float2 *__restrict__ tabs)
{
    extern __shared__ float2 sm[];
    const size_t n = (size_t)g.FX * g.FZ;
    float *mine = ws + (size_t)blockIdx.x * decon_ws_floats(g);
    float2 *Z, *tsm, *chunk = nullptr;
    if (STAGED) {
        Z = (float2 *)mine;
        mine += 2 * n;
        tsm = sm;
        chunk = sm + decon_tab_len(g);
    } else {
        Z = sm;
        tsm = sm + n;
    }
    DeconIter itr{};
    if (g.iters > 0) {
        itr.B = (float2 *)mine;
        itr.P = mine + 2 * n;
        itr.X = itr.P + n;
        itr.XP = itr.X + n;
    }
    WfftPlan P0, P1;
    decon_plans(g, tabs, tsm, P0, P1);
    for (int w = blockIdx.x; w < g.totalnum; w += gridDim.x) {
        decon_window<STAGED>(g, mig, psf, winout, w, Z, P0, P1, chunk, cap, itr);
        __syncthreads();   // the next window's fill overwrites Z and the shared scalars
    }
}

// Overlap-add of the window slots in window order (:656-673), float accumulators with the
// reference's double-then-round update, cropped to nx x nz (:724-731).
__global__ void k_decon_gather(DeconGeo g, const float *__restrict__ winout, const float *__restrict__ coefr,
                               float *__restrict__ dec, float *__restrict__ coef)
{
    const size_t np = (size_t)g.nx * g.nz;
    const int nout = g.outwinx * g.outwinz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
        const int px = (int)(i / g.nz), pz = (int)(i % g.nz);
        // windows a (x) with a*stepwinx - halfoutwx <= px <= a*stepwinx - halfoutwx + outwinx - 1
        int alo = px + g.halfoutwx - g.outwinx + 1;
        alo = alo <= 0 ? 0 : (alo + g.stepwinx - 1) / g.stepwinx;
        int ahi = (px + g.halfoutwx) / g.stepwinx;
        if (ahi > g.stepnumx - 1) ahi = g.stepnumx - 1;
        int blo = pz + g.halfoutwz - g.outwinz + 1;
        blo = blo <= 0 ? 0 : (blo + g.stepwinz - 1) / g.stepwinz;
        int bhi = (pz + g.halfoutwz) / g.stepwinz;
        if (bhi > g.stepnumz - 1) bhi = g.stepnumz - 1;
        float acc = 0.f, cacc = 0.f;
        for (int a = alo; a <= ahi; a++)
            for (int b = blo; b <= bhi; b++) {
                const int ixx = px - (a * g.stepwinx - g.halfoutwx), izz = pz - (b * g.stepwinz - g.halfoutwz);
                const int ipc = ixx * g.outwinz + izz;
                const float cr = __ldg(coefr + ipc);
                const float v = winout[(size_t)(a * g.stepnumz + b) * nout + ipc];
                acc = (float)((double)acc + (double)v * (double)cr);
                cacc = cacc + cr;
            }
        dec[i] = acc;
        coef[i] = cacc;
    }
}

}  // namespace swd
