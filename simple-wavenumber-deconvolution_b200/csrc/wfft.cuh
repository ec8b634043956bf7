// wfft.cuh -- one-warp complex FFTs of any length up to 512 for the deconvolution windows.
//
// A warp owns one transform and keeps it in registers: element e = lane + 32*r of a length-M
// buffer (M a power of two, 32 <= M <= 1024) sits in register r of lane `lane`.  Forward
// transforms of length M run decimation-in-frequency (natural order in, bit-reversed out);
// inverse ones decimation-in-time (bit-reversed in, natural out), so a forward -> pointwise ->
// inverse chain never permutes.  Butterflies whose partners are 32 or more elements apart pair
// registers of one lane; the last five stages pair lanes through __shfl_xor_sync.
//
// Lengths L that are not a power of two (the windows' fullw = filterwin + psfwin - 1 is always
// odd; the reference's own geometry gives the prime 101) use Bluestein's chirp-z identity
//   sum_j x_j e^{s 2 pi i jk/L} = c_k sum_j (x_j c_j) conj(c_{k-j}),   c_m = e^{s pi i m^2/L},
// a linear convolution done as a cyclic one of length M >= 2L - 1 with two length-M FFTs and
// the precomputed transform K of the symmetric chirp b~ (b~_m = b~_{M-m} = e^{pi i m^2/L} for
// m < L, 0 elsewhere): forward (s = -1) convolves with b, inverse (s = +1) with conj(b), whose
// transform is conj(K) because b~ is symmetric.  Power-of-two lengths L >= 32 transform
// directly (M = L) and store in natural order.
//
// The tables (chirp, K / M in bit-reversed order, twiddles) are built by k_wfft_tables in
// double precision and rounded to float once.  Complex products are written with explicit
// fused multiply-adds, so every caller of these functions rounds identically.
#pragma once
#include <cuda_runtime.h>

namespace swd {

// a*b and a*conj(b) with a fixed contraction: re = fma(a.x, b.x, -(a.y*b.y)), ...
__device__ __forceinline__ float2 wmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -__fmul_rn(a.y, b.y)), fmaf(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 wmulc(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, __fmul_rn(a.y, b.y)), fmaf(a.y, b.x, -__fmul_rn(a.x, b.y)));
}
__device__ __forceinline__ float2 wadd(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 wsub(float2 a, float2 b) { return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)); }
__device__ __forceinline__ float2 wshfl(float2 v, int m)
{
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// Transform length L and its tables.  Table layout (float2): [chirp L][K M][twiddles M/2];
// the chirp and K are unused when pow2.
struct WfftPlan {
    int L, M, logM, pow2;
    const float2 *chirp;   // e^{+pi i j^2 / L}, j < L
    const float2 *kern;    // K[bitrev(e)] / M, e < M
    const float2 *tw;      // e^{-2 pi i j / M}, j < M/2
};

__host__ __device__ inline int wfft_M(int L)
{
    int M = 32;
    const bool p2 = L >= 32 && (L & (L - 1)) == 0;
    if (p2) return L;
    while (M < 2 * L - 1) M <<= 1;
    return M;
}
__host__ __device__ inline size_t wfft_table_len(int L) { const int M = wfft_M(L); return (size_t)L + M + M / 2; }

__host__ __device__ inline WfftPlan wfft_plan(int L, const float2 *tables)
{
    WfftPlan p;
    p.L = L;
    p.M = wfft_M(L);
    p.pow2 = p.M == L;
    int lg = 0;
    while ((1 << lg) < p.M) lg++;
    p.logM = lg;
    p.chirp = tables;
    p.kern = tables + L;
    p.tw = tables + L + p.M;
    return p;
}

// Tables of one length L into t[0 .. wfft_table_len(L)), in double, rounded once.  Launch
// with any grid; threads stride over the entries.
__global__ void k_wfft_tables(float2 *t, int L)
{
    const int M = wfft_M(L), n = (int)wfft_table_len(L);
    int lg = 0;
    while ((1 << lg) < M) lg++;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s, c;
        if (i < L) {                       // chirp e^{+pi i j^2 / L}, argument reduced exactly
            const long long q = ((long long)i * i) % (2LL * L);
            sincospi((double)q / (double)L, &s, &c);
            t[i] = make_float2((float)c, (float)s);
        } else if (i < L + M) {            // K / M at bit-reversed position
            const int e = i - L;
            const int k = (int)(__brev((unsigned)e) >> (32 - lg));
            double re = 0.0, im = 0.0;
            for (int m = 0; m < M; m++) {
                const int j = m < L ? m : (m > M - L ? M - m : -1);
                if (j < 0) continue;
                const long long qc = ((long long)j * j) % (2LL * L);
                double bs, bc;
                sincospi((double)qc / (double)L, &bs, &bc);
                const long long qw = ((long long)m * k) % M;
                double ws, wc;
                sincospi(-2.0 * (double)qw / (double)M, &ws, &wc);
                re += bc * wc - bs * ws;
                im += bc * ws + bs * wc;
            }
            t[i] = make_float2((float)(re / M), (float)(im / M));
        } else {                           // twiddles e^{-2 pi i j / M}
            const int j = i - L - M;
            sincospi(-2.0 * (double)j / (double)M, &s, &c);
            t[i] = make_float2((float)c, (float)s);
        }
    }
}

// Forward-type DIF of the warp's M = 32*R elements (bit-reversed out); conj twiddles when inv.
template <int R>
__device__ __forceinline__ void warp_dif(float2 (&v)[R], const float2 *tw, bool inv)
{
    constexpr int M = 32 * R;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int hr = R / 2; hr >= 1; hr >>= 1) {
        const int step = M / (64 * hr);
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (r & hr) continue;
            float2 w = tw[(lane + 32 * (r & (hr - 1))) * step];
            if (inv) w.y = -w.y;
            const float2 a = v[r], b = v[r + hr];
            v[r] = wadd(a, b);
            v[r + hr] = wmul(wsub(a, b), w);
        }
    }
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool lo = (lane & h) == 0;
        float2 w = tw[(lane & (h - 1)) * (M / (2 * h))];
        if (inv) w.y = -w.y;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const float2 o = wshfl(v[r], h);
            v[r] = lo ? wadd(v[r], o) : wmul(wsub(o, v[r]), w);
        }
    }
}

// DIT of bit-reversed input (natural out); conj twiddles when inv.
template <int R>
__device__ __forceinline__ void warp_dit(float2 (&v)[R], const float2 *tw, bool inv)
{
    constexpr int M = 32 * R;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int h = 1; h <= 16; h <<= 1) {
        const bool lo = (lane & h) == 0;
        float2 w = tw[(lane & (h - 1)) * (M / (2 * h))];
        if (inv) w.y = -w.y;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const float2 o = wshfl(v[r], h);
            // lower' = lower + upper*w, upper' = lower - upper*w
            v[r] = lo ? wadd(v[r], wmul(o, w)) : wsub(o, wmul(v[r], w));
        }
    }
#pragma unroll
    for (int hr = 1; hr <= R / 2; hr <<= 1) {
        const int step = M / (64 * hr);
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (r & hr) continue;
            float2 w = tw[(lane + 32 * (r & (hr - 1))) * step];
            if (inv) w.y = -w.y;
            const float2 a = v[r], b = wmul(v[r + hr], w);
            v[r] = wadd(a, b);
            v[r + hr] = wsub(a, b);
        }
    }
}

// One transform of length P.L on x[j * sin], in place, by the calling warp (all 32 lanes).
// sign -1: forward e^{-2 pi i jk/L}; +1: inverse e^{+...}; unnormalised.
template <int R>
__device__ __forceinline__ void warp_fft(float2 *x, int sin, const WfftPlan &P, int sign)
{
    float2 v[R];
    const int lane = threadIdx.x & 31;
    const bool inv = sign > 0;
    if (P.pow2) {
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = x[(size_t)(lane + 32 * r) * sin];
        warp_dif<R>(v, P.tw, inv);
        const int lg = P.logM;
#pragma unroll
        for (int r = 0; r < R; r++) x[(size_t)(__brev((unsigned)(lane + 32 * r)) >> (32 - lg)) * sin] = v[r];
        return;
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int j = lane + 32 * r;
        float2 a = make_float2(0.f, 0.f);
        if (j < P.L) {
            const float2 c = P.chirp[j];
            a = inv ? wmul(x[(size_t)j * sin], c) : wmulc(x[(size_t)j * sin], c);
        }
        v[r] = a;
    }
    warp_dif<R>(v, P.tw, false);
#pragma unroll
    for (int r = 0; r < R; r++) {
        const float2 k = P.kern[lane + 32 * r];
        v[r] = inv ? wmulc(v[r], k) : wmul(v[r], k);
    }
    warp_dit<R>(v, P.tw, true);
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int k = lane + 32 * r;
        if (k < P.L) {
            const float2 c = P.chirp[k];
            x[(size_t)k * sin] = inv ? wmul(v[r], c) : wmulc(v[r], c);
        }
    }
}

// The calling warp's transforms t = warp, warp + warps, ... < B of one register width R (a
// function of its own, so each width gets its own register allocation).
template <int R>
__device__ __noinline__ void warp_fft_loop(float2 *s, const WfftPlan P, int B, int sin, int str, int sign)
{
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int t = warp; t < B; t += nw) warp_fft<R>(s + (size_t)t * str, sin, P, sign);
}

// B transforms of length P.L over the buffer s (element j of transform t at s[t*str + j*sin]),
// one warp per transform; whole block, ends with __syncthreads().
__device__ __forceinline__ void fft_pass(float2 *s, const WfftPlan &P, int B, int sin, int str, int sign)
{
    switch (P.logM) {
    case 5: warp_fft_loop<1>(s, P, B, sin, str, sign); break;
    case 6: warp_fft_loop<2>(s, P, B, sin, str, sign); break;
    case 7: warp_fft_loop<4>(s, P, B, sin, str, sign); break;
    case 8: warp_fft_loop<8>(s, P, B, sin, str, sign); break;
    case 9: warp_fft_loop<16>(s, P, B, sin, str, sign); break;
    default: warp_fft_loop<32>(s, P, B, sin, str, sign); break;
    }
    __syncthreads();
}

}  // namespace swd
