// fft.cuh -- block-level complex FFTs in shared memory for power-of-two lengths.
//
// Forward transforms are decimation-in-frequency (natural order in, bit-reversed out);
// inverse transforms are decimation-in-time (bit-reversed in, natural out), so a
// forward -> pointwise -> inverse chain never permutes.  Butterflies with distance >= 32
// run through shared memory with __syncthreads(); the last five forward stages (first
// five inverse stages), whose partners sit in the same 32-element segment, run in
// registers with __shfl_xor_sync.  Sign conventions are cuFFT's/FFTW's: forward
// exp(-2*pi*i*j*k/N), inverse exp(+...), both unnormalised.
//
// Twiddles come from a table tw[j] = exp(-2*pi*i*j/N), j < N/2, built on the host in
// double precision, so the transform error stays at a few float ulps times log2(N).
#pragma once
#include <cuda_runtime.h>

namespace swd {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) { return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }  // a*conj(b)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

__device__ __forceinline__ float2 shfl_xor2(float2 v, int m)
{
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// Forward DIF on s[0..N) (N power of two, N >= 32), twiddle table tw of length N/2.
// All threads of the block must call it; blockDim.x must be a multiple of 32.
__device__ void block_fft_dif(float2 *s, int N, const float2 *__restrict__ tw)
{
    const int tid = threadIdx.x, nthr = blockDim.x;
    // stages with half-size d >= 32 through shared memory
    for (int d = N >> 1; d >= 32; d >>= 1) {
        const int tstride = N / (2 * d);   // twiddle index step for this stage
        for (int b = tid; b < N / 2; b += nthr) {
            const int k = b % d, base = (b / d) * 2 * d;
            const float2 a = s[base + k], c = s[base + k + d];
            s[base + k] = cadd(a, c);
            s[base + k + d] = cmul(csub(a, c), __ldg(tw + k * tstride));
        }
        __syncthreads();
    }
    // stages d = 16 .. 1 in registers: each warp owns whole 32-element segments
    const int lane = tid & 31, warp = tid >> 5, nw = nthr >> 5;
    for (int seg = warp; seg < N / 32; seg += nw) {
        float2 v = s[seg * 32 + lane];
        for (int d = 16; d >= 1; d >>= 1) {
            const float2 o = shfl_xor2(v, d);
            const bool lo = (lane & d) == 0;
            const int k = lane & (d - 1);
            // lower element: a + c; upper element: (a - c) * W_{2d}^k
            v = lo ? cadd(v, o) : cmul(csub(o, v), __ldg(tw + k * (N / (2 * d))));
        }
        s[seg * 32 + lane] = v;
    }
    __syncthreads();
}

// Inverse DIT on bit-reversed s[0..N) -> natural order (unnormalised, exp(+...)).
__device__ void block_ifft_dit(float2 *s, int N, const float2 *__restrict__ tw)
{
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nw = nthr >> 5;
    for (int seg = warp; seg < N / 32; seg += nw) {
        float2 v = s[seg * 32 + lane];
        for (int d = 1; d <= 16; d <<= 1) {
            const float2 o = shfl_xor2(v, d);
            const bool lo = (lane & d) == 0;
            const int k = lane & (d - 1);
            const float2 w = __ldg(tw + k * (N / (2 * d)));
            // t = conj(W)^k * upper; lower' = lower + t; upper' = lower - t
            if (lo) v = cadd(v, cmulc(o, w));
            else v = csub(o, cmulc(v, w));
        }
        s[seg * 32 + lane] = v;
    }
    __syncthreads();
    for (int d = 32; d < N; d <<= 1) {
        const int tstride = N / (2 * d);
        for (int b = tid; b < N / 2; b += nthr) {
            const int k = b % d, base = (b / d) * 2 * d;
            const float2 a = s[base + k];
            const float2 t = cmulc(s[base + k + d], __ldg(tw + k * tstride));
            s[base + k] = cadd(a, t);
            s[base + k + d] = csub(a, t);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int bitrev(int j, int logn) { return (int)(__brev((unsigned)j) >> (32 - logn)); }

}  // namespace swd
