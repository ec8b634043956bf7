// prop_tma.cuh -- velocity kernels whose pressure reads are staged by the Tensor Memory
// Accelerator.
//
// The velocity updates read the pressure at 2*LC columns around each cell and at a window of
// rows around it; the plain kernels issue those loads per thread (8 float4 column loads and 3
// row chunks for LC = 4), which holds registers while they are in flight.  Here persistent CTAs
// walk the grid's tiles (8 columns x 128 rows, the plain kernels' block layout) and, per tile,
// one thread issues cp.async.bulk.tensor copies of the pressure box (the tile widened by LC-1 /
// LC columns and 4*NB rows) into a shared-memory stage, completing on an mbarrier; two stages
// let the next tile's copy run while the current one is computed.  The per-cell code is the
// plain kernels' own (v_update4_l, src_v_phase_l) with the pressure read from the stage
// (PTile), so every guarded cell gets the same bits.  Velocities, material coefficients and the
// CPML memories are read and written per thread as before.
//
// TMA rules kept here: the box's first row (z0 - 4*NB) is a multiple of 4 floats (16 bytes);
// the first column may be negative or past the grid (the fill value 0 is never used by a
// guarded cell); stages start on 128-byte boundaries; each wait on an mbarrier gives up after
// a bounded number of tries, sets the error word and returns.
#pragma once
#include <cuda.h>
#include "prop.cuh"

namespace swd {

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *b, unsigned parity)
{
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(done) : "r"(smem_u32(b)), "r"(parity) : "memory");
    return done != 0;
}

// 2D tiled bulk copy global -> shared (no multicast), completion counted on bar
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int inner, int outer, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cta.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(smem_u32(dst)), "l"(map), "r"(inner), "r"(outer), "r"(smem_u32(bar)) : "memory");
}

// Tile geometry of the TMA velocity kernels
template <int LC>
struct VTile {
    static constexpr int NB = (LC + 3) / 4;                 // row chunks of the z window
    static constexpr int TX = 8, TZ = 128;                  // tile: one column per warp, four rows per lane
    static constexpr int PC = TX + 2 * LC - 1;              // box columns x0-(LC-1) .. x0+TX+LC-1
    static constexpr int PR = TZ + 8 * NB;                  // box rows z0-4NB .. z0+TZ+4NB-1
    static constexpr int SLOT = (PC * PR + 31) / 32 * 32;   // floats per box slot (128-byte aligned)
    static constexpr unsigned BOX_BYTES = PC * PR * 4;
    static constexpr int STAGES = 2;
    static constexpr long long WAIT_TRIES = 1ll << 24;     // bound of one mbarrier wait
};

// shared memory of a TMA velocity kernel with nbox pressure boxes per stage
template <int LC>
constexpr size_t vtile_smem(int nbox) { return sizeof(float) * VTile<LC>::STAGES * nbox * VTile<LC>::SLOT; }

// Tile loop shared by the kernels: NBOX boxes per stage from maps[0..NBOX); body(x0, z0, stage)
// computes a tile from the stage.  Returns false after a wait that gave up (err set).
template <int LC, int NBOX, class Body>
__device__ __forceinline__ bool vtile_loop(const Geo &g, const CUtensorMap *const *maps, int *err, Body body)
{
    using T = VTile<LC>;
    extern __shared__ __align__(128) float vt_sm[];
    __shared__ __align__(8) unsigned long long bar[T::STAGES];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int ntz_t = (g.ntz + T::TZ - 1) / T::TZ, ntile = ntz_t * ((g.ntx + T::TX - 1) / T::TX);
    auto issue = [&](int t, int s) {
        const int x0 = (t / ntz_t) * T::TX, z0 = (t % ntz_t) * T::TZ;
        float *st = vt_sm + (size_t)s * NBOX * T::SLOT;
        mbar_expect_tx(&bar[s], NBOX * T::BOX_BYTES);
#pragma unroll
        for (int b = 0; b < NBOX; b++) tma_load_2d(st + b * T::SLOT, maps[b], z0 - 4 * T::NB, x0 - (LC - 1), &bar[s]);
    };
    if (tid == 0) {
        for (int s = 0; s < T::STAGES; s++) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0)
        for (int s = 0; s < T::STAGES; s++) {
            const int t = blockIdx.x + s * gridDim.x;
            if (t < ntile) issue(t, s);
        }
    // bounded wait for use k of a stage; true when it completed
    auto wait_use = [&](int kk) {
        long long tries = 0;
        while (!mbar_try_wait(&bar[kk % T::STAGES], (kk / T::STAGES) & 1))
            if (++tries > T::WAIT_TRIES) return false;
        return true;
    };
    int k = 0;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x, k++) {
        const int s = k % T::STAGES;
        // The decision to give up is the whole CTA's: every thread waits (bounded), then the
        // block agrees.  On giving up no further tile is issued, and thread 0 waits (bounded
        // again) for the copies still in flight into this CTA's stages before all threads return
        // together, so the CTA does not exit under its own bulk copies.
        if (__syncthreads_or(!wait_use(k))) {
            if (tid == 0) {
                atomicExch(err, 1);
                for (int j = 0; j < T::STAGES; j++)
                    if (t + j * gridDim.x < ntile) wait_use(k + j);
            }
            __syncthreads();
            return false;
        }
        body((t / ntz_t) * T::TX, (t % ntz_t) * T::TZ, vt_sm + (size_t)s * NBOX * T::SLOT);
        __syncthreads();   // every thread is done with stage s before it is refilled
        if (tid == 0) {
            const int tn = t + T::STAGES * gridDim.x;
            if (tn < ntile) issue(tn, s);
        }
    }
    return true;
}

// Forward velocities of one wavefield (k_fwd_v<LC, 1, false> with TMA-staged pressure)
template <int LC>
__global__ void __launch_bounds__(256) k_fwd_v_tma(const FwdArgs a, const __grid_constant__ CUtensorMap tp, int *err)
{
    using T = VTile<LC>;
    const CUtensorMap *maps[1] = {&tp};
    const Geo &g = a.g;
    vtile_loop<LC, 1>(g, maps, err, [&](int x0, int z0t, const float *st) {
        const int x = x0 + threadIdx.y, z0 = z0t + 4 * threadIdx.x;
        if (x < g.ntx && z0 < g.ntz)
            v_update4_l<LC, false>(g, a.c, a.m, a.w[0], g.odx, g.odz, x, z0,
                                   PTile{st, x0 - (LC - 1), z0t - 4 * T::NB, T::PR});
    });
}

// Backward velocities of both wavefields (k_bwd_v with TMA-staged pressures): box 0 the
// receiver pressure, box 1 the source pressure
template <int LC>
__global__ void __launch_bounds__(256) k_bwd_v_tma(const BwdArgs a, const __grid_constant__ CUtensorMap tpr,
                                                   const __grid_constant__ CUtensorMap tps, int *err)
{
    using T = VTile<LC>;
    const CUtensorMap *maps[2] = {&tpr, &tps};
    const Geo &g = a.g;
    const int it = *a.itp + a.itoff;
    vtile_loop<LC, 2>(g, maps, err, [&](int x0, int z0t, const float *st) {
        const int x = x0 + threadIdx.y, z0 = z0t + 4 * threadIdx.x;
        if (x >= g.ntx || z0 >= g.ntz) return;
        const size_t ip = (size_t)x * g.ldz + z0;
        bool in[4];
        const bool any = interior4(g, x, z0, in);
        if (any && it < a.nt - 2)
            src_v_phase_l<LC>(a, x, z0, ip, in, PTile{st + T::SLOT, x0 - (LC - 1), z0t - 4 * T::NB, T::PR});
        v_update4_l<LC, true>(g, a.c, a.m, a.r, -g.odx, -g.odz, x, z0, PTile{st, x0 - (LC - 1), z0t - 4 * T::NB, T::PR});
    });
}

}  // namespace swd
