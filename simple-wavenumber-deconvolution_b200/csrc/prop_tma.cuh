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
            v_update4_l<LC, false>(g, a.c, a.m, a.w[0], x, z0,
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
        v_update4_l<LC, true>(g, a.c, a.m, a.r, x, z0, PTile{st, x0 - (LC - 1), z0t - 4 * T::NB, T::PR});
    });
}

}  // namespace swd

namespace swd {

// ------------------------------------------------------------------------------------
// Fully staged step kernels.  Every stencil operand of a tile (8 columns x 128 rows, the plain
// kernels' block layout) is moved by cp.async.bulk.tensor into a shared-memory stage: the
// neighbour columns and rows the taps read, the field updated in place and its material
// coefficient.  The bytes in flight are then bounded by shared memory instead of by the
// registers that per-thread loads must hold until they land, which is what limits the plain
// kernels on grids larger than L2.  Persistent CTAs walk the tiles with STAGES stages in
// flight; the CPML memories (frame tiles only), strips, sources and receivers are read per
// thread as in the plain kernels, and the per-cell arithmetic is theirs term by term, so the
// results are the same bits.
// ------------------------------------------------------------------------------------
constexpr int ST_TX = 8, ST_TZ = 128, ST_MAXBOX = 8;

// Boxes of one stage: box b covers rows z0t + dz[b] .. + rows and columns x0 + dx[b] .. + cols
// of its tensor map (box extents are fixed in the map) and lands at float offset off[b] of the
// stage; off[] are multiples of 32 floats (128 bytes).
struct StageBoxes {
    int nbox;
    int dz[ST_MAXBOX], dx[ST_MAXBOX], off[ST_MAXBOX];
    int stage_floats;
    unsigned bytes;
};

// Warp-specialised tile pipeline of the fully staged kernels.  The CTA is ST_CONS consumer
// warps (threadIdx.y = 0 .. ST_CONS-1, the tile's columns) and one producer warp (threadIdx.y ==
// ST_CONS).  Per stage s two mbarriers: full[s] completes when the stage's boxes have landed
// (expect_tx by the producer), empty[s] when all consumer warps are done with it (one arrive per
// warp).  The producer refills a stage as soon as it is empty, so no block-wide barrier stands
// between a tile's compute and the next copy.  body(x0, z0t, stage) runs on the consumers; a
// barrier it needs among them is cons_sync() (named barrier 1).
// Bounded waits: a wait that gives up sets the error word and a shared abort flag, which every
// other wait checks; the consumers take the decision to stop together (a vote on named barrier 1
// after each wait, so none is left inside body's barriers), and the producer, once it stops
// issuing, waits (bounded) for the copies it issued into stages not yet consumed, so the CTA does
// not exit under its own bulk copies.
constexpr int ST_CONS = 8;

__device__ __forceinline__ void cons_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// true when p holds on any consumer thread (all consumers call it)
__device__ __forceinline__ bool cons_any(bool p)
{
    unsigned r;
    asm volatile("{\n .reg .pred q, o;\n setp.ne.u32 q, %1, 0;\n barrier.red.or.pred o, 1, 256, q;\n selp.u32 %0, 1, 0, o;\n}"
                 : "=r"(r) : "r"((unsigned)p) : "memory");
    return r != 0;
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

template <int STAGES, class Body>
__device__ __forceinline__ void stage_loop_ws(const Geo &g, const CUtensorMap *const *maps, const StageBoxes &sb,
                                              int *err, Body body)
{
    extern __shared__ __align__(128) float st_sm[];
    __shared__ __align__(8) unsigned long long full[STAGES], empty[STAGES];
    __shared__ int abort_flag;
    const int warp = threadIdx.y, lane = threadIdx.x;
    const int ntz_t = (g.ntz + ST_TZ - 1) / ST_TZ, ntile = ntz_t * ((g.ntx + ST_TX - 1) / ST_TX);
    volatile int *ab = &abort_flag;
    auto give_up = [&]() {
        atomicExch(err, 1);
        *ab = 1;
    };
    // bounded wait; stops early once another wait gave up (unless drain)
    auto wait = [&](unsigned long long *b, unsigned parity, bool drain) {
        long long tries = 0;
        while (!mbar_try_wait(b, parity)) {
            if (!drain && *ab) return false;
            if (++tries > VTile<4>::WAIT_TRIES) {
                give_up();
                return false;
            }
        }
        return true;
    };
    if (warp == 0 && lane == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], ST_CONS);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == ST_CONS) {   // producer
        if (lane != 0) return;
        int k = 0;
        for (int t = blockIdx.x; t < ntile; t += gridDim.x, k++) {
            const int s = k % STAGES;
            if (k >= STAGES && !wait(&empty[s], ((k / STAGES) - 1) & 1, false)) break;
            const int x0 = (t / ntz_t) * ST_TX, z0 = (t % ntz_t) * ST_TZ;
            float *st = st_sm + (size_t)s * sb.stage_floats;
            mbar_expect_tx(&full[s], sb.bytes);
            for (int b = 0; b < sb.nbox; b++)
                tma_load_2d(st + sb.off[b], maps[b], z0 + sb.dz[b], x0 + sb.dx[b], &full[s]);
        }
        if (*ab) {
            // the last use j of each stage that was issued: wait for its copies to land
            for (int j = k - 1; j >= 0 && j >= k - STAGES; j--) wait(&full[j % STAGES], (j / STAGES) & 1, true);
        }
        return;
    }
    int k = 0;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x, k++) {
        const int s = k % STAGES;
        const bool ok = wait(&full[s], (k / STAGES) & 1, false);
        if (cons_any(!ok)) {
            if (warp == 0 && lane == 0) give_up();
            return;
        }
        body((t / ntz_t) * ST_TX, (t % ntz_t) * ST_TZ, st_sm + (size_t)s * sb.stage_floats);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// Stage layout of the forward pressure kernel: vx on columns x0-LC .. x0+TX+LC-2 (the x taps),
// vz on rows z0t-4NB .. z0t+TZ+4NB-1 (the z taps), p and ck on the tile.
template <int LC>
struct FwdPStage {
    static constexpr int NB = (LC + 3) / 4;
    static constexpr int VXC = ST_TX + 2 * LC - 1, VZR = ST_TZ + 8 * NB;
    static constexpr int OVX = 0, OVZ = OVX + (VXC * ST_TZ + 31) / 32 * 32, OP = OVZ + (ST_TX * VZR + 31) / 32 * 32,
                         OCK = OP + ST_TX * ST_TZ, FLOATS = OCK + ST_TX * ST_TZ;
    static constexpr unsigned BYTES = 4u * (VXC * ST_TZ + ST_TX * VZR + 2 * ST_TX * ST_TZ);
    static constexpr int STAGES = 3;
    __host__ __device__ static StageBoxes boxes()
    {
        StageBoxes b{};
        b.nbox = 4;
        b.dz[0] = 0;      b.dx[0] = -LC; b.off[0] = OVX;   // vx: TZ rows x VXC columns
        b.dz[1] = -4 * NB; b.dx[1] = 0;  b.off[1] = OVZ;   // vz: VZR rows x TX columns
        b.dz[2] = 0;      b.dx[2] = 0;   b.off[2] = OP;    // p
        b.dz[3] = 0;      b.dx[3] = 0;   b.off[3] = OCK;   // ck
        b.stage_floats = FLOATS;
        b.bytes = BYTES;
        return b;
    }
};

template <int LC>
constexpr size_t fwd_p_stage_smem() { return sizeof(float) * FwdPStage<LC>::STAGES * FwdPStage<LC>::FLOATS; }

// Whether the tile (x0.., z0t..) holds a cell of the strip band (block_has_strips for a tile)
__device__ __forceinline__ bool tile_has_strips(int x0, int z0t, int ntx, int ntz, int pmlc, int Lc)
{
    const int x1 = x0 + ST_TX - 1, z1 = z0t + ST_TZ - 1;
    auto hit = [&](int xa, int xb, int za, int zb) { return x0 <= xb && x1 >= xa && z0t <= zb && z1 >= za; };
    const int xl = pmlc, xr = ntx - pmlc - 1, zt = pmlc, zb = ntz - pmlc - 1;
    return hit(xl, xr, zt, zt + Lc - 1) || hit(xl, xr, zb - Lc + 1, zb) || hit(xl, xl + Lc - 1, zt, zb) ||
           hit(xr - Lc + 1, xr, zt, zb);
}

// Forward pressure step of one wavefield on a staged tile (k_fwd_p<LC, 1, FP_PLAIN> with every
// stencil operand read from the stage): the same per-cell arithmetic as p_update4, then the
// source, the receivers, the kz columns and the strips as k_fwd_p writes them.
template <int LC>
__global__ void __launch_bounds__(32 * (ST_CONS + 1)) k_fwd_p_staged(const FwdArgs a, const __grid_constant__ CUtensorMap tvx,
                                                      const __grid_constant__ CUtensorMap tvz,
                                                      const __grid_constant__ CUtensorMap tp,
                                                      const __grid_constant__ CUtensorMap tck, int *err)
{
    using S = FwdPStage<LC>;
    const CUtensorMap *maps[4] = {&tvx, &tvz, &tp, &tck};
    const StageBoxes sb = S::boxes();
    const Geo &g = a.g;
    const int it = *a.itp + a.itoff;
    const Wave w = a.w[0];
    stage_loop_ws<S::STAGES>(g, maps, sb, err, [&](int x0, int z0t, const float *st) {
        const int x = x0 + threadIdx.y, z0 = z0t + 4 * threadIdx.x;
        const bool in = x < g.ntx && z0 < g.ntz;
        const float *svx = st + S::OVX, *svz = st + S::OVZ + threadIdx.y * S::VZR, *sp = st + S::OP, *sck = st + S::OCK;
        const int zr = z0 - z0t;   // row of z0 in the tile
        const int wc = (in && a.seis) ? __ldg(a.wells.wcol + x) : -1;
        float4 pn = make_float4(0.f, 0.f, 0.f, 0.f);
        if (in) {
            const size_t ip = (size_t)x * g.ldz + z0;
            const int ntx = g.ntx, ntz = g.ntz;
            pn = ld4(sp + threadIdx.y * ST_TZ + zr);
            bool upd[4], any = false;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int z = z0 + k;
                upd[k] = z >= LC && z <= ntz - LC && x >= LC && x <= ntx - LC;
                any |= upd[k];
            }
            if (any) {
                float4 dvx = make_float4(0.f, 0.f, 0.f, 0.f), dvz = make_float4(0.f, 0.f, 0.f, 0.f);
                const Taps<LC> tx(g.cx), tz(g.cz);
                ZWin<LC> vw;
                vw.load(svz + 4 * S::NB, zr);   // row zr of the staged vz column, with its halo
                // vx column x + c sits at stage column x + c - (x0 - LC)
                const float *vxc = svx + (size_t)(threadIdx.y + LC) * ST_TZ + zr;
#pragma unroll
                for (int ic = 0; ic < LC; ic++) {
                    const float4 va = ld4(vxc + ic * ST_TZ), vb = ld4(vxc - (ic + 1) * ST_TZ);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        el(dvx, k) += tx.c[ic] * (elc(va, k) - elc(vb, k));
                        el(dvz, k) += tz.c[ic] * (vw.at(k + ic) - vw.at(k - ic - 1));
                    }
                }
                float4 phx = make_float4(0.f, 0.f, 0.f, 0.f), phz = make_float4(0.f, 0.f, 0.f, 0.f);
                const float ax = __ldg(a.c.ax + x);
                if (ax != 0.f) {
                    const float bx = __ldg(a.c.bx + x);
                    float4 po = ld4(w.pvx + ip);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        el(phx, k) = bx * elc(po, k) + ax * elc(dvx, k);
                        if (upd[k]) el(po, k) = elc(phx, k);
                    }
                    st4(w.pvx + ip, po);
                }
                const float4 az = ldg4(a.c.az + z0);
                if (az.x != 0.f || az.y != 0.f || az.z != 0.f || az.w != 0.f) {
                    const float4 bz = ldg4(a.c.bz + z0);
                    float4 po = ld4(w.pvz + ip);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        el(phz, k) = elc(bz, k) * elc(po, k) + elc(az, k) * elc(dvz, k);
                        if (upd[k] && elc(az, k) != 0.f) el(po, k) = elc(phz, k);
                        else el(phz, k) = 0.f;
                    }
                    st4(w.pvz + ip, po);
                }
                const float4 kc = ld4(sck + threadIdx.y * ST_TZ + zr);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const float sk = elc(dvx, k) + elc(phx, k) + elc(dvz, k) + elc(phz, k);
                    if (upd[k]) el(pn, k) = elc(kc, k) * sk + elc(pn, k);
                }
            }
            if (x == a.sx) {
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (a.sz == z0 + k) { el(pn, k) += a.wav0[it]; any = true; }
            }
            if (any) st4(w.p + ip, pn);
            if (wc >= 0) {
                const int4 tr = __ldg(reinterpret_cast<const int4 *>(a.wells.wmap + (size_t)wc * g.ldz + z0));
                const int t4[4] = {tr.x, tr.y, tr.z, tr.w};
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (t4[k] >= 0 && z0 + k < g.ntz) a.seis[(size_t)t4[k] * a.nt + it] = elc(pn, k);
                if (a.colmap) {
                    float2 *cb = a.colbuf + ((size_t)wc * a.nt + it) * g.ldz + z0;
#pragma unroll
                    for (int k = 0; k < 4; k++) cb[k] = make_float2(elc(pn, k), elc(pn, k));
                }
            }
        }
        // strips: uncompressed store, or per-(step, tile) scaled 16-bit codes (tile = plain block)
        if (a.strips.buf && tile_has_strips(x0, z0t, g.ntx, g.ntz, g.pmlc, LC)) {
            int si[4];
#pragma unroll
            for (int k = 0; k < 4; k++) si[k] = (in && z0 + k < g.ntz) ? strip_index(x, z0 + k, g.ntx, g.ntz, g.pmlc, LC) : -1;
            if (a.strips.prec == 0) {
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (si[k] >= 0) ((float *)a.strips.buf)[(size_t)it * a.strips.slen + si[k]] = elc(pn, k);
            } else {
                __shared__ float smax;
                if (threadIdx.x == 0 && threadIdx.y == 0) smax = 0.f;
                cons_sync();
                float v = 0.f;
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (si[k] >= 0) v = fmaxf(v, fabsf(elc(pn, k)));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
                if (threadIdx.x == 0 && v > 0.f) atomicMax((int *)&smax, __float_as_int(v));
                cons_sync();
                const float mx = smax, inv = enc16_inv(mx);
                const int slot = (x0 / ST_TX) * ((g.ntz + ST_TZ - 1) / ST_TZ) + z0t / ST_TZ;
                if (threadIdx.x == 0 && threadIdx.y == 0) a.strips.scale[(size_t)it * a.strips.nscale + slot] = mx;
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (si[k] >= 0)
                        ((unsigned short *)a.strips.buf)[(size_t)it * a.strips.slen + si[k]] = enc16(elc(pn, k), mx, inv, a.strips.prec);
                cons_sync();   // smax is read before a later strip tile resets it
            }
        }
    });
}

}  // namespace swd
