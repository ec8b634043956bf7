// prop_fused.cuh -- one launch per time step: fused staggered-grid FDTD step kernels.
//
// Each CTA owns a TX x TZ tile (x by z) of the padded grid and performs the whole time step
// for it from shared memory:
//   forward (v first):  p_old cross (tile + a (2Lc-1)-cell halo along x and along z) and the
//     material tile are staged in shared memory with coalesced column loads; vx_new is
//     computed on the tile widened by Lc-1 / Lc columns, vz_new on the tile widened by rows
//     (the halo part is recomputed from the same inputs, bit-identical to what the owning CTA
//     computes); then p_new on the tile, with CPML, source, receivers, strips, kz columns.
//   backward: the receiver wavefield as above (wide guards, -dx/-dz, hard injection), the
//     source wavefield p first (interior only, -dt, source subtraction, strip restore) on the
//     tile widened by Lc-1 / Lc, then v on the tile, and the FP64 imaging condition.
// Because halo values are recomputed, every updated field is double-buffered: a step reads
// the `in` copies and writes the `out` copies (the CPML memory of the p update, read only at
// its own cell, stays in place).  Cells outside the update guards are never written, so both
// copies of a field must be initialised identically (zero, or the final forward state for
// the source wavefield).
//
// Arithmetic is term-for-term that of prop.cuh / the reference kernels, so results match the
// one-cell-per-thread kernels up to FMA contraction choices.
#pragma once
#include "prop.cuh"

namespace swd {

struct Field2 {                 // double-buffered wavefield of one step
    const float *p, *vx, *vz, *ppx, *ppz;   // in
    float *po, *vxo, *vzo, *ppxo, *ppzo;    // out
    float *pvx, *pvz;                       // in place
};

struct FStepArgs {
    Geo g;
    Cpml c;
    const float *vp, *rho;
    Field2 w[2];
    const int *itp;
    int itoff;
    const float *wav0, *wav1;
    int sx, sz, nt;
    Wells wells;
    float *seis;
    Strips strips;
    const int *colmap;
    float2 *colbuf;
};

struct BStepArgs {
    Geo g;
    Cpml c;
    const float *vp, *rho;
    Field2 r;                   // receiver wavefield (CPML)
    const float *ps, *vxs, *vzs;      // source wavefield in
    float *pso, *vxso, *vzso;         // source wavefield out
    const int *itp;             // time index = *itp + itoff
    int itoff;
    const float *wavsub;        // wavelet; rick[it+1] is subtracted at the source
    int sx, sz, nt;
    Strips strips;              // restore
    Wells wells;
    const float *rdata;
    double *I, *S, *R;
};

template <int LC, int TX, int TZ>
struct Tile {
    static constexpr int H = 2 * LC - 1;
    static constexpr int PX = TX + 2 * H, PZ = TZ + 2 * H;     // p cross (rectangle, corners unused)
    static constexpr int VXN = TX + 2 * LC - 1;                  // vx_new columns: x0-LC .. x1+LC-2
    static constexpr int VZN = TZ + 2 * LC - 1;                  // vz_new rows:    z0-LC .. z1+LC-2
    static constexpr int RX = TX + 2 * LC, RZ = TZ + 2 * LC;     // rho: x0-LC .. x1+LC-1, same in z
    static constexpr int NT = 256, NWARP = NT / 32;
};

__device__ __forceinline__ bool in_grid(int x, int z, const Geo &g) { return x >= 0 && x < g.ntx && z >= 0 && z < g.ntz; }

// stage rho on [x0-LC, x1+LC) x [z0-LC, z1+LC); out-of-grid cells read as 1 (never used by
// an updated cell, keeps reciprocals finite)
template <int LC, int TX, int TZ>
__device__ __forceinline__ void load_rho(float *sR, const float *__restrict__ rho, const Geo &g, int x0, int z0)
{
    using T = Tile<LC, TX, TZ>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < T::RX; c += T::NWARP) {
        const int x = x0 - LC + c;
        for (int r = lane; r < T::RZ; r += 32) {
            const int z = z0 - LC + r;
            sR[c * T::RZ + r] = in_grid(x, z, g) ? __ldg(rho + (size_t)x * g.ldz + z) : 1.f;
        }
    }
}

// stage the cross [x0-H, x1+H) x [z0, z1) U [x0, x1) x [z0-H, z1+H) of a field
template <int LC, int TX, int TZ>
__device__ __forceinline__ void load_cross(float *sP, const float *__restrict__ src, const Geo &g, int x0, int z0)
{
    using T = Tile<LC, TX, TZ>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < T::PX; c += T::NWARP) {
        const int x = x0 - T::H + c;
        const bool center = c >= T::H && c < T::H + TX;
        const int rlo = center ? 0 : T::H, rhi = center ? T::PZ : T::H + TZ;
        for (int r = rlo + lane; r < rhi; r += 32) {
            const int z = z0 - T::H + r;
            sP[c * T::PZ + r] = in_grid(x, z, g) ? src[(size_t)x * g.ldz + z] : 0.f;
        }
    }
}

// velocity phase of a v-first field: vx_new on columns [x0-LC, x1+LC-1), vz_new on rows
// [z0-LC, z1+LC-1); own cells written to the out buffers.  WIDE: receiver guards.
template <int LC, int TX, int TZ, bool WIDE>
__device__ __forceinline__ void v_phase(const Geo &g, const Cpml &c, const Field2 &f, float odx, float odz,
                                        const float *sP, const float *sR, float *sVX, float *sVZ, int x0, int z0)
{
    using T = Tile<LC, TX, TZ>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ntx = g.ntx, ntz = g.ntz;
    // vx
    for (int k = warp; k < T::VXN * (TZ / 32); k += T::NWARP) {
        const int cc = k / (TZ / 32), rr = (k % (TZ / 32)) * 32 + lane;
        const int x = x0 - LC + cc, z = z0 + rr;
        float vn = 0.f;
        if (in_grid(x, z, g)) {
            const size_t ip = (size_t)x * g.ldz + z;
            const bool gx = WIDE ? (x >= LC - 1 && x <= ntx - LC - 1)
                                 : (z >= LC && z <= ntz - LC && x >= LC - 1 && x <= ntx - LC - 1);
            if (gx) {
                const int sc = cc + (T::H - LC), sr = rr + T::H;
                float d = 0.f;
#pragma unroll
                for (int ic = 0; ic < LC; ic++) d += g.rc[ic] * (sP[(sc + ic + 1) * T::PZ + sr] - sP[(sc - ic) * T::PZ + sr]) * odx;
                const float a = __ldg(c.axh + x);
                const bool own = cc >= LC && cc < LC + TX;
                float phi = 0.f;
                if (a != 0.f) {
                    phi = __ldg(c.bxh + x) * f.ppx[ip] + a * d;
                    if (own) f.ppxo[ip] = phi;
                }
                const float orho = __frcp_rn(0.5f * (sR[cc * T::RZ + rr + LC] + sR[(cc + 1) * T::RZ + rr + LC]));
                vn = g.dt * orho * (d + phi) + f.vx[ip];
                if (own) f.vxo[ip] = vn;
            } else {
                vn = f.vx[ip];
            }
        }
        sVX[cc * TZ + rr] = vn;
    }
    // vz
    for (int k = warp; k < TX * ((T::VZN + 31) / 32); k += T::NWARP) {
        const int cc = k / ((T::VZN + 31) / 32), rr = (k % ((T::VZN + 31) / 32)) * 32 + lane;
        if (rr >= T::VZN) continue;
        const int x = x0 + cc, z = z0 - LC + rr;
        float vn = 0.f;
        if (in_grid(x, z, g)) {
            const size_t ip = (size_t)x * g.ldz + z;
            const bool gz = WIDE ? (z >= LC - 1 && z <= ntz - LC - 1)
                                 : (z >= LC - 1 && z <= ntz - LC - 1 && x >= LC && x <= ntx - LC);
            if (gz) {
                const int sc = cc + T::H, sr = rr + (T::H - LC);
                float d = 0.f;
#pragma unroll
                for (int ic = 0; ic < LC; ic++) d += g.rc[ic] * (sP[sc * T::PZ + sr + ic + 1] - sP[sc * T::PZ + sr - ic]) * odz;
                const float a = __ldg(c.azh + z);
                const bool own = rr >= LC && rr < LC + TZ;
                float phi = 0.f;
                if (a != 0.f) {
                    phi = __ldg(c.bzh + z) * f.ppz[ip] + a * d;
                    if (own) f.ppzo[ip] = phi;
                }
                const float orho = __frcp_rn(0.5f * (sR[(cc + LC) * T::RZ + rr] + sR[(cc + LC) * T::RZ + rr + 1]));
                vn = g.dt * orho * (d + phi) + f.vz[ip];
                if (own) f.vzo[ip] = vn;
            } else {
                vn = f.vz[ip];
            }
        }
        sVZ[cc * T::VZN + rr] = vn;
    }
}

// pressure of a v-first field on the own tile from the staged velocities.  Returns p_new
// (p_old where not updated) and whether the cell was updated.
template <int LC, int TX, int TZ>
__device__ __forceinline__ float p_cell(const Geo &g, const Cpml &c, const float *__restrict__ vp, const Field2 &f,
                                        float odx, float odz, const float *sP, const float *sR, const float *sVX,
                                        const float *sVZ, int cc, int rr, int x, int z, bool &upd)
{
    using T = Tile<LC, TX, TZ>;
    float pn = sP[(cc + T::H) * T::PZ + rr + T::H];
    upd = false;
    if (!(z >= LC && z <= g.ntz - LC && x >= LC && x <= g.ntx - LC)) return pn;
    float dvx = 0.f, dvz = 0.f;
#pragma unroll
    for (int ic = 0; ic < LC; ic++) {
        dvx += g.rc[ic] * (sVX[(cc + LC + ic) * TZ + rr] - sVX[(cc + LC - ic - 1) * TZ + rr]) * odx;
        dvz += g.rc[ic] * (sVZ[cc * T::VZN + rr + LC + ic] - sVZ[cc * T::VZN + rr + LC - ic - 1]) * odz;
    }
    const size_t ip = (size_t)x * g.ldz + z;
    float phx = 0.f, phz = 0.f;
    const float ax = __ldg(c.ax + x);
    if (ax != 0.f) {
        phx = __ldg(c.bx + x) * f.pvx[ip] + ax * dvx;
        f.pvx[ip] = phx;
    }
    const float az = __ldg(c.az + z);
    if (az != 0.f) {
        phz = __ldg(c.bz + z) * f.pvz[ip] + az * dvz;
        f.pvz[ip] = phz;
    }
    const float v = __ldg(vp + ip);
    upd = true;
    return g.dt * sR[(cc + LC) * T::RZ + rr + LC] * v * v * (dvx + phx + dvz + phz) + pn;
}

// ---------------------------------------------------------------------------------------
// forward step
// ---------------------------------------------------------------------------------------
template <int LC, int NW, int TX, int TZ>
__global__ void __launch_bounds__(256) k_fwd_step(FStepArgs a)
{
    const int it = *a.itp + a.itoff;
    using T = Tile<LC, TX, TZ>;
    __shared__ float sP[T::PX * T::PZ];
    __shared__ float sR[T::RX * T::RZ];
    __shared__ float sVX[T::VXN * TZ];
    __shared__ float sVZ[TX * T::VZN];
    __shared__ float sPn[NW][TX * TZ];
    __shared__ float smax;
    const Geo &g = a.g;
    const int x0 = blockIdx.y * TX, z0 = blockIdx.x * TZ;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    load_rho<LC, TX, TZ>(sR, a.rho, g, x0, z0);
#pragma unroll
    for (int w = 0; w < NW; w++) {
        load_cross<LC, TX, TZ>(sP, a.w[w].p, g, x0, z0);
        __syncthreads();
        v_phase<LC, TX, TZ, false>(g, a.c, a.w[w], g.odx, g.odz, sP, sR, sVX, sVZ, x0, z0);
        __syncthreads();
        for (int k = warp; k < TX * (TZ / 32); k += T::NWARP) {
            const int cc = k / (TZ / 32), rr = (k % (TZ / 32)) * 32 + lane;
            const int x = x0 + cc, z = z0 + rr;
            float pn = 0.f;
            if (x < g.ntx && z < g.ntz) {
                bool upd;
                pn = p_cell<LC, TX, TZ>(g, a.c, a.vp, a.w[w], g.odx, g.odz, sP, sR, sVX, sVZ, cc, rr, x, z, upd);
                if (x == a.sx && z == a.sz) { pn += (w == 0 ? a.wav0[it] : a.wav1[it]); upd = true; }
                if (upd) a.w[w].po[(size_t)x * g.ldz + z] = pn;
            }
            sPn[w][cc * TZ + rr] = pn;
        }
        __syncthreads();
    }
    // receivers, kz columns, strips of field 0 from the own tile
    if (threadIdx.x == 0) smax = 0.f;
    float vmax = 0.f;
    for (int k = warp; k < TX * (TZ / 32); k += T::NWARP) {
        const int cc = k / (TZ / 32), rr = (k % (TZ / 32)) * 32 + lane;
        const int x = x0 + cc, z = z0 + rr;
        if (x >= g.ntx || z >= g.ntz) continue;
        const float p0 = sPn[0][cc * TZ + rr];
        // seis == nullptr: no record wanted (the RTM forward pass when no synthetic is asked for)
        const int wc = (a.seis || a.colmap) ? __ldg(a.wells.wcol + x) : -1;
        if (wc >= 0) {
            const int tr = __ldg(a.wells.wmap + (size_t)wc * g.ldz + z);
            if (tr >= 0 && a.seis) a.seis[(size_t)tr * a.nt + it] = p0;
            if (a.colmap) a.colbuf[((size_t)wc * a.nt + it) * g.ldz + z] = make_float2(p0, sPn[NW - 1][cc * TZ + rr]);
        }
        if (a.strips.buf) {
            const int si = strip_index(x, z, g.ntx, g.ntz, g.pmlc, LC);
            if (si >= 0) {
                if (a.strips.prec == 0) ((float *)a.strips.buf)[(size_t)it * a.strips.slen + si] = p0;
                else vmax = fmaxf(vmax, fabsf(p0));
            }
        }
    }
    if (a.strips.buf && a.strips.prec != 0) {
        // per-(step, tile) scale: normalise by the tile's max |p| on its strip cells
        for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        __syncthreads();
        if (lane == 0 && vmax > 0.f) atomicMax((int *)&smax, __float_as_int(vmax));
        __syncthreads();
        const float mx = smax, inv = enc16_inv(mx);
        const int slot = blockIdx.y * gridDim.x + blockIdx.x;
        if (threadIdx.x == 0) a.strips.scale[(size_t)it * a.strips.nscale + slot] = mx;
        for (int k = warp; k < TX * (TZ / 32); k += T::NWARP) {
            const int cc = k / (TZ / 32), rr = (k % (TZ / 32)) * 32 + lane;
            const int x = x0 + cc, z = z0 + rr;
            if (x >= g.ntx || z >= g.ntz) continue;
            const int si = strip_index(x, z, g.ntx, g.ntz, g.pmlc, LC);
            if (si < 0) continue;
            ((unsigned short *)a.strips.buf)[(size_t)it * a.strips.slen + si] = enc16(sPn[0][cc * TZ + rr], mx, inv, a.strips.prec);
        }
    }
}

// ---------------------------------------------------------------------------------------
// backward step
// ---------------------------------------------------------------------------------------
template <int LC, int TX, int TZ>
__device__ __forceinline__ float strip_value(const Strips &st, int it, int si, int x, int z, int nscale_z)
{
    if (st.prec == 0) return ((const float *)st.buf)[(size_t)it * st.slen + si];
    const int slot = (x / TX) * nscale_z + (z / TZ);
    const float mx = st.scale[(size_t)it * st.nscale + slot];
    if (mx == 0.f) return 0.f;
    return dec16(((const unsigned short *)st.buf)[(size_t)it * st.slen + si], mx, st.prec);
}

template <int LC, int TX, int TZ>
__global__ void __launch_bounds__(256) k_bwd_step(BStepArgs a)
{
    const int it = *a.itp + a.itoff;
    using T = Tile<LC, TX, TZ>;
    // source-field staging: v_old on the (TX+2H) x (TZ+2H) rectangle, p_new on the
    // (TX+2LC-1) x (TZ+2LC-1) rectangle [x0-LC+1, x1+LC-1] x [z0-LC+1, z1+LC-1]
    constexpr int SN = TX + 2 * LC - 1, SNZ = TZ + 2 * LC - 1;
    constexpr int U0 = T::PX * T::PZ + T::VXN * TZ + TX * T::VZN;      // receiver phase
    constexpr int U1 = 2 * T::PX * T::PZ + SN * SNZ;                    // source phase
    __shared__ float sU[U0 > U1 ? U0 : U1];
    __shared__ float sR[T::RX * T::RZ];
    __shared__ float sPr[TX * TZ];
    __shared__ float sDp[TX * TZ];
    const Geo &g = a.g;
    const int x0 = blockIdx.y * TX, z0 = blockIdx.x * TZ;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ntx = g.ntx, ntz = g.ntz, pmlc = g.pmlc;
    load_rho<LC, TX, TZ>(sR, a.rho, g, x0, z0);
    // ---- receiver wavefield: v then p, hard injection
    {
        float *sP = sU, *sVX = sU + T::PX * T::PZ, *sVZ = sVX + T::VXN * TZ;
        load_cross<LC, TX, TZ>(sP, a.r.p, g, x0, z0);
        __syncthreads();
        v_phase<LC, TX, TZ, true>(g, a.c, a.r, -g.odx, -g.odz, sP, sR, sVX, sVZ, x0, z0);
        __syncthreads();
        for (int k = warp; k < TX * (TZ / 32); k += T::NWARP) {
            const int cc = k / (TZ / 32), rr = (k % (TZ / 32)) * 32 + lane;
            const int x = x0 + cc, z = z0 + rr;
            float pn = 0.f;
            if (x < ntx && z < ntz) {
                bool upd;
                pn = p_cell<LC, TX, TZ>(g, a.c, a.vp, a.r, -g.odx, -g.odz, sP, sR, sVX, sVZ, cc, rr, x, z, upd);
                const int wc = __ldg(a.wells.wcol + x);
                if (wc >= 0) {
                    const int tr = __ldg(a.wells.wmap + (size_t)wc * g.ldz + z);
                    if (tr >= 0) { pn = a.rdata[(size_t)tr * a.nt + it]; upd = true; }
                }
                if (upd) a.r.po[(size_t)x * g.ldz + z] = pn;
            }
            sPr[cc * TZ + rr] = pn;
        }
        __syncthreads();
    }
    // ---- source wavefield: p first on the widened tile, then v on the tile
    {
        float *sVXo = sU, *sVZo = sU + T::PX * T::PZ, *sPs = sVZo + T::PX * T::PZ;
        // v_old on [x0-H, x1+H) x [z0-H, z1+H) (rectangles)
        for (int c = warp; c < T::PX; c += T::NWARP) {
            const int x = x0 - T::H + c;
            for (int r = lane; r < T::PZ; r += 32) {
                const int z = z0 - T::H + r;
                const bool ok = in_grid(x, z, g);
                const size_t ip = (size_t)x * g.ldz + z;
                sVXo[c * T::PZ + r] = ok ? a.vxs[ip] : 0.f;
                sVZo[c * T::PZ + r] = ok ? a.vzs[ip] : 0.f;
            }
        }
        __syncthreads();
        // p_new on [x0-LC+1, x1+LC-1] x [z0-LC+1, z1+LC-1]; dp/dt kept for own cells
        for (int c = warp; c < SN; c += T::NWARP) {
            const int x = x0 - LC + 1 + c;
            for (int r = lane; r < SNZ; r += 32) {
                const int z = z0 - LC + 1 + r;
                float p = 0.f, dp = 0.f;
                if (in_grid(x, z, g)) {
                    const size_t ip = (size_t)x * g.ldz + z;
                    p = a.ps[ip];
                    if (z >= pmlc && z <= ntz - pmlc - 1 && x >= pmlc && x <= ntx - pmlc - 1) {
                        const int sc = c + (T::H - LC + 1), sr = r + (T::H - LC + 1);   // this cell in the rectangles
                        float dvx = 0.f, dvz = 0.f;
#pragma unroll
                        for (int ic = 0; ic < LC; ic++) {
                            dvx += g.rc[ic] * (sVXo[(sc + ic) * T::PZ + sr] - sVXo[(sc - ic - 1) * T::PZ + sr]) * g.odx;
                            dvz += g.rc[ic] * (sVZo[sc * T::PZ + sr + ic] - sVZo[sc * T::PZ + sr - ic - 1]) * g.odz;
                        }
                        const float v = __ldg(a.vp + ip);
                        const float rh = sR[(c + 1) * T::RZ + r + 1];
                        p = (-g.dt) * rh * v * v * (dvx + dvz) + p;
                        dp = rh * v * v * (dvx + dvz);
                        if (x == a.sx && z == a.sz) p -= a.wavsub[it + 1];
                        const int si = strip_index(x, z, ntx, ntz, pmlc, LC);
                        if (si >= 0) p = strip_value<LC, TX, TZ>(a.strips, it, si, x, z, gridDim.x);
                        const bool own = c >= LC - 1 && c < LC - 1 + TX && r >= LC - 1 && r < LC - 1 + TZ;
                        if (own) {
                            a.pso[ip] = p;
                            sDp[(c - LC + 1) * TZ + (r - LC + 1)] = dp;
                        }
                    } else if (x == a.sx && z == a.sz) {
                        p -= a.wavsub[it + 1];
                        const bool own = c >= LC - 1 && c < LC - 1 + TX && r >= LC - 1 && r < LC - 1 + TZ;
                        if (own) a.pso[ip] = p;
                    }
                }
                sPs[c * SNZ + r] = p;
            }
        }
        __syncthreads();
        // v_new on the own tile (interior) and the imaging condition
        for (int k = warp; k < TX * (TZ / 32); k += T::NWARP) {
            const int cc = k / (TZ / 32), rr = (k % (TZ / 32)) * 32 + lane;
            const int x = x0 + cc, z = z0 + rr;
            if (x >= ntx || z >= ntz) continue;
            if (!(z >= pmlc && z <= ntz - pmlc - 1 && x >= pmlc && x <= ntx - pmlc - 1)) continue;
            const size_t ip = (size_t)x * g.ldz + z;
            const int sc = cc + LC - 1, sr = rr + LC - 1;    // this cell in sPs
            float d = 0.f;
#pragma unroll
            for (int ic = 0; ic < LC; ic++) d += g.rc[ic] * (sPs[(sc + ic + 1) * SNZ + sr] - sPs[(sc - ic) * SNZ + sr]) * g.odx;
            float orho = __frcp_rn(0.5f * (sR[(cc + LC) * T::RZ + rr + LC] + sR[(cc + LC + 1) * T::RZ + rr + LC]));
            a.vxso[ip] = (-g.dt) * orho * d + sVXo[(cc + T::H) * T::PZ + rr + T::H];
            d = 0.f;
#pragma unroll
            for (int ic = 0; ic < LC; ic++) d += g.rc[ic] * (sPs[sc * SNZ + sr + ic + 1] - sPs[sc * SNZ + sr - ic]) * g.odz;
            orho = __frcp_rn(0.5f * (sR[(cc + LC) * T::RZ + rr + LC] + sR[(cc + LC) * T::RZ + rr + LC + 1]));
            a.vzso[ip] = (-g.dt) * orho * d + sVZo[(cc + T::H) * T::PZ + rr + T::H];
            const double dp = (double)sDp[cc * TZ + rr], pr = (double)sPr[cc * TZ + rr];
            a.I[ip] += dp * pr;
            a.S[ip] += dp * dp;
            if (a.R) a.R[ip] += pr * pr;
        }
    }
}

}  // namespace swd
