// prop.cuh -- staggered-grid acoustic FDTD kernels (sm_100a).
//
// Layout in HBM: every field is x-major with z fastest and a leading dimension ldz that is
// ntz rounded up to 32, so a warp (32 lanes along z) reads one aligned 128-byte line.
// Material is read as three precomputed coefficient arrays (struct Mat: dt times the
// half-node buoyancies and dt*rho*vp^2, formed once per model).  CPML memory variables are only
// read and written where the profile coefficient a is non-zero (the PML frame).
//
// Arithmetic follows the reference kernels (acoustic_HLVSPRTMLc.cu:24-221, 434-817;
// forward/acoustic_hilbert_fftkz_HLForLc.cu:168-558) so FP32 results agree to rounding noise:
// derivative sums in tap order (each tap as (rc*odx)*(a-b), struct Taps), phi = b*phi + a*d,
// v += dt*b*(d+phi), p += dt*rho*vp*vp*(dvx+phi_x+dvz+phi_z).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace swd {

constexpr int MAXLC = 8;

struct Geo {
    int ntx, ntz, ldz, pmlc, Lc;
    float odx, odz;     // (float)(1.0/(double)dx), (float)(1.0/(double)dz)
    float dt;
    float rc[MAXLC];
    // stencil coefficients folded with the spacing, formed on the host in float:
    // cx = rc * odx, cz = rc * odz, ncx = rc * (-odx), ncz = rc * (-odz)
    float cx[MAXLC], cz[MAXLC], ncx[MAXLC], ncz[MAXLC];
    // lean box [lx0, lx1) x [lz0, lz1): cells whose CPML coefficients a (both grids) are zero,
    // inside the strip band, so every update guard holds (empty when lx0 >= lx1)
    int lx0, lx1, lz0, lz1;
};

// Whether the calling (32, 8) block's 8 columns x 128 rows lie in the lean box: there every cell
// is updated, no CPML memory term is formed (its coefficient is zero, so the general path adds
// the same zero) and no strip cell is met, and the step kernels take a path without those
// branches.  Block-uniform.
__device__ __forceinline__ bool lean_block(const Geo &g)
{
    const int x0 = blockIdx.y * 8, z0 = blockIdx.x * 128;
    return x0 >= g.lx0 && x0 + 8 <= g.lx1 && z0 >= g.lz0 && z0 + 128 <= g.lz1;
}

struct Cpml {
    const float *ax, *axh, *az, *azh, *bx, *bxh, *bz, *bzh;
};

// Material coefficients of the updates, formed once per model (k_material) with the same
// operations and order the per-cell expressions use, so the updates are unchanged bit for
// bit:  cbx = dt * rcp(0.5*(rho[x] + rho[x+1])),  cbz = dt * rcp(0.5*(rho[z] + rho[z+1])),
// ck = ((dt*rho)*vp)*vp.  vx += cbx*(d + phi), vz += cbz*(d + phi), p += ck*(sum).
struct Mat {
    const float *cbx, *cbz, *ck;
    const float *kap;    // (rho*vp)*vp, the dp/dt factor of the imaging condition
};

// dp/dt of the source wavefield, stored by the forward pass on the interior for a backward
// pass that does not reconstruct the source wavefield.  Layout [step][x - pmlc][z - zlo] with
// row pitch ldr (the interior rows rounded out to whole 4-cell chunks); prec 0 f32, else a
// 16-bit code of enc16 with one scale (max |dp/dt|) per (step, warp of cell4), i.e. per 128
// rows of one column, so no block-wide reduction is needed.  Stores and loads are streaming
// (evict-first): each step's values are read once, by the backward pass.
struct DpStore {
    void *buf;       // nullptr: not stored
    float *scale;
    int prec, zlo, ldr, nwarps;
    long long step;  // elements per step
};

// forward pressure-kernel modes
constexpr int FP_PLAIN = 0, FP_BORN = 1, FP_STORE = 2, FP_SCAT = 3;

// One wavefield updated in place.
struct Wave {
    float *p, *vx, *vz;
    float *ppx, *ppz;   // CPML memory of the v updates (phi_p_x, phi_p_z)
    float *pvx, *pvz;   // CPML memory of the p update (phi_vx_x, phi_vz_z)
};

// Receivers grouped by well column: wcol[x] = well index or -1; wmap[w*ldz + z] = trace or -1.
struct Wells {
    const int *wcol;
    const int *wmap;
};

// Strip storage of the source-wavefield boundary band (Lc cells inside the interior
// edge).  Layout per step: [top nx*Lc][bottom nx*Lc][left Lc*nzs][right Lc*nzs], z fastest
// within each strip.  prec: 0 f32, 1 f16, 2 bf16; compressed strips carry one scale per
// (step, x-block) in `scale`.
struct Strips {
    void *buf;
    float *scale;
    int slen, prec, nscale;
};

// Batched launches (blockIdx.z = shot of the batch): per-shot scalars and offsets.  Every
// per-shot grid array of a batch is one allocation with a fixed per-shot stride (bstride
// elements, guard bands included); traces, wavelets and well maps are concatenated.
struct ShotDesc {
    int sx, sz, nt;
    int tshift;          // nt - (longest nt of the batch): backward time index offset
    int wav_off;         // first wavelet sample of the shot
    int wmap_off;        // first well row of the shot in the batch's wmap
    long long seis_off;  // first trace sample of the shot in seis / rdata
};

struct Batch {
    const ShotDesc *desc;   // nullptr: not batched
    long long bstride;      // elements between consecutive shots' grid arrays
    long long strip_bytes;  // bytes between consecutive shots' strip stores
    long long scale_stride; // floats between consecutive shots' strip scales
    int nshots;
};

__device__ __forceinline__ Wave shift_wave(Wave w, long long o)
{
    w.p += o; w.vx += o; w.vz += o; w.ppx += o; w.ppz += o; w.pvx += o; w.pvz += o;
    return w;
}

__device__ __forceinline__ Strips shift_strips(Strips s, const Batch &bt, int b)
{
    if (s.buf) {
        s.buf = (char *)s.buf + (size_t)b * bt.strip_bytes;
        if (s.scale) s.scale += (size_t)b * bt.scale_stride;
    }
    return s;
}

__device__ __forceinline__ size_t cidx(int x, int z, int ldz) { return (size_t)x * ldz + z; }

// Whether the (32, 8) block of cell4() (rows 128*bx .. +127, columns 8*by .. +7) holds a cell
// of the strip band; uniform over the block, so blocks without strip cells skip the strip
// code, including the block reduction of 16-bit strips.
__device__ __forceinline__ bool block_has_strips(int ntx, int ntz, int pmlc, int Lc)
{
    const int x0 = blockIdx.y * 8, x1 = x0 + 7, z0 = blockIdx.x * 128, z1 = z0 + 127;
    auto hit = [&](int xa, int xb, int za, int zb) { return x0 <= xb && x1 >= xa && z0 <= zb && z1 >= za; };
    const int xl = pmlc, xr = ntx - pmlc - 1, zt = pmlc, zb = ntz - pmlc - 1;
    return hit(xl, xr, zt, zt + Lc - 1) || hit(xl, xr, zb - Lc + 1, zb) || hit(xl, xl + Lc - 1, zt, zb) ||
           hit(xr - Lc + 1, xr, zt, zb);
}

// 16-bit codes of a value v relative to its block's max |v| (mx >= |v|): prec 1 IEEE half of
// v/mx * 32768, prec 2 bfloat16 of v/mx, prec 3 int16 fixed point round(v/mx * 32767).  The
// quotient is v times the correctly rounded reciprocal of mx (enc16_inv, once per scale; no
// division per value), so |q| exceeds 1 by at most a rounding, which the codes absorb; for a
// subnormal mx, whose reciprocal would overflow, inv is 0 and the quotient is divided out.
__device__ __forceinline__ float enc16_inv(float mx) { return mx >= 1.17549435e-38f ? __frcp_rn(mx) : 0.f; }

__device__ __forceinline__ unsigned short enc16(float v, float mx, float inv, int prec)
{
    const float q = inv != 0.f ? v * inv : (mx > 0.f ? v / mx : 0.f);
    if (prec == 1) return __half_as_ushort(__float2half_rn(q * 32768.f));
    if (prec == 2) return __bfloat16_as_ushort(__float2bfloat16_rn(q));
    return (unsigned short)(short)__float2int_rn(q * 32767.f);
}

__device__ __forceinline__ float dec16(unsigned short u, float mx, int prec)
{
    if (prec == 1) return (__half2float(__ushort_as_half(u)) * (1.f / 32768.f)) * mx;
    if (prec == 2) return __bfloat162float(__ushort_as_bfloat16(u)) * mx;
    return ((float)(short)u * (1.f / 32767.f)) * mx;
}

// Index of cell (x, z) in the per-step strip vector, or -1.
__device__ __forceinline__ int strip_index(int x, int z, int ntx, int ntz, int pmlc, int Lc)
{
    const int nx = ntx - 2 * pmlc, nzs = ntz - 2 * pmlc - 2 * Lc;
    if (x < pmlc || x > ntx - pmlc - 1 || z < pmlc || z > ntz - pmlc - 1) return -1;
    if (z < pmlc + Lc) return (x - pmlc) * Lc + (z - pmlc);
    if (z >= ntz - pmlc - Lc) return Lc * nx + (x - pmlc) * Lc + (z - (ntz - pmlc - Lc));
    if (x < pmlc + Lc) return 2 * Lc * nx + (x - pmlc) * nzs + (z - pmlc - Lc);
    if (x >= ntx - pmlc - Lc) return 2 * Lc * nx + Lc * nzs + (x - (ntx - pmlc - Lc)) * nzs + (z - pmlc - Lc);
    return -1;
}

// ------------------------------------------------------------------------------------
// Plain path: two launches per time step, fields updated in place.  Each thread owns four
// consecutive cells of one column (z0 .. z0+3, z0 a multiple of 4) and moves them with
// 128-bit loads: an x-direction tap is one float4 of the neighbouring column, the
// z-direction taps come from the float4 chunks just above and below, already in
// registers.  Every field array carries a guard band (GUARD floats on both sides) so the
// chunks next to the grid edge are readable; their values only feed cells that fail the
// update guards.  Per-cell arithmetic is that of the reference kernels, element by element.
// ------------------------------------------------------------------------------------
constexpr int GUARD = 64;

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
// bring the line of a global address into L2 (no register result)
__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("{\n\t.reg .u64 ga;\n\tcvta.to.global.u64 ga, %0;\n\tprefetch.global.L2 [ga];\n\t}" ::"l"(p));
}
__device__ __forceinline__ float4 ldg4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float &el(float4 &v, int k) { return (&v.x)[k]; }
__device__ __forceinline__ float elc(const float4 &v, int k) { return (&v.x)[k]; }

// Stencil coefficients folded with the grid spacing: c[ic] = rc[ic] * (1/dx), so a tap costs
// one subtraction and one fused multiply-add (the reference forms rc*(a-b)*odx per tap; the
// folded form differs from it by rounding only).  The products are formed once on the host
// (Geo::cx ...), so the taps read them from the kernel's parameter bank instead of holding them
// in registers; the float product is the same on either side.
template <int LC>
struct Taps {
    const float (&c)[MAXLC];
    __device__ __forceinline__ Taps(const float (&f)[MAXLC]) : c(f) {}
};

// z-window of a column around z0: w[NB*4 + k] holds z0 + k for k in [-NB*4, 4 + NB*4)
template <int LC>
struct ZWin {
    static constexpr int NB = (LC + 3) / 4;
    float v[4 * (2 * NB + 1)];
    __device__ __forceinline__ void load(const float *col, int z0)
    {
#pragma unroll
        for (int b = -NB; b <= NB; b++) {
            const float4 q = ld4(col + z0 + 4 * b);
            v[4 * (b + NB) + 0] = q.x; v[4 * (b + NB) + 1] = q.y;
            v[4 * (b + NB) + 2] = q.z; v[4 * (b + NB) + 3] = q.w;
        }
    }
    __device__ __forceinline__ float at(int k) const { return v[4 * NB + k]; }   // z0 + k
};

// Where a velocity update reads the pressure: global memory (PGlobal), or a shared-memory tile
// staged by TMA (PTile: column x - c0, row z - r0, pr rows per column).  Both give the same
// values on every cell the update guards let through.
struct PGlobal {
    const float *p;
    int ldz;
    __device__ __forceinline__ float4 col(int x, int z0) const { return ld4(p + (size_t)x * ldz + z0); }
    template <int LC>
    __device__ __forceinline__ void zwin(ZWin<LC> &w, int x, int z0) const { w.load(p + (size_t)x * ldz, z0); }
};

struct PTile {
    const float *s;
    int c0, r0, pr;
    __device__ __forceinline__ float4 col(int x, int z0) const { return ld4(s + (x - c0) * pr + (z0 - r0)); }
    template <int LC>
    __device__ __forceinline__ void zwin(ZWin<LC> &w, int x, int z0) const { w.load(s + (x - c0) * pr - r0, z0); }
};

// velocity half step (reference kernels _vx/_vz, acoustic_HLVSPRTMLc.cu:24-118; receiver
// variants (WIDE) with the wider guards and -dx/-dz, :623-715), the pressure read through pl.
// Within each half the coefficient and the old velocity are loaded with the pressure taps,
// before the CPML branch and its store: a load after a store through a pointer the compiler
// cannot prove distinct waits for the branch, which adds a memory latency per half.  The
// arithmetic is the reference's, term by term.
// Scattered-field hooks (SC): 1 also returns the update sums d + phi of the four cells in
// (*sx, *sz) (zero where a velocity is not updated); 2 adds dcb * (*sx, *sz) to the update, the
// secondary source of an exact scattered field (coefficient difference dcbx, dcbz).
template <int LC, bool WIDE, class PL, int SC = 0, bool LEAN = false>
__device__ __forceinline__ void v_update4_l(const Geo &g, const Cpml &c, const Mat &m, Wave w, int x, int z0, const PL &pl, float4 *sx = nullptr, float4 *sz = nullptr,
                                            const float *dcbx = nullptr, const float *dcbz = nullptr)
{
    if constexpr (SC == 1) {
        *sx = make_float4(0.f, 0.f, 0.f, 0.f);
        *sz = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const int ntx = g.ntx, ntz = g.ntz, ldz = g.ldz;
    const size_t ip = (size_t)x * ldz + z0;
    const Taps<LC> tx(WIDE ? g.ncx : g.cx), tz(WIDE ? g.ncz : g.cz);
    // ---- vx: x taps from the neighbouring columns
    const bool colx = LEAN || (x >= LC - 1 && x <= ntx - LC - 1);
    if (colx) {
        bool gx[4];
        bool any = false;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int z = z0 + k;
            gx[k] = LEAN || (WIDE ? (z <= ntz - 1) : (z >= LC && z <= ntz - LC));
            any |= gx[k];
        }
        if (any) {
            const float4 cb = ldg4(m.cbx + ip);
            float4 v = ld4(w.vx + ip);
            float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int ic = 0; ic < LC; ic++) {
                const float4 a = pl.col(x + ic + 1, z0), b = pl.col(x - ic, z0);
#pragma unroll
                for (int k = 0; k < 4; k++) el(d, k) += tx.c[ic] * (elc(a, k) - elc(b, k));
            }
            float4 phi = make_float4(0.f, 0.f, 0.f, 0.f);
            const float ax = LEAN ? 0.f : __ldg(c.axh + x);
            if (!LEAN && ax != 0.f) {
                const float bx = __ldg(c.bxh + x);
                float4 po = ld4(w.ppx + ip);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    el(phi, k) = bx * elc(po, k) + ax * elc(d, k);
                    if (gx[k]) el(po, k) = elc(phi, k);
                }
                st4(w.ppx + ip, po);
            }
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (gx[k]) el(v, k) = elc(cb, k) * (elc(d, k) + elc(phi, k)) + elc(v, k);
            if constexpr (SC == 1) {
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (gx[k]) el(*sx, k) = elc(d, k) + elc(phi, k);
            }
            if constexpr (SC == 2) {
                const float4 db = ldg4(dcbx + ip);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (gx[k]) el(v, k) = fmaf(elc(db, k), elc(*sx, k), elc(v, k));
            }
            st4(w.vx + ip, v);
        }
    }
    // ---- vz: z taps from the column's own window
    const bool colz = LEAN || (WIDE ? (x >= 0 && x <= ntx - 1) : (x >= LC && x <= ntx - LC));
    if (colz) {
        bool gz[4];
        bool any = false;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int z = z0 + k;
            gz[k] = LEAN || (z >= LC - 1 && z <= ntz - LC - 1);
            any |= gz[k];
        }
        if (any) {
            const float4 cb = ldg4(m.cbz + ip);
            float4 v = ld4(w.vz + ip);
            ZWin<LC> pw;
            pl.zwin(pw, x, z0);
            float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int k = 0; k < 4; k++)
#pragma unroll
                for (int ic = 0; ic < LC; ic++) el(d, k) += tz.c[ic] * (pw.at(k + ic + 1) - pw.at(k - ic));
            float4 phi = make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 az = LEAN ? make_float4(0.f, 0.f, 0.f, 0.f) : ldg4(c.azh + z0);
            if (!LEAN && (az.x != 0.f || az.y != 0.f || az.z != 0.f || az.w != 0.f)) {
                const float4 bz = ldg4(c.bzh + z0);
                float4 po = ld4(w.ppz + ip);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    el(phi, k) = elc(bz, k) * elc(po, k) + elc(az, k) * elc(d, k);
                    if (gz[k] && elc(az, k) != 0.f) el(po, k) = elc(phi, k);
                    else el(phi, k) = 0.f;
                }
                st4(w.ppz + ip, po);
            }
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (gz[k]) el(v, k) = elc(cb, k) * (elc(d, k) + elc(phi, k)) + elc(v, k);
            if constexpr (SC == 1) {
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (gz[k]) el(*sz, k) = elc(d, k) + elc(phi, k);
            }
            if constexpr (SC == 2) {
                const float4 db = ldg4(dcbz + ip);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (gz[k]) el(v, k) = fmaf(elc(db, k), elc(*sz, k), elc(v, k));
            }
            st4(w.vz + ip, v);
        }
    }
}

template <int LC, bool WIDE, bool LEAN = false>
__device__ __forceinline__ void v_update4(const Geo &g, const Cpml &c, const Mat &m, Wave w, int x, int z0)
{
    v_update4_l<LC, WIDE, PGlobal, 0, LEAN>(g, c, m, w, x, z0, PGlobal{w.p, g.ldz});
}

// pressure step with CPML (reference kernel _p, :121-173) on the four cells; returns the
// new values in pn (old values where not updated) and the per-cell update flags.  The
// coefficient ck is loaded with the old pressure, before the CPML branches and their stores
// (see v_update4_l).  NEG: the receiver wavefield's -dx/-dz; LEAN: a block of the lean box.
template <int LC, bool NEG = false, bool LEAN = false>
__device__ __forceinline__ void p_update4(const Geo &g, const Cpml &c, const Mat &m, Wave w, int x, int z0,
                                          float4 &pn, bool upd[4], float4 *ssum = nullptr)
{
    const int ntx = g.ntx, ntz = g.ntz, ldz = g.ldz;
    const size_t ip = (size_t)x * ldz + z0;
    pn = ld4(w.p + ip);
    bool any = false;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int z = z0 + k;
        upd[k] = LEAN || (z >= LC && z <= ntz - LC && x >= LC && x <= ntx - LC);
        any |= upd[k];
    }
    if (!any) return;
    const float4 kc = ldg4(m.ck + ip);
    float4 dvx = make_float4(0.f, 0.f, 0.f, 0.f), dvz = make_float4(0.f, 0.f, 0.f, 0.f);
    const Taps<LC> tx(NEG ? g.ncx : g.cx), tz(NEG ? g.ncz : g.cz);
    ZWin<LC> vw;
    vw.load(w.vz + (size_t)x * ldz, z0);
#pragma unroll
    for (int ic = 0; ic < LC; ic++) {
        const float4 a = ld4(w.vx + ip + (size_t)ic * ldz), b = ld4(w.vx + ip - (size_t)(ic + 1) * ldz);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            el(dvx, k) += tx.c[ic] * (elc(a, k) - elc(b, k));
            el(dvz, k) += tz.c[ic] * (vw.at(k + ic) - vw.at(k - ic - 1));
        }
    }
    float4 phx = make_float4(0.f, 0.f, 0.f, 0.f), phz = make_float4(0.f, 0.f, 0.f, 0.f);
    const float ax = LEAN ? 0.f : __ldg(c.ax + x);
    if (!LEAN && ax != 0.f) {
        const float bx = __ldg(c.bx + x);
        float4 po = ld4(w.pvx + ip);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            el(phx, k) = bx * elc(po, k) + ax * elc(dvx, k);
            if (upd[k]) el(po, k) = elc(phx, k);
        }
        st4(w.pvx + ip, po);
    }
    const float4 az = LEAN ? make_float4(0.f, 0.f, 0.f, 0.f) : ldg4(c.az + z0);
    if (!LEAN && (az.x != 0.f || az.y != 0.f || az.z != 0.f || az.w != 0.f)) {
        const float4 bz = ldg4(c.bz + z0);
        float4 po = ld4(w.pvz + ip);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            el(phz, k) = elc(bz, k) * elc(po, k) + elc(az, k) * elc(dvz, k);
            if (upd[k] && elc(az, k) != 0.f) el(po, k) = elc(phz, k);
            else el(phz, k) = 0.f;
        }
        st4(w.pvz + ip, po);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float sk = elc(dvx, k) + elc(phx, k) + elc(dvz, k) + elc(phz, k);
        if (ssum) el(*ssum, k) = upd[k] ? sk : 0.f;
        if (upd[k]) el(pn, k) = elc(kc, k) * sk + elc(pn, k);
    }
}

// ------------------------------------------------------------------------------------
// State checkpoints of one wavefield (p, vx, vz and the four CPML memories), taken before
// step it whenever it % every == 0, snapshot it / every.  Layout: data
// [snapshot][array 7][ntx*ldz] elements of prec (0 f32, or a 16-bit code of enc16); 16-bit
// snapshots carry one scale (the max |value|) per (snapshot, array, 128 x 8 block) in
// scale[snapshot][array][nblocks].
// ------------------------------------------------------------------------------------
struct Ckpt {
    void *buf;
    float *scale;
    int every;           // 0: no checkpoints
    int prec;
    int nblocks;
    long long fstride;   // ntx * ldz
};

__device__ __forceinline__ float *wave_array(const Wave &w, int i)
{
    return i == 0 ? w.p : i == 1 ? w.vx : i == 2 ? w.vz : i == 3 ? w.ppx : i == 4 ? w.ppz : i == 5 ? w.pvx : w.pvz;
}

// Called by every thread of a (32, 8) block with its four cells (valid when `in`).
__device__ __forceinline__ void ckpt_save(const Ckpt &ck, const Wave &w, int snap, bool in, size_t ip)
{
    const int slot = blockIdx.y * gridDim.x + blockIdx.x;
    if (ck.prec == 0) {
        if (!in) return;
#pragma unroll 1
        for (int i = 0; i < 7; i++)
            st4((float *)ck.buf + ((size_t)snap * 7 + i) * ck.fstride + ip, ld4(wave_array(w, i) + ip));
        return;
    }
    __shared__ float smax[7];
    if (threadIdx.x < 7 && threadIdx.y == 0) smax[threadIdx.x] = 0.f;
    __syncthreads();
    float4 v[7];
#pragma unroll
    for (int i = 0; i < 7; i++) {
        v[i] = in ? ld4(wave_array(w, i) + ip) : make_float4(0.f, 0.f, 0.f, 0.f);
        float m = fmaxf(fmaxf(fabsf(v[i].x), fabsf(v[i].y)), fmaxf(fabsf(v[i].z), fabsf(v[i].w)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0 && m > 0.f) atomicMax((int *)&smax[i], __float_as_int(m));
    }
    __syncthreads();
    if (threadIdx.x < 7 && threadIdx.y == 0)
        ck.scale[((size_t)snap * 7 + threadIdx.x) * ck.nblocks + slot] = smax[threadIdx.x];
    if (!in) return;
#pragma unroll
    for (int i = 0; i < 7; i++) {
        const float mx = smax[i], inv = enc16_inv(mx);
        const size_t o = ((size_t)snap * 7 + i) * ck.fstride + ip;
        ushort4 h;
        h.x = enc16(v[i].x, mx, inv, ck.prec); h.y = enc16(v[i].y, mx, inv, ck.prec);
        h.z = enc16(v[i].z, mx, inv, ck.prec); h.w = enc16(v[i].w, mx, inv, ck.prec);
        *reinterpret_cast<ushort4 *>((unsigned short *)ck.buf + o) = h;
    }
}

// ------------------------------------------------------------------------------------
// Forward modelling
// ------------------------------------------------------------------------------------
struct FwdArgs {
    Geo g;
    Cpml c;
    const float *vp, *rho;
    Mat m;
    Wave w[2];           // w[1] is the Hilbert twin when NW == 2
    // time index = *itp + itoff (a device counter, so one captured graph serves every
    // chunk of steps); wavelet samples come from the device arrays wav0 / wav1
    const int *itp;
    int itoff;
    const float *wav0, *wav1;
    int sx, sz, nt;
    Wells wells;
    float *seis;         // [r_n][nt]
    Strips strips;       // save (forward pass of RTM), buf == nullptr to skip
    const int *colmap;   // well column -> kz column slot, or nullptr
    float2 *colbuf;      // [ncol][nt][ldz] (p, twin p)
    // Born modelling / adjoint support, read by the BORN instantiation of k_fwd_p only:
    //   s0_out  receives field 0's p-update sum S0 = dvx+phi_x+dvz+phi_z of step it at
    //           s0_out[(it % s0_mod) * s0_stride + cell] (0 where p is not updated); nullable
    //   dkappa  bulk-modulus perturbation; with NW == 2 field 1 gets the secondary source
    //           dt * dkappa * S0 after its own update and the receivers record field 1
    // seis == nullptr records nothing.
    float *s0_out;
    long long s0_stride;
    int s0_mod;
    const float *dkappa;
    Ckpt ck;             // field-0 state checkpoints, taken by the CKPT instantiation of k_fwd_v
    Batch bt;            // the BATCH instantiations (NW == 1): shot = blockIdx.z
    DpStore ds;          // the FP_STORE instantiation (NW == 1): dp/dt of each step
    // Exact scattered field (the SCAT instantiations, NW == 2): field 0 propagates in the
    // background model (m), field 1 is the difference u(m1) - u(m) of the perturbed and the
    // background wavefields, propagated in the perturbed model m1 with the secondary sources
    // dcb * (d + phi) of field 0 in the velocity updates and dck * S0 in the pressure update
    // (dcb, dck: coefficient differences m1 - m, formed in double).  The receivers record field
    // 1; colcomp >= 0 writes field 1's column into that component of colbuf only.
    Mat m1;
    const float *dcbx, *dcbz, *dck;
    int colcomp;
};

// The shot's view of a batched forward launch; false when the shot's record has ended.
__device__ __forceinline__ bool fwd_view(FwdArgs &a, int it)
{
    const int b = blockIdx.z;
    const ShotDesc d = a.bt.desc[b];
    if (it >= d.nt) return false;
    a.w[0] = shift_wave(a.w[0], (long long)b * a.bt.bstride);
    a.sx = d.sx; a.sz = d.sz; a.nt = d.nt;
    a.wav0 += d.wav_off;
    a.wells.wcol += (size_t)b * a.g.ntx;
    a.wells.wmap += (size_t)d.wmap_off * a.g.ldz;
    if (a.seis) a.seis += d.seis_off;
    a.strips = shift_strips(a.strips, a.bt, b);
    return true;
}

__device__ __forceinline__ bool interior(int x, int z, const Geo &g)
{
    return z >= g.pmlc && z <= g.ntz - g.pmlc - 1 && x >= g.pmlc && x <= g.ntx - g.pmlc - 1;
}

// The stored dp/dt chunk of cell4 (x, z0): element offset in its step, or -1 outside the store.
__device__ __forceinline__ long long dp_offset(const DpStore &ds, const Geo &g, int x, int z0)
{
    if (x < g.pmlc || x > g.ntx - g.pmlc - 1 || z0 < ds.zlo || z0 >= ds.zlo + ds.ldr) return -1;
    return (long long)(x - g.pmlc) * ds.ldr + (z0 - ds.zlo);
}

__device__ __forceinline__ int warp_slot()
{
    return (blockIdx.y * gridDim.x + blockIdx.x) * (blockDim.y) + threadIdx.y;
}

// dp/dt = kap * S of the interior cells of this thread's chunk (zero on the chunk's other
// cells), the warp's max for 16-bit codes, then a streaming store.  Whole warps call it.
__device__ __forceinline__ void store_dpdt(const DpStore &ds, const Mat &m, const Geo &g, int it, int x, int z0,
                                           bool in, float4 s)
{
    const long long off = in ? dp_offset(ds, g, x, z0) : -1;
    float4 dp = make_float4(0.f, 0.f, 0.f, 0.f);
    if (off >= 0) {
        const float4 kp = ldg4(m.kap + (size_t)x * g.ldz + z0);
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (z0 + k >= g.pmlc && z0 + k <= g.ntz - g.pmlc - 1) el(dp, k) = elc(kp, k) * elc(s, k);
    }
    const size_t base = (size_t)it * ds.step;
    if (ds.prec == 0) {
        if (off >= 0) __stcs(reinterpret_cast<float4 *>((float *)ds.buf + base + off), dp);
        return;
    }
    float mx = fmaxf(fmaxf(fabsf(dp.x), fabsf(dp.y)), fmaxf(fabsf(dp.z), fabsf(dp.w)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (threadIdx.x == 0) __stcs(ds.scale + (size_t)it * ds.nwarps + warp_slot(), mx);
    if (off >= 0) {
        const float inv = enc16_inv(mx);
        ushort4 h;
        h.x = enc16(dp.x, mx, inv, ds.prec); h.y = enc16(dp.y, mx, inv, ds.prec);
        h.z = enc16(dp.z, mx, inv, ds.prec); h.w = enc16(dp.w, mx, inv, ds.prec);
        __stcs(reinterpret_cast<ushort4 *>((unsigned short *)ds.buf + base + off), h);
    }
}

// stored dp/dt of the chunk at step `it` (decoded), zero outside the store
__device__ __forceinline__ float4 load_dpdt(const DpStore &ds, const Geo &g, int it, int x, int z0)
{
    const long long off = dp_offset(ds, g, x, z0);
    if (off < 0) return make_float4(0.f, 0.f, 0.f, 0.f);
    const size_t base = (size_t)it * ds.step;
    if (ds.prec == 0) return __ldcs(reinterpret_cast<const float4 *>((const float *)ds.buf + base + off));
    const float mx = __ldcs(ds.scale + (size_t)it * ds.nwarps + warp_slot());
    const ushort4 h = __ldcs(reinterpret_cast<const ushort4 *>((const unsigned short *)ds.buf + base + off));
    return make_float4(dec16(h.x, mx, ds.prec), dec16(h.y, mx, ds.prec), dec16(h.z, mx, ds.prec), dec16(h.w, mx, ds.prec));
}

// Programmatic dependent launch.  The RTM step kernels are launched (SWD_OPT_PDL) so that the
// next launch's CTAs may be scheduled while this launch's last CTAs still run.  Each step kernel
// first waits until its predecessor grid has completed and its memory is visible, then lets its
// own dependents be scheduled: they are placed only once every CTA of this grid has started, and
// they wait in turn, so no CTA waits on one that cannot run.  Without the launch attribute both
// instructions return at once.
__device__ __forceinline__ void pdl_begin()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// block (32, 8): lane -> four rows, warp -> one column; a block covers 128 rows x 8 columns
__device__ __forceinline__ void cell4(int &x, int &z0)
{
    z0 = (blockIdx.x * 32 + threadIdx.x) * 4;
    x = blockIdx.y * 8 + threadIdx.y;
}

// MB > 0 bounds the registers to MB blocks of 256 per SM (the variant for passes whose working
// set streams from HBM, where more resident warps keep more bytes in flight; same bits).  The
// twins without checkpoints are bounded to 5 blocks: the plain twin 48 registers instead of 52
// (AFor's velocity step 12.5 -> 11.6 us on 1601x801), the scattered-field twin 48 instead of 54
// (90.5 -> 80.6 us on 4001x1601).  The batched kernel, whose batch streams from HBM, takes 6
// (40 registers, no spill: 27.5 -> 24.3 us per step of four 1601x801 shots).
template <int LC, int NW, bool CKPT, bool BATCH = false, bool SCAT = false, int MB = 0>
__global__ void __launch_bounds__(256, MB > 0 ? MB : ((NW == 2 && LC <= 4 && !CKPT) ? 5 : (BATCH && LC <= 4) ? 6 : 0))
    k_fwd_v(const FwdArgs a0)
{
    pdl_begin();
    FwdArgs a = a0;
    if constexpr (BATCH) {
        if (!fwd_view(a, *a.itp + a.itoff)) return;
    }
    int x, z0;
    cell4(x, z0);
    if constexpr (CKPT) {
        const int it = *a.itp + a.itoff;
        if (it % a.ck.every == 0)
            ckpt_save(a.ck, a.w[0], it / a.ck.every, x < a.g.ntx && z0 < a.g.ntz, (size_t)x * a.g.ldz + z0);
    }
    if (x >= a.g.ntx || z0 >= a.g.ntz) return;
    if constexpr (SCAT) {
        static_assert(NW == 2, "the scattered field runs beside its background");
        float4 sx, sz;
        const PGlobal p0{a.w[0].p, a.g.ldz}, p1{a.w[1].p, a.g.ldz};
        if (lean_block(a.g)) {
            v_update4_l<LC, false, PGlobal, 1, true>(a.g, a.c, a.m, a.w[0], x, z0, p0, &sx, &sz);
            v_update4_l<LC, false, PGlobal, 2, true>(a.g, a.c, a.m1, a.w[1], x, z0, p1, &sx, &sz, a.dcbx,
                                                     a.dcbz);
        } else {
            v_update4_l<LC, false, PGlobal, 1>(a.g, a.c, a.m, a.w[0], x, z0, p0, &sx, &sz);
            v_update4_l<LC, false, PGlobal, 2>(a.g, a.c, a.m1, a.w[1], x, z0, p1, &sx, &sz, a.dcbx,
                                               a.dcbz);
        }
    } else if (lean_block(a.g)) {
#pragma unroll
        for (int k = 0; k < NW; k++) v_update4<LC, false, true>(a.g, a.c, a.m, a.w[k], x, z0);
    } else {
#pragma unroll
        for (int k = 0; k < NW; k++) v_update4<LC, false>(a.g, a.c, a.m, a.w[k], x, z0);
    }
}

// Blocks per SM of the batched pressure kernels, LC <= 4: the per-shot view of the arguments
// holds every shifted wave pointer in registers (96 and 120 unbounded, 2 blocks per SM); at 4
// blocks (64 registers) a batched survey ran 21% faster than unbounded and 5% faster than at 3
// blocks, with the same stack.  With the lean path the backward one is faster still at 5 (48
// registers, an 80-byte spill: 66.1 -> 62.4 us per step of four 1601x801 shots), the forward one
// not (32.0 against 32.3 us).
constexpr int BATCH_P_MIN_BLOCKS = 4;
constexpr int BATCH_BWD_P_MIN_BLOCKS = 5;

// Blocks per SM asked of the register allocator: 5 (48 registers) for one wavefield and for the
// twins of the modelling forward and of the scattered field (small spills there), 4 (64
// registers, no spill) for the Born twin and the batched kernel; left free for LC > 4.  The twin at its free 80 registers ran 3
// blocks per SM and its launches took 8% longer.
template <int LC, int NW, int MODE, bool BATCH>
constexpr int fwd_p_min_blocks()
{
    if (LC > 4) return 1;
    if (BATCH) return BATCH_P_MIN_BLOCKS;
    if (NW == 1) return MODE == FP_BORN ? 1 : 5;
    // Born twin: 4 (64 registers, no spill); the scattered-field twin at 5 (48 registers, a
    // 108-byte spill) ran 72.5 -> 68.9 us per step on 4001x1601, ahead of 4 blocks
    return (MODE == FP_PLAIN || MODE == FP_SCAT) ? 5 : 4;
}

// MB > 0 asks the register allocator for MB blocks of 256 per SM instead of the default bound
// (the autotuner's register-bound variants of the plain kernel; same code, same bits)
template <int LC, int NW, int MODE, bool BATCH = false, int MB = 0>
__global__ void __launch_bounds__(256, (MB > 0 ? MB : fwd_p_min_blocks<LC, NW, MODE, BATCH>()))
    k_fwd_p(const FwdArgs a0)
{
    pdl_begin();
    constexpr bool BORN = MODE == FP_BORN, SCAT = MODE == FP_SCAT;
    FwdArgs a = a0;
    const int it = *a.itp + a.itoff;
    if constexpr (BATCH) {
        if (!fwd_view(a, it)) return;
    }
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    const bool in = x < g.ntx && z0 < g.ntz;
    const bool lean = lean_block(g);
    float4 pn[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) pn[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f);   // field 0's p-update sum (Born, store)
    if (in) {
        const size_t ip = (size_t)x * g.ldz + z0;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            bool upd[4];
            const Mat &mw = (SCAT && w == 1) ? a.m1 : a.m;
            float4 *ss = (MODE != FP_PLAIN && w == 0) ? &s0 : nullptr;
            if (lean) p_update4<LC, false, true>(g, a.c, mw, a.w[w], x, z0, pn[w], upd, ss);
            else p_update4<LC>(g, a.c, mw, a.w[w], x, z0, pn[w], upd, ss);
            bool any = upd[0] || upd[1] || upd[2] || upd[3];
            if constexpr (SCAT) {
                if (w == 1) {
                    const float4 dk = ldg4(a.dck + ip);
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (upd[k]) el(pn[w], k) = fmaf(elc(dk, k), elc(s0, k), elc(pn[w], k));
                }
            }
            if constexpr (BORN) {
                if (w == 0 && a.s0_out) st4(a.s0_out + (size_t)(it % a.s0_mod) * a.s0_stride + ip, s0);
                if (w == 1 && a.dkappa) {
                    const float4 dk = ldg4(a.dkappa + ip);
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (upd[k]) el(pn[w], k) += g.dt * elc(dk, k) * elc(s0, k);
                }
            }
            if (x == a.sx && !(SCAT && w == 1)) {   // the source is the same in both models
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (a.sz == z0 + k) { el(pn[w], k) += (w == 0 ? a.wav0[it] : a.wav1[it]); any = true; }
            }
            if (any) st4(a.w[w].p + ip, pn[w]);
        }
        const int wc = a.seis ? __ldg(a.wells.wcol + x) : -1;
        if (wc >= 0) {
            const int4 tr = __ldg(reinterpret_cast<const int4 *>(a.wells.wmap + (size_t)wc * g.ldz + z0));
            const int t[4] = {tr.x, tr.y, tr.z, tr.w};
            constexpr int rf = ((BORN || SCAT) && NW == 2) ? 1 : 0;   // Born / scattered data: field 1
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (t[k] >= 0 && z0 + k < g.ntz) a.seis[(size_t)t[k] * a.nt + it] = elc(pn[rf], k);
            if (a.colmap) {
                float2 *cb = a.colbuf + ((size_t)wc * a.nt + it) * g.ldz + z0;
                if constexpr (SCAT) {
#pragma unroll
                    for (int k = 0; k < 4; k++) (&cb[k].x)[a.colcomp] = elc(pn[1], k);
                } else {
#pragma unroll
                    for (int k = 0; k < 4; k++) cb[k] = make_float2(elc(pn[0], k), elc(pn[NW - 1], k));
                }
            }
        }
    }
    // dp/dt = kappa * S on the interior, for the backward pass of the stored-source mode
    if constexpr (MODE == FP_STORE) store_dpdt(a.ds, a.m, g, it, x, z0, in, s0);
    // strips (field 0): uncompressed store, or per-(step, block) scaled half/bf16
    if (a.strips.buf && !lean && block_has_strips(g.ntx, g.ntz, g.pmlc, LC)) {
        int si[4];
#pragma unroll
        for (int k = 0; k < 4; k++) si[k] = (in && z0 + k < g.ntz) ? strip_index(x, z0 + k, g.ntx, g.ntz, g.pmlc, LC) : -1;
        if (a.strips.prec == 0) {
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (si[k] >= 0) ((float *)a.strips.buf)[(size_t)it * a.strips.slen + si[k]] = elc(pn[0], k);
        } else {
            __shared__ float smax;
            if (threadIdx.x == 0 && threadIdx.y == 0) smax = 0.f;
            __syncthreads();
            float v = 0.f;
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (si[k] >= 0) v = fmaxf(v, fabsf(elc(pn[0], k)));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
            if (threadIdx.x == 0 && v > 0.f) atomicMax((int *)&smax, __float_as_int(v));
            __syncthreads();
            const float mx = smax, inv = enc16_inv(mx);
            const int slot = blockIdx.y * gridDim.x + blockIdx.x;
            if (threadIdx.x == 0 && threadIdx.y == 0) a.strips.scale[(size_t)it * a.strips.nscale + slot] = mx;
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (si[k] >= 0)
                    ((unsigned short *)a.strips.buf)[(size_t)it * a.strips.slen + si[k]] = enc16(elc(pn[0], k), mx, inv, a.strips.prec);
        }
    }
}

// ------------------------------------------------------------------------------------
// RTM backward step, two launches (reference order acoustic_HLVSPRTMLc.cu:1079-1148):
//   B1: source p (interior, -dt) + dp/dt + source subtraction + strip restore;
//       receiver vx, vz (CPML, -dx/-dz, wide guards)
//   B2: source vx, vz (interior, -dt); receiver p (CPML) + hard injection; imaging
// ------------------------------------------------------------------------------------
struct BwdArgs {
    Geo g;
    Cpml c;
    const float *vp, *rho;
    Mat m;
    Wave s;              // source wavefield (p, vx, vz only)
    Wave r;              // receiver wavefield
    float *dpdt;
    const int *itp;      // time index = *itp + itoff
    int itoff;
    const float *wavsub; // wavelet; rick[it+1] is subtracted at the source
    int sx, sz, nt;
    Strips strips;       // restore
    Wells wells;
    const float *rdata;  // [r_n][nt] preprocessed data injected at the receivers
    double *I, *S, *R;   // FP64 imaging accumulators (R nullable)
    float *Ip, *Sp, *Rp; // FP32 sums of the current block of IMG_BLOCK steps (nullptr: FP64 every step)
    Batch bt;            // the BATCH instantiations: shot = blockIdx.z
    DpStore ds;          // stored-source backward (k_bwd_rcv_*): dp/dt of forward step it+1
};

// The shot's view of a batched backward launch: its own time index (every shot of a batch
// starts the backward pass at its own nt - 2, so shorter records finish early); false once
// the shot is done.
__device__ __forceinline__ bool bwd_view(BwdArgs &a, int &it)
{
    const int b = blockIdx.z;
    const ShotDesc d = a.bt.desc[b];
    it += d.tshift;
    if (it < 0) return false;
    const long long o = (long long)b * a.bt.bstride;
    a.s = shift_wave(a.s, o);
    a.r = shift_wave(a.r, o);
    a.dpdt += o;
    a.I += o;
    a.S += o;
    if (a.R) a.R += o;
    if (a.Ip) { a.Ip += o; a.Sp += o; }
    if (a.Rp) a.Rp += o;
    a.sx = d.sx; a.sz = d.sz; a.nt = d.nt;
    a.wavsub += d.wav_off;
    a.wells.wcol += (size_t)b * a.g.ntx;
    a.wells.wmap += (size_t)d.wmap_off * a.g.ldz;
    a.rdata += d.seis_off;
    a.strips = shift_strips(a.strips, a.bt, b);
    return true;
}

// one restored strip value; the scale slot is the forward block that saved the cell
__device__ __forceinline__ float strip_restore(const Strips &st, int it, int si, int x, int z, int nz_blocks)
{
    if (st.prec == 0) return ((const float *)st.buf)[(size_t)it * st.slen + si];
    const int slot = (x / 8) * nz_blocks + (z / 128);
    const float mx = st.scale[(size_t)it * st.nscale + slot];
    if (mx == 0.f) return 0.f;
    return dec16(((const unsigned short *)st.buf)[(size_t)it * st.slen + si], mx, st.prec);
}

// Phases of one RTM backward step on the four cells (x, z0..z0+3), shared by both launch
// pairings.  in[k]: interior cell; any: some cell of the four is interior.
//
// Source wavefield pressure of step it, interior only (fdtd_2d_GPU_kernel_p_backward
// :434-485, -dt), source subtraction, boundary-strip overwrite (:575-620); returns
// dp/dt = kap * div v in dp (0 outside the interior).
template <int LC, bool LEAN = false>
__device__ __forceinline__ void src_p_phase(const BwdArgs &a, int it, int x, int z0, size_t ip, const bool in[4],
                                            bool any, float4 &dp)
{
    const Geo &g = a.g;
    const int ldz = g.ldz;
    dp = make_float4(0.f, 0.f, 0.f, 0.f);
    const bool src_here = x == a.sx && a.sz >= z0 && a.sz < z0 + 4;
    if (any) {
        float4 dvx = make_float4(0.f, 0.f, 0.f, 0.f), dvz = make_float4(0.f, 0.f, 0.f, 0.f);
        const Taps<LC> tx(g.cx), tz(g.cz);
        ZWin<LC> vw;
        vw.load(a.s.vz + (size_t)x * ldz, z0);
#pragma unroll
        for (int ic = 0; ic < LC; ic++) {
            const float4 p1 = ld4(a.s.vx + ip + (size_t)ic * ldz), p2 = ld4(a.s.vx + ip - (size_t)(ic + 1) * ldz);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                el(dvx, k) += tx.c[ic] * (elc(p1, k) - elc(p2, k));
                el(dvz, k) += tz.c[ic] * (vw.at(k + ic) - vw.at(k - ic - 1));
            }
        }
        // (-dt)*rho*vp*vp = -ck and rho*vp*vp = kap exactly (same products, same order), so
        // the material coefficients replace vp and rho; ck is also what the receiver p reads
        const float4 ck = ldg4(a.m.ck + ip), kap = ldg4(a.m.kap + ip);
        float4 p = ld4(a.s.p + ip);
        const int nzb = (g.ntz + 127) / 128;
        const bool band = !LEAN && block_has_strips(g.ntx, g.ntz, g.pmlc, LC);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!in[k]) continue;
            el(p, k) = (-elc(ck, k)) * (elc(dvx, k) + elc(dvz, k)) + elc(p, k);
            el(dp, k) = elc(kap, k) * (elc(dvx, k) + elc(dvz, k));
            if (src_here && a.sz == z0 + k) el(p, k) -= a.wavsub[it + 1];
            if (band) {
                const int si = strip_index(x, z0 + k, g.ntx, g.ntz, g.pmlc, LC);
                if (si >= 0) el(p, k) = strip_restore(a.strips, it, si, x, z0 + k, nzb);
            }
        }
        if (src_here) {
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (a.sz == z0 + k && !in[k]) el(p, k) -= a.wavsub[it + 1];
        }
        st4(a.s.p + ip, p);
    } else if (src_here) {
        a.s.p[ip + (a.sz - z0)] -= a.wavsub[it + 1];
    }
}

// Source wavefield velocities, interior only (:488-573, -dt), the source pressure read through pl
template <int LC, class PL>
__device__ __forceinline__ void src_v_phase_l(const BwdArgs &a, int x, int z0, size_t ip, const bool in[4], const PL &pl)
{
    const Geo &g = a.g;
    const Taps<LC> tx(g.cx), tz(g.cz);
    float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int ic = 0; ic < LC; ic++) {
        const float4 p1 = pl.col(x + ic + 1, z0), p2 = pl.col(x - ic, z0);
#pragma unroll
        for (int k = 0; k < 4; k++) el(d, k) += tx.c[ic] * (elc(p1, k) - elc(p2, k));
    }
    // (-dt)*rcp(...) = -cbx exactly
    const float4 cbx = ldg4(a.m.cbx + ip);
    float4 vx = ld4(a.s.vx + ip);
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (in[k]) el(vx, k) = (-elc(cbx, k)) * elc(d, k) + elc(vx, k);
    st4(a.s.vx + ip, vx);
    ZWin<LC> pw;
    pl.zwin(pw, x, z0);
    d = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
        for (int ic = 0; ic < LC; ic++) el(d, k) += tz.c[ic] * (pw.at(k + ic + 1) - pw.at(k - ic));
    const float4 cbz = ldg4(a.m.cbz + ip);
    float4 vz = ld4(a.s.vz + ip);
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (in[k]) el(vz, k) = (-elc(cbz, k)) * elc(d, k) + elc(vz, k);
    st4(a.s.vz + ip, vz);
}

template <int LC>
__device__ __forceinline__ void src_v_phase(const BwdArgs &a, int x, int z0, size_t ip, const bool in[4])
{
    src_v_phase_l<LC>(a, x, z0, ip, in, PGlobal{a.s.p, a.g.ldz});
}

// Receiver wavefield pressure (CPML, -dx/-dz) and hard injection of the data (:717-782)
template <int LC, bool LEAN = false>
__device__ __forceinline__ float4 rcv_p_phase(const BwdArgs &a, int it, int x, int z0, size_t ip)
{
    const Geo &g = a.g;
    float4 pr;
    bool upd[4];
    p_update4<LC, true, LEAN>(g, a.c, a.m, a.r, x, z0, pr, upd);
    bool wr = upd[0] || upd[1] || upd[2] || upd[3];
    const int wc = __ldg(a.wells.wcol + x);
    if (wc >= 0) {
        const int4 tr = __ldg(reinterpret_cast<const int4 *>(a.wells.wmap + (size_t)wc * g.ldz + z0));
        const int t[4] = {tr.x, tr.y, tr.z, tr.w};
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (t[k] >= 0 && z0 + k < g.ntz) { el(pr, k) = a.rdata[(size_t)t[k] * a.nt + it]; wr = true; }
    }
    if (wr) st4(a.r.p + ip, pr);
    return pr;
}

__device__ __forceinline__ bool interior4(const Geo &g, int x, int z0, bool in[4])
{
    bool any = false;
#pragma unroll
    for (int k = 0; k < 4; k++) { in[k] = z0 + k < g.ntz && interior(x, z0 + k, g); any |= in[k]; }
    return any;
}

template <int LC, bool BATCH = false>
__global__ void __launch_bounds__(256) k_bwd_1(const BwdArgs a0)
{
    pdl_begin();
    BwdArgs a = a0;
    int it = *a.itp + a.itoff;
    if constexpr (BATCH) {
        if (!bwd_view(a, it)) return;
    }
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    if (x >= g.ntx || z0 >= g.ntz) return;
    const size_t ip = (size_t)x * g.ldz + z0;
    bool in[4];
    const bool any = interior4(g, x, z0, in);
    float4 dp;
    src_p_phase<LC>(a, it, x, z0, ip, in, any, dp);
    if (any) st4(a.dpdt + ip, dp);
    // receiver wavefield velocities (wide guards, negative spacing)
    v_update4<LC, true>(g, a.c, a.m, a.r, x, z0);
}

// Imaging condition of one backward step on four cells (sum_image_GPU_kernel_image,
// acoustic_HLVSPRTMLc.cu:785-817): I += dp/dt * p_r, S += (dp/dt)^2, R += p_r^2.  Without
// partial buffers every step adds its exact products into the FP64 accumulators.  With them
// the products are summed in FP32 (one FMA rounding per step) over blocks of IMG_BLOCK steps
// and each block sum is added into FP64 on the block's last step, it % IMG_BLOCK == 0, which
// includes the pass's final step it = 0; per step that moves 16 bytes per cell instead of 32.
constexpr int IMG_BLOCK = 64;

__device__ __forceinline__ void fold4(double *acc, float *part, const bool in[4], float4 v, bool fold)
{
    if (fold) {
        double2 *A2 = reinterpret_cast<double2 *>(acc);
        double2 a0 = A2[0], a1 = A2[1];
        double *av[4] = {&a0.x, &a0.y, &a1.x, &a1.y};
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (in[k]) *av[k] += (double)elc(v, k);
        A2[0] = a0;
        A2[1] = a1;
        st4(part, make_float4(0.f, 0.f, 0.f, 0.f));
    } else {
        st4(part, v);
    }
}

__device__ __forceinline__ void image4(const BwdArgs &a, size_t ip, const bool in[4], float4 dp4, float4 pr, int it)
{
    if (a.Ip) {
        const bool fold = it % IMG_BLOCK == 0;
        float4 pi = ld4(a.Ip + ip), ps = ld4(a.Sp + ip);
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (in[k]) {
                el(pi, k) = fmaf(elc(dp4, k), elc(pr, k), elc(pi, k));
                el(ps, k) = fmaf(elc(dp4, k), elc(dp4, k), elc(ps, k));
            }
        fold4(a.I + ip, a.Ip + ip, in, pi, fold);
        fold4(a.S + ip, a.Sp + ip, in, ps, fold);
        if (a.Rp) {
            float4 pq = ld4(a.Rp + ip);
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (in[k]) el(pq, k) = fmaf(elc(pr, k), elc(pr, k), elc(pq, k));
            fold4(a.R + ip, a.Rp + ip, in, pq, fold);
        }
        return;
    }
    double2 *I2 = reinterpret_cast<double2 *>(a.I + ip), *S2 = reinterpret_cast<double2 *>(a.S + ip);
    double2 i0 = I2[0], i1 = I2[1], s0 = S2[0], s1 = S2[1];
    double *iv[4] = {&i0.x, &i0.y, &i1.x, &i1.y}, *sv[4] = {&s0.x, &s0.y, &s1.x, &s1.y};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (!in[k]) continue;
        const double dp = (double)elc(dp4, k);
        *iv[k] += dp * (double)elc(pr, k);
        *sv[k] += dp * dp;
    }
    I2[0] = i0; I2[1] = i1; S2[0] = s0; S2[1] = s1;
    if (a.R) {
        double2 *R2 = reinterpret_cast<double2 *>(a.R + ip);
        double2 q0 = R2[0], q1 = R2[1];
        double *rv[4] = {&q0.x, &q0.y, &q1.x, &q1.y};
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (in[k]) *rv[k] += (double)elc(pr, k) * (double)elc(pr, k);
        R2[0] = q0; R2[1] = q1;
    }
}

// L2 prefetch of the imaging operands a step will read last
__device__ __forceinline__ void image_prefetch(const BwdArgs &a, size_t ip, int it)
{
    if (a.Ip) {
        prefetch_l2(a.Ip + ip);
        prefetch_l2(a.Sp + ip);
        if (it % IMG_BLOCK != 0) return;
    }
    prefetch_l2(a.I + ip);
    prefetch_l2(a.S + ip);
}

template <int LC, bool BATCH = false>
__global__ void __launch_bounds__(256, (LC <= 4 && !BATCH) ? 5 : 1) k_bwd_2(const BwdArgs a0)
{
    pdl_begin();
    BwdArgs a = a0;
    int it = *a.itp + a.itoff;
    if constexpr (BATCH) {
        if (!bwd_view(a, it)) return;
    }
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    if (x >= g.ntx || z0 >= g.ntz) return;
    const size_t ip = (size_t)x * g.ldz + z0;
    bool in[4];
    const bool any = interior4(g, x, z0, in);
    if (any) {   // the imaging operands are read last: start their DRAM reads now
        image_prefetch(a, ip, it);
        prefetch_l2(a.dpdt + ip);
    }
    if (any) src_v_phase<LC>(a, x, z0, ip, in);
    const float4 pr = rcv_p_phase<LC>(a, it, x, z0, ip);
    // imaging condition (sum_image_GPU_kernel_image :785-817)
    if (any) image4(a, ip, in, ld4(a.dpdt + ip), pr, it);
}

// ------------------------------------------------------------------------------------
// RTM backward step with the phases paired by kind (default; same per-cell arithmetic and the
// same images, bit for bit, as k_bwd_1 + k_bwd_2):
//   BV(it): receiver vx, vz of step it; source vx, vz of step it + 1 (none on the first
//           backward step, it = nt - 2, which starts from the final forward velocities)
//   BP(it): source p of step it (strips, source subtraction); receiver p of step it and the
//           injection; imaging with dp/dt from registers
// Each launch needs one kind of material coefficient for both wavefields (cbx, cbz; ck, kap)
// and dp/dt never goes to memory: 20 bytes less per interior cell and step.  The source
// velocities lag by one step (v of step 0 is never formed), so the angle gathers, which read
// them after every step, use k_bwd_1 + k_bwd_2.
// ------------------------------------------------------------------------------------
// MB as in k_fwd_v
template <int LC, bool BATCH = false, int MB = 0>
__global__ void __launch_bounds__(256, MB) k_bwd_v(const BwdArgs a0)
{
    pdl_begin();
    BwdArgs a = a0;
    int it = *a.itp + a.itoff;
    if constexpr (BATCH) {
        if (!bwd_view(a, it)) return;
    }
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    if (x >= g.ntx || z0 >= g.ntz) return;
    const size_t ip = (size_t)x * g.ldz + z0;
    if (lean_block(g)) {   // every cell interior, no CPML term, no strip
        const bool in[4] = {true, true, true, true};
        if (it < a.nt - 2) src_v_phase<LC>(a, x, z0, ip, in);
        v_update4<LC, true, true>(g, a.c, a.m, a.r, x, z0);
        return;
    }
    bool in[4];
    const bool any = interior4(g, x, z0, in);
    if (any && it < a.nt - 2) src_v_phase<LC>(a, x, z0, ip, in);
    v_update4<LC, true>(g, a.c, a.m, a.r, x, z0);
}

template <int LC, bool BATCH = false, int MB = 0>
__global__ void __launch_bounds__(256, MB > 0 ? MB : (LC > 4 ? 1 : BATCH ? BATCH_BWD_P_MIN_BLOCKS : 5)) k_bwd_p(const BwdArgs a0)
{
    pdl_begin();
    BwdArgs a = a0;
    int it = *a.itp + a.itoff;
    if constexpr (BATCH) {
        if (!bwd_view(a, it)) return;
    }
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    if (x >= g.ntx || z0 >= g.ntz) return;
    const size_t ip = (size_t)x * g.ldz + z0;
    if (lean_block(g)) {   // every cell interior, no CPML term, no strip
        const bool in[4] = {true, true, true, true};
        image_prefetch(a, ip, it);
        float4 dp;
        src_p_phase<LC, true>(a, it, x, z0, ip, in, true, dp);
        const float4 pr = rcv_p_phase<LC, true>(a, it, x, z0, ip);
        image4(a, ip, in, dp, pr, it);
        return;
    }
    bool in[4];
    const bool any = interior4(g, x, z0, in);
    if (any) image_prefetch(a, ip, it);
    float4 dp;
    src_p_phase<LC>(a, it, x, z0, ip, in, any, dp);
    const float4 pr = rcv_p_phase<LC>(a, it, x, z0, ip);
    if (any) image4(a, ip, in, dp, pr, it);
}

// ------------------------------------------------------------------------------------
// Backward step of the stored-source mode: the forward pass stored dp/dt, so only the
// receiver wavefield propagates.  Backward index it images with the dp/dt of forward step
// it + 1, the step whose pressure update the reconstruction at index it undoes.
//   R1: receiver vx, vz (CPML, -dx/-dz, wide guards)
//   R2: receiver p (CPML) + hard injection; FP64 imaging with the stored dp/dt
// ------------------------------------------------------------------------------------
template <int LC>
__global__ void __launch_bounds__(256) k_bwd_rcv_v(const BwdArgs a)
{
    pdl_begin();
    int x, z0;
    cell4(x, z0);
    if (x >= a.g.ntx || z0 >= a.g.ntz) return;
    if (lean_block(a.g)) v_update4<LC, true, true>(a.g, a.c, a.m, a.r, x, z0);
    else v_update4<LC, true>(a.g, a.c, a.m, a.r, x, z0);
}

template <int LC>
__global__ void __launch_bounds__(256, 5) k_bwd_rcv_p(const BwdArgs a)
{
    pdl_begin();
    const int it = *a.itp + a.itoff;
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    if (x >= g.ntx || z0 >= g.ntz) return;
    const int ldz = g.ldz;
    const size_t ip = (size_t)x * ldz + z0;
    const bool lean = lean_block(g);   // every cell interior and updated, no CPML term
    bool in[4];
    bool any = false;
#pragma unroll
    for (int k = 0; k < 4; k++) { in[k] = lean || (z0 + k < g.ntz && interior(x, z0 + k, g)); any |= in[k]; }
    if (any) image_prefetch(a, ip, it);
    float4 pr;
    bool upd[4];
    if (lean) p_update4<LC, true, true>(g, a.c, a.m, a.r, x, z0, pr, upd);
    else p_update4<LC, true>(g, a.c, a.m, a.r, x, z0, pr, upd);
    bool wr = upd[0] || upd[1] || upd[2] || upd[3];
    const int wc = __ldg(a.wells.wcol + x);
    if (wc >= 0) {
        const int4 tr = __ldg(reinterpret_cast<const int4 *>(a.wells.wmap + (size_t)wc * ldz + z0));
        const int t[4] = {tr.x, tr.y, tr.z, tr.w};
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (t[k] >= 0 && z0 + k < g.ntz) { el(pr, k) = a.rdata[(size_t)t[k] * a.nt + it]; wr = true; }
    }
    if (wr) st4(a.r.p + ip, pr);
    if (any) image4(a, ip, in, load_dpdt(a.ds, g, it + 1, x, z0), pr, it);
}

// ------------------------------------------------------------------------------------
// Angle-domain common-image gathers (sum_image_GPU_kernel_imageCIG, acoustic_HLVSPRTMLc.cu:
// 819-905, which the reference never launches), formed in each backward step's imaging launch:
// Poynting vectors -p*v of the source and receiver wavefields, their dot and magnitude
// products over the last delt steps (a ring of delt slots), the reflection half-angle
// 0.5*acos(dot/mag) in degrees, and p_s*p_r spread over the five 1-degree bins around it with
// weights exp(-ii^2/18) (bins < 2 and >= thetan dropped; cells with an undefined angle
// skipped).  Float arithmetic without contraction, the reference's mixed float/double angle.
// ------------------------------------------------------------------------------------
struct CigArgs {
    Geo g;
    Wave s, r;           // p, vx, vz of the source and receiver wavefields after the step
    const int *itp;      // time index = *itp + itoff
    int itoff, nt, thetan, delt;
    float *ring;         // [delt][2][ntx*ldz]
    float *cig;          // [ntx*ldz][thetan]
};

// one interior cell (x, z) of the gathers after backward step it
__device__ __forceinline__ void cig_cell(const CigArgs &a, int it, int x, int z)
{
    const Geo &g = a.g;
    const size_t fs = (size_t)g.ntx * g.ldz, ip = (size_t)x * g.ldz + z;
    const float ps = a.s.p[ip], pr = a.r.p[ip];
    const float fx = __fmul_rn(-ps, a.s.vx[ip]), fz = __fmul_rn(-ps, a.s.vz[ip]);
    const float fxr = __fmul_rn(-pr, a.r.vx[ip]), fzr = __fmul_rn(-pr, a.r.vz[ip]);
    const int slot = it % a.delt;
    a.ring[(size_t)slot * 2 * fs + ip] = __fadd_rn(__fmul_rn(fx, fxr), __fmul_rn(fz, fzr));
    a.ring[((size_t)slot * 2 + 1) * fs + ip] = __fmul_rn(sqrtf(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fz, fz))),
                                                         sqrtf(__fadd_rn(__fmul_rn(fxr, fxr), __fmul_rn(fzr, fzr))));
    if (a.nt - 2 - it + 1 < a.delt) return;
    float pre = 0.f, pst = 0.f;
    for (int ii = 0; ii < a.delt; ii++) {
        pre = __fadd_rn(pre, a.ring[(size_t)ii * 2 * fs + ip]);
        pst = __fadd_rn(pst, a.ring[((size_t)ii * 2 + 1) * fs + ip]);
    }
    const float tht = __fdiv_rn(pre, pst);
    const float ftheta = (float)(__ddiv_rn(__dmul_rn(__dmul_rn(0.5, (double)acosf(tht)), 180.0), 3.1415926));
    if (isnan(ftheta)) return;
    const float pp = __fmul_rn(ps, pr);
    float *c = a.cig + ip * a.thetan;
#pragma unroll
    for (int ii = -2; ii <= 2; ii++) {
        const int itheta = (int)ceilf((float)__dsub_rn((double)__fadd_rn(ftheta, (float)ii), 0.5));
        const float betaf = (float)(1.0 * ii * ii / (2.0 * 9.0));
        if (itheta >= 2 && itheta < a.thetan) c[itheta] = __fadd_rn(c[itheta], __fmul_rn(pp, expf(-betaf)));
    }
}

// k_bwd_2 with the gathers fused into its imaging: after the thread's own cells are updated
// (source v here, source p and receiver v by k_bwd_1, receiver p here), each interior cell's
// Poynting vectors are formed from the values the thread just wrote or that the previous
// launch left, i.e. from the state after the whole step.
template <int LC>
__global__ void __launch_bounds__(256) k_bwd_2_cig(const BwdArgs a, const CigArgs c)
{
    pdl_begin();
    const int it = *a.itp + a.itoff;
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    if (x >= g.ntx || z0 >= g.ntz) return;
    const size_t ip = (size_t)x * g.ldz + z0;
    bool in[4];
    const bool any = interior4(g, x, z0, in);
    if (any) src_v_phase<LC>(a, x, z0, ip, in);
    const float4 pr = rcv_p_phase<LC>(a, it, x, z0, ip);
    if (any) {
        image4(a, ip, in, ld4(a.dpdt + ip), pr, it);
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (in[k]) cig_cell(c, it, x, z0 + k);
    }
}

}  // namespace swd
