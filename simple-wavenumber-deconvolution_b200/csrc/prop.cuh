// prop.cuh -- staggered-grid acoustic FDTD kernels (sm_100a).
//
// Layout in HBM: every field is x-major with z fastest and a leading dimension ldz that is
// ntz rounded up to 32, so a warp (32 lanes along z) reads one aligned 128-byte line.
// Material is read as vp and rho (8 B/cell); dt*rho*vp^2 and the half-node buoyancy
// 1/(0.5*(rho_i + rho_i+1)) are formed in registers.  CPML memory variables are only
// read and written where the profile coefficient a is non-zero (the PML frame).
//
// Arithmetic follows the reference kernels term by term (acoustic_HLVSPRTMLc.cu:24-221,
// 434-817; forward/acoustic_hilbert_fftkz_HLForLc.cu:168-558) so FP32 results agree to
// rounding noise: derivative sums in tap order, phi = b*phi + a*d, v += dt*b*(d+phi),
// p += dt*rho*vp*vp*(dvx+phi_x+dvz+phi_z).
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
};

struct Cpml {
    const float *ax, *axh, *az, *azh, *bx, *bxh, *bz, *bzh;
};

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

__device__ __forceinline__ size_t cidx(int x, int z, int ldz) { return (size_t)x * ldz + z; }

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
// velocity half step:  vx, vz from p (reference kernels _vx/_vz, :24-118; receiver
// variants with the wider guards and -dx/-dz, :623-715).  WIDE selects the receiver
// back-propagation guards.
// ------------------------------------------------------------------------------------
template <int LC, bool WIDE>
__device__ __forceinline__ void v_update(const Geo &g, const Cpml &c, const float *__restrict__ rho,
                                         Wave w, float odx, float odz, int x, int z)
{
    const int ntx = g.ntx, ntz = g.ntz, ldz = g.ldz;
    const size_t ip = cidx(x, z, ldz);
    const bool gx = WIDE ? (z >= 0 && z <= ntz - 1 && x >= LC - 1 && x <= ntx - LC - 1)
                         : (z >= LC && z <= ntz - LC && x >= LC - 1 && x <= ntx - LC - 1);
    if (gx) {
        float d = 0.f;
#pragma unroll
        for (int ic = 0; ic < LC; ic++) d += g.rc[ic] * (w.p[ip + (ic + 1) * ldz] - w.p[ip - ic * ldz]) * odx;
        const float a = __ldg(c.axh + x);
        float phi = 0.f;
        if (a != 0.f) {
            phi = __ldg(c.bxh + x) * w.ppx[ip] + a * d;
            w.ppx[ip] = phi;
        }
        const float orho = __frcp_rn(0.5f * (__ldg(rho + ip) + __ldg(rho + ip + ldz)));
        w.vx[ip] = g.dt * orho * (d + phi) + w.vx[ip];
    }
    const bool gz = WIDE ? (z >= LC - 1 && z <= ntz - LC - 1 && x >= 0 && x <= ntx - 1)
                         : (z >= LC - 1 && z <= ntz - LC - 1 && x >= LC && x <= ntx - LC);
    if (gz) {
        float d = 0.f;
#pragma unroll
        for (int ic = 0; ic < LC; ic++) d += g.rc[ic] * (w.p[ip + (ic + 1)] - w.p[ip - ic]) * odz;
        const float a = __ldg(c.azh + z);
        float phi = 0.f;
        if (a != 0.f) {
            phi = __ldg(c.bzh + z) * w.ppz[ip] + a * d;
            w.ppz[ip] = phi;
        }
        const float orho = __frcp_rn(0.5f * (__ldg(rho + ip) + __ldg(rho + ip + 1)));
        w.vz[ip] = g.dt * orho * (d + phi) + w.vz[ip];
    }
}

// pressure step with CPML (reference kernel _p, :121-173).  Returns true if p was updated.
template <int LC>
__device__ __forceinline__ bool p_update(const Geo &g, const Cpml &c, const float *__restrict__ vp,
                                         const float *__restrict__ rho, Wave w, float odx, float odz,
                                         int x, int z, float &pnew)
{
    const int ntx = g.ntx, ntz = g.ntz, ldz = g.ldz;
    const size_t ip = cidx(x, z, ldz);
    pnew = w.p[ip];
    if (!(z >= LC && z <= ntz - LC && x >= LC && x <= ntx - LC)) return false;
    float dvx = 0.f, dvz = 0.f;
#pragma unroll
    for (int ic = 0; ic < LC; ic++) {
        dvx += g.rc[ic] * (w.vx[ip + ic * ldz] - w.vx[ip - (ic + 1) * ldz]) * odx;
        dvz += g.rc[ic] * (w.vz[ip + ic] - w.vz[ip - (ic + 1)]) * odz;
    }
    float phx = 0.f, phz = 0.f;
    const float ax = __ldg(c.ax + x);
    if (ax != 0.f) {
        phx = __ldg(c.bx + x) * w.pvx[ip] + ax * dvx;
        w.pvx[ip] = phx;
    }
    const float az = __ldg(c.az + z);
    if (az != 0.f) {
        phz = __ldg(c.bz + z) * w.pvz[ip] + az * dvz;
        w.pvz[ip] = phz;
    }
    const float v = __ldg(vp + ip);
    pnew = g.dt * __ldg(rho + ip) * v * v * (dvx + phx + dvz + phz) + pnew;
    return true;
}

// ------------------------------------------------------------------------------------
// Forward modelling, two launches per time step (all fields in place).
// ------------------------------------------------------------------------------------
struct FwdArgs {
    Geo g;
    Cpml c;
    const float *vp, *rho;
    Wave w[2];           // w[1] is the Hilbert twin when NW == 2
    float amp[2];        // wavelet samples added at the source after the p update
    int sx, sz, it, nt;
    Wells wells;
    float *seis;         // [r_n][nt]
    Strips strips;       // save (forward pass of RTM), buf == nullptr to skip
    const int *colmap;   // well column -> kz column slot, or nullptr
    float2 *colbuf;      // [ncol][nt][ldz] (p, twin p)
};

template <int LC, int NW>
__global__ void __launch_bounds__(256) k_fwd_v(FwdArgs a)
{
    const int z = blockIdx.x * 32 + threadIdx.x;
    const int x = blockIdx.y * 8 + threadIdx.y;
    if (x >= a.g.ntx || z >= a.g.ntz) return;
#pragma unroll
    for (int k = 0; k < NW; k++) v_update<LC, false>(a.g, a.c, a.rho, a.w[k], a.g.odx, a.g.odz, x, z);
}

template <typename S> __device__ __forceinline__ S to_store(float v);
template <> __device__ __forceinline__ float to_store<float>(float v) { return v; }
template <> __device__ __forceinline__ __half to_store<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_store<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

template <int LC, int NW>
__global__ void __launch_bounds__(256) k_fwd_p(FwdArgs a)
{
    const int z = blockIdx.x * 32 + threadIdx.x;
    const int x = blockIdx.y * 8 + threadIdx.y;
    const Geo &g = a.g;
    const bool in = (x < g.ntx && z < g.ntz);
    float pn[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) pn[k] = 0.f;
    if (in) {
        const size_t ip = cidx(x, z, g.ldz);
#pragma unroll
        for (int k = 0; k < NW; k++) {
            bool upd = p_update<LC>(g, a.c, a.vp, a.rho, a.w[k], g.odx, g.odz, x, z, pn[k]);
            if (x == a.sx && z == a.sz) { pn[k] += a.amp[k]; upd = true; }
            if (upd) a.w[k].p[ip] = pn[k];
        }
        // receivers
        const int wc = __ldg(a.wells.wcol + x);
        if (wc >= 0) {
            const int tr = __ldg(a.wells.wmap + (size_t)wc * g.ldz + z);
            if (tr >= 0) a.seis[(size_t)tr * a.nt + a.it] = pn[0];
        }
        if (a.colmap) {
            const int cs = __ldg(a.colmap + x);
            if (cs >= 0) a.colbuf[((size_t)cs * a.nt + a.it) * g.ldz + z] = make_float2(pn[0], NW > 1 ? pn[NW - 1] : 0.f);
        }
    }
    // strips (field 0): uncompressed store, or per-(step, x-block) scaled half/bf16
    if (a.strips.buf) {
        const int si = in ? strip_index(x, z, g.ntx, g.ntz, g.pmlc, LC) : -1;
        if (a.strips.prec == 0) {
            if (si >= 0) ((float *)a.strips.buf)[(size_t)a.it * a.strips.slen + si] = pn[0];
        } else {
            // scale = max |p| over this block's strip cells; the block owns whole columns of
            // its x-range inside one 32-row z-band, so the scale slot is (step, blockIdx).
            __shared__ float smax;
            if (threadIdx.x == 0 && threadIdx.y == 0) smax = 0.f;
            __syncthreads();
            float v = si >= 0 ? fabsf(pn[0]) : 0.f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
            if (threadIdx.x == 0 && v > 0.f) atomicMax((int *)&smax, __float_as_int(v));
            __syncthreads();
            const float mx = smax;
            const int slot = blockIdx.y * gridDim.x + blockIdx.x;
            if (mx > 0.f) {
                // normalise first (|p|/mx <= 1 even when mx is denormal), then scale into the
                // half range; the restore undoes it in the same order
                if (threadIdx.x == 0 && threadIdx.y == 0) a.strips.scale[(size_t)a.it * a.strips.nscale + slot] = mx;
                if (si >= 0) {
                    const float q = pn[0] / mx;
                    if (a.strips.prec == 1) ((__half *)a.strips.buf)[(size_t)a.it * a.strips.slen + si] = to_store<__half>(q * 32768.f);
                    else ((__nv_bfloat16 *)a.strips.buf)[(size_t)a.it * a.strips.slen + si] = to_store<__nv_bfloat16>(q);
                }
            } else {
                // an all-zero block: store zeros so the restore never reads stale halves
                if (threadIdx.x == 0 && threadIdx.y == 0) a.strips.scale[(size_t)a.it * a.strips.nscale + slot] = 0.f;
                if (si >= 0) {
                    if (a.strips.prec == 1) ((__half *)a.strips.buf)[(size_t)a.it * a.strips.slen + si] = __float2half_rn(0.f);
                    else ((__nv_bfloat16 *)a.strips.buf)[(size_t)a.it * a.strips.slen + si] = __float2bfloat16_rn(0.f);
                }
            }
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
    Wave s;              // source wavefield (p, vx, vz only)
    Wave r;              // receiver wavefield
    float *dpdt;
    float sub;           // rick[it+1]
    int sx, sz, it, nt;
    Strips strips;       // restore
    Wells wells;
    const float *rdata;  // [r_n][nt] preprocessed data injected at the receivers
    double *I, *S, *R;   // FP64 imaging accumulators (R nullable)
};

// restore: value = (stored / unit) * mx, unit = 32768 for half, 1 for bf16
template <typename S>
__device__ __forceinline__ float strip_load(const Strips &st, int it, int si, float mx)
{
    const float unit = sizeof(S) == 2 && st.prec == 1 ? 32768.f : 1.f;
    return ((float)((const S *)st.buf)[(size_t)it * st.slen + si] / unit) * mx;
}
template <>
__device__ __forceinline__ float strip_load<float>(const Strips &st, int it, int si, float)
{
    return ((const float *)st.buf)[(size_t)it * st.slen + si];
}

template <int LC>
__global__ void __launch_bounds__(256) k_bwd_1(BwdArgs a)
{
    const int z = blockIdx.x * 32 + threadIdx.x;
    const int x = blockIdx.y * 8 + threadIdx.y;
    const Geo &g = a.g;
    if (x >= g.ntx || z >= g.ntz) return;
    const int ldz = g.ldz, pmlc = g.pmlc;
    const size_t ip = cidx(x, z, ldz);
    // source wavefield pressure, interior only (fdtd_2d_GPU_kernel_p_backward :434-485)
    if (z >= pmlc && z <= g.ntz - pmlc - 1 && x >= pmlc && x <= g.ntx - pmlc - 1) {
        float dvx = 0.f, dvz = 0.f;
#pragma unroll
        for (int ic = 0; ic < LC; ic++) {
            dvx += g.rc[ic] * (a.s.vx[ip + ic * ldz] - a.s.vx[ip - (ic + 1) * ldz]) * g.odx;
            dvz += g.rc[ic] * (a.s.vz[ip + ic] - a.s.vz[ip - (ic + 1)]) * g.odz;
        }
        const float v = __ldg(a.vp + ip), rh = __ldg(a.rho + ip);
        float p = (-g.dt) * rh * v * v * (dvx + dvz) + a.s.p[ip];
        a.dpdt[ip] = rh * v * v * (dvx + dvz);
        if (x == a.sx && z == a.sz) p -= a.sub;
        // boundary strips overwrite (fdtd_2d_GPU_kernel_borders_backward :575-620)
        const int si = strip_index(x, z, g.ntx, g.ntz, pmlc, LC);
        if (si >= 0) {
            if (a.strips.prec == 0) p = strip_load<float>(a.strips, a.it, si, 1.f);
            else {
                // the forward kernel's scale slot for this cell: same block tiling
                const int slot = (x / 8) * ((g.ntz + 31) / 32) + (z / 32);
                const float mx = a.strips.scale[(size_t)a.it * a.strips.nscale + slot];
                p = mx == 0.f ? 0.f
                              : (a.strips.prec == 1 ? strip_load<__half>(a.strips, a.it, si, mx)
                                                    : strip_load<__nv_bfloat16>(a.strips, a.it, si, mx));
            }
        }
        a.s.p[ip] = p;
    } else if (x == a.sx && z == a.sz) {
        a.s.p[ip] -= a.sub;
    }
    // receiver wavefield velocities (wide guards, negative spacing)
    v_update<LC, true>(g, a.c, a.rho, a.r, -g.odx, -g.odz, x, z);
}

template <int LC>
__global__ void __launch_bounds__(256) k_bwd_2(BwdArgs a)
{
    const int z = blockIdx.x * 32 + threadIdx.x;
    const int x = blockIdx.y * 8 + threadIdx.y;
    const Geo &g = a.g;
    if (x >= g.ntx || z >= g.ntz) return;
    const int ldz = g.ldz, pmlc = g.pmlc;
    const size_t ip = cidx(x, z, ldz);
    const bool interior = (z >= pmlc && z <= g.ntz - pmlc - 1 && x >= pmlc && x <= g.ntx - pmlc - 1);
    // source wavefield velocities, interior only (:488-573)
    if (interior) {
        float d = 0.f;
#pragma unroll
        for (int ic = 0; ic < LC; ic++) d += g.rc[ic] * (a.s.p[ip + (ic + 1) * ldz] - a.s.p[ip - ic * ldz]) * g.odx;
        float orho = __frcp_rn(0.5f * (__ldg(a.rho + ip) + __ldg(a.rho + ip + ldz)));
        a.s.vx[ip] = (-g.dt) * orho * d + a.s.vx[ip];
        d = 0.f;
#pragma unroll
        for (int ic = 0; ic < LC; ic++) d += g.rc[ic] * (a.s.p[ip + (ic + 1)] - a.s.p[ip - ic]) * g.odz;
        orho = __frcp_rn(0.5f * (__ldg(a.rho + ip) + __ldg(a.rho + ip + 1)));
        a.s.vz[ip] = (-g.dt) * orho * d + a.s.vz[ip];
    }
    // receiver pressure + hard injection (:717-782)
    float pr;
    bool upd = p_update<LC>(g, a.c, a.vp, a.rho, a.r, -g.odx, -g.odz, x, z, pr);
    const int wc = __ldg(a.wells.wcol + x);
    if (wc >= 0) {
        const int tr = __ldg(a.wells.wmap + (size_t)wc * ldz + z);
        if (tr >= 0) { pr = a.rdata[(size_t)tr * a.nt + a.it]; upd = true; }
    }
    if (upd) a.r.p[ip] = pr;
    // imaging condition in FP64 (sum_image_GPU_kernel_image :785-817)
    if (interior) {
        const double dp = (double)a.dpdt[ip];
        a.I[ip] += dp * (double)pr;
        a.S[ip] += dp * dp;
        if (a.R) a.R[ip] += (double)pr * (double)pr;
    }
}

}  // namespace swd
