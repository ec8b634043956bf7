// born.cuh -- exact discrete adjoint of the forward step, and checkpoint restore (sm_100a).
//
// The forward step (prop.cuh) is a linear map A on the state u = (p, vx, vz, psi_x, psi_z,
// phi_x, phi_z) (psi: CPML memory of the velocity updates, phi: of the pressure update):
// A = P o V with
//   V:  psi_x' = b'x psi_x + a'x Dx+ p,  vx' = vx + dt/rho_x (Dx+ p + psi_x')   on Gx
//       (z analogue on Gz; psi only where a' != 0)
//   P:  phi_x' = bx phi_x + ax Dx- vx,   p' = p + dt kappa (Dx- vx + phi_x' + Dz- vz + phi_z')
//       on Gp (phi only where a != 0),  kappa = rho vp^2.
// Born modelling adds dt dkappa S0^n to p after step n (S0 = the background's p-update
// sum) and records p at the receivers after each step: u^{n+1} = A u^n + B_n dkappa,
// d^n = R u^{n+1}.  Its adjoint is
//   lambda^k = A^T lambda^{k+1} + R^T d*^k,   grad_kappa += dt S0^k lambda_p^k,
// with A^T = V^T P^T.  Per adjoint step two launches, each "gather, then pointwise":
//   k_adj_v: v^ += Dx-^T Qx, Dz-^T Qz   (P^T gather)
//            rx = Gx dt/rho_x v^x;  Rx = rx + a'x (rx + psi^x);  psi^x = b'x (rx + psi^x)
//   k_adj_p: p^ += Dx+^T Rx + Dz+^T Rz  (V^T gather);  p^ += residual at the receivers;
//            grad += dt S0^k p^;
//            q = Gp dt kappa p^;  Qx = q + ax (q + phi^x);  phi^x = bx (q + phi^x)
//            (P^T pointwise for the next, earlier step)
// The transposed stencils are gathers over the neighbours that lie inside the source
// mask, so every read is in bounds and no atomics are needed.  Q and R live in scratch
// arrays: each kernel reads only the other's scratch at neighbour cells and writes its
// own cells.
#pragma once
#include "prop.cuh"

namespace swd {

struct AdjArgs {
    Geo g;
    Cpml c;
    const float *vp, *rho;
    const float *ck;     // dt*rho*vp*vp (the forward pressure coefficient)
    Wave l;              // adjoint state: p^, v^x, v^z, psi^x (ppx), psi^z (ppz), phi^x (pvx), phi^z (pvz)
    float *qx, *qz, *rx, *rz;
    const int *itp;      // step index k = *itp + itoff (counts down)
    int itoff;
    int nt;
    Wells wells;
    const float *resid;  // [r_n][nt] adjoint source, summed over traces that share a cell
    const float *s0;     // background p-update sums, slot k % s0_mod
    long long s0_stride;
    int s0_mod;
    double *grad;        // d J / d kappa, FP64 accumulation
};

__device__ __forceinline__ bool in_range(int v, int lo, int hi) { return v >= lo && v <= hi; }

template <int LC>
__global__ void __launch_bounds__(256) k_adj_v(AdjArgs a)
{
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    if (x >= g.ntx || z0 >= g.ntz) return;
    const int ntx = g.ntx, ntz = g.ntz, ldz = g.ldz;
    const size_t ip = (size_t)x * ldz + z0;
    // ---- P^T gathers: v^x += Dx-^T Qx (Qx non-zero on the Gp columns [LC, ntx-LC])
    float4 vx = ld4(a.l.vx + ip), vz = ld4(a.l.vz + ip);
#pragma unroll
    for (int ic = 0; ic < LC; ic++) {
        const int xa = x - ic, xb = x + ic + 1;
        const float4 qa = in_range(xa, LC, ntx - LC) ? ld4(a.qx + (size_t)xa * ldz + z0) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 qb = in_range(xb, LC, ntx - LC) ? ld4(a.qx + (size_t)xb * ldz + z0) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 4; k++) el(vx, k) += g.rc[ic] * (elc(qa, k) - elc(qb, k)) * g.odx;
    }
    // v^z += Dz-^T Qz (Qz non-zero on rows [LC, ntz-LC] of the Gp columns)
    if (in_range(x, LC, ntx - LC)) {
        ZWin<LC> qw;
        qw.load(a.qz + (size_t)x * ldz, z0);
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int ic = 0; ic < LC; ic++) {
                const int za = z0 + k - ic, zb = z0 + k + ic + 1;
                const float qa = in_range(za, LC, ntz - LC) ? qw.at(k - ic) : 0.f;
                const float qb = in_range(zb, LC, ntz - LC) ? qw.at(k + ic + 1) : 0.f;
                el(vz, k) += g.rc[ic] * (qa - qb) * g.odz;
            }
    }
    st4(a.l.vx + ip, vx);
    st4(a.l.vz + ip, vz);
    // ---- V^T pointwise: x part on Gx = cols [LC-1, ntx-LC-1] x rows [LC, ntz-LC]
    float4 Rx = make_float4(0.f, 0.f, 0.f, 0.f), Rz = make_float4(0.f, 0.f, 0.f, 0.f);
    if (in_range(x, LC - 1, ntx - LC - 1)) {
        const float4 r0 = ldg4(a.rho + ip), r1 = ldg4(a.rho + ip + ldz);
        const float ax = __ldg(a.c.axh + x);
        float4 ps = ax != 0.f ? ld4(a.l.ppx + ip) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float bx = ax != 0.f ? __ldg(a.c.bxh + x) : 0.f;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!in_range(z0 + k, LC, ntz - LC)) continue;
            const float orho = __frcp_rn(0.5f * (elc(r0, k) + elc(r1, k)));
            const float r = g.dt * orho * elc(vx, k);
            if (ax != 0.f) {
                el(Rx, k) = r + ax * (r + elc(ps, k));
                el(ps, k) = bx * (r + elc(ps, k));
            } else {
                el(Rx, k) = r;
            }
        }
        if (ax != 0.f) st4(a.l.ppx + ip, ps);
    }
    // z part on Gz = cols [LC, ntx-LC] x rows [LC-1, ntz-LC-1]
    if (in_range(x, LC, ntx - LC)) {
        const float4 r0 = ldg4(a.rho + ip);
        const float r4 = __ldg(a.rho + ip + 4);
        const float4 az = ldg4(a.c.azh + z0);
        const bool pml = az.x != 0.f || az.y != 0.f || az.z != 0.f || az.w != 0.f;
        float4 ps = pml ? ld4(a.l.ppz + ip) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 bz = pml ? ldg4(a.c.bzh + z0) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!in_range(z0 + k, LC - 1, ntz - LC - 1)) continue;
            const float rn = k < 3 ? elc(r0, k + 1) : r4;
            const float orho = __frcp_rn(0.5f * (elc(r0, k) + rn));
            const float r = g.dt * orho * elc(vz, k);
            if (elc(az, k) != 0.f) {
                el(Rz, k) = r + elc(az, k) * (r + elc(ps, k));
                el(ps, k) = elc(bz, k) * (r + elc(ps, k));
            } else {
                el(Rz, k) = r;
            }
        }
        if (pml) st4(a.l.ppz + ip, ps);
    }
    st4(a.rx + ip, Rx);
    st4(a.rz + ip, Rz);
}

template <int LC>
__global__ void __launch_bounds__(256) k_adj_p(AdjArgs a)
{
    const int it = *a.itp + a.itoff;
    int x, z0;
    cell4(x, z0);
    const Geo &g = a.g;
    if (x >= g.ntx || z0 >= g.ntz) return;
    const int ntx = g.ntx, ntz = g.ntz, ldz = g.ldz;
    const size_t ip = (size_t)x * ldz + z0;
    float4 p = ld4(a.l.p + ip);
    // ---- V^T gathers: p^ += Dx+^T Rx (Rx on Gx columns [LC-1, ntx-LC-1]) + Dz+^T Rz
#pragma unroll
    for (int ic = 0; ic < LC; ic++) {
        const int xa = x - ic - 1, xb = x + ic;
        const float4 ra = in_range(xa, LC - 1, ntx - LC - 1) ? ld4(a.rx + (size_t)xa * ldz + z0) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 rb = in_range(xb, LC - 1, ntx - LC - 1) ? ld4(a.rx + (size_t)xb * ldz + z0) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 4; k++) el(p, k) += g.rc[ic] * (elc(ra, k) - elc(rb, k)) * g.odx;
    }
    if (in_range(x, LC, ntx - LC)) {
        ZWin<LC> rw;
        rw.load(a.rz + (size_t)x * ldz, z0);
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int ic = 0; ic < LC; ic++) {
                const int za = z0 + k - ic - 1, zb = z0 + k + ic;
                const float ra = in_range(za, LC - 1, ntz - LC - 1) ? rw.at(k - ic - 1) : 0.f;
                const float rb = in_range(zb, LC - 1, ntz - LC - 1) ? rw.at(k + ic) : 0.f;
                el(p, k) += g.rc[ic] * (ra - rb) * g.odz;
            }
    }
    // ---- adjoint source at the receivers (R^T)
    const int wc = __ldg(a.wells.wcol + x);
    if (wc >= 0) {
        const int4 tr = __ldg(reinterpret_cast<const int4 *>(a.wells.wmap + (size_t)wc * ldz + z0));
        const int t[4] = {tr.x, tr.y, tr.z, tr.w};
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (t[k] >= 0 && z0 + k < ntz) el(p, k) += __ldg(a.resid + (size_t)t[k] * a.nt + it);
    }
    st4(a.l.p + ip, p);
    // ---- imaging: grad += dt * S0^k * p^ (S0 is zero off Gp)
    const bool colp = in_range(x, LC, ntx - LC);
    if (colp) {
        const float4 s = ldg4(a.s0 + (size_t)(it % a.s0_mod) * a.s0_stride + ip);
        double2 *gp = reinterpret_cast<double2 *>(a.grad + ip);
        double2 g0 = gp[0], g1 = gp[1];
        g0.x += (double)g.dt * (double)s.x * (double)p.x;
        g0.y += (double)g.dt * (double)s.y * (double)p.y;
        g1.x += (double)g.dt * (double)s.z * (double)p.z;
        g1.y += (double)g.dt * (double)s.w * (double)p.w;
        gp[0] = g0;
        gp[1] = g1;
    }
    // ---- P^T pointwise for the next (earlier) step, on Gp = cols/rows [LC, n-LC]
    float4 Qx = make_float4(0.f, 0.f, 0.f, 0.f), Qz = make_float4(0.f, 0.f, 0.f, 0.f);
    if (colp) {
        // dt*rho*vp*vp*p^ = ck*p^ exactly (the same products in the same order)
        const float4 kc = ldg4(a.ck + ip);
        const float ax = __ldg(a.c.ax + x);
        const float bx = ax != 0.f ? __ldg(a.c.bx + x) : 0.f;
        float4 fx = ax != 0.f ? ld4(a.l.pvx + ip) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 az = ldg4(a.c.az + z0);
        const bool pmlz = az.x != 0.f || az.y != 0.f || az.z != 0.f || az.w != 0.f;
        const float4 bz = pmlz ? ldg4(a.c.bz + z0) : make_float4(0.f, 0.f, 0.f, 0.f);
        float4 fz = pmlz ? ld4(a.l.pvz + ip) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!in_range(z0 + k, LC, ntz - LC)) continue;
            const float q = elc(kc, k) * elc(p, k);
            if (ax != 0.f) {
                el(Qx, k) = q + ax * (q + elc(fx, k));
                el(fx, k) = bx * (q + elc(fx, k));
            } else {
                el(Qx, k) = q;
            }
            if (elc(az, k) != 0.f) {
                el(Qz, k) = q + elc(az, k) * (q + elc(fz, k));
                el(fz, k) = elc(bz, k) * (q + elc(fz, k));
            } else {
                el(Qz, k) = q;
            }
        }
        if (ax != 0.f) st4(a.l.pvx + ip, fx);
        if (pmlz) st4(a.l.pvz + ip, fz);
    }
    st4(a.qx + ip, Qx);
    st4(a.qz + ip, Qz);
}

// Restore snapshot `snap` of a checkpoint store into the wavefield w; launched on the grid
// of the saving kernel so the scale slots line up.
__global__ void __launch_bounds__(256) k_ckpt_restore(Ckpt ck, Wave w, int snap, int ntx, int ntz, int ldz)
{
    int x, z0;
    cell4(x, z0);
    if (x >= ntx || z0 >= ntz) return;
    const size_t ip = (size_t)x * ldz + z0;
    const int slot = blockIdx.y * gridDim.x + blockIdx.x;
#pragma unroll 1
    for (int i = 0; i < 7; i++) {
        const size_t o = ((size_t)snap * 7 + i) * ck.fstride + ip;
        float4 v;
        if (ck.prec == 0) {
            v = ld4((const float *)ck.buf + o);
        } else {
            const float mx = ck.scale[((size_t)snap * 7 + i) * ck.nblocks + slot];
            const ushort4 h = *reinterpret_cast<const ushort4 *>((const unsigned short *)ck.buf + o);
            v = make_float4(dec16(h.x, mx, ck.prec), dec16(h.y, mx, ck.prec), dec16(h.z, mx, ck.prec),
                            dec16(h.w, mx, ck.prec));
        }
        st4(wave_array(w, i) + ip, v);
    }
}

// adjoint source: out = in, then the traces that alias another trace's cell are added
// into that trace (alias list of (dst, src) pairs: dst records the same cell as src)
__global__ void k_sum_aliases(float *out, const int2 *alias, int nalias, int nt)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nt; j += gridDim.x * blockDim.x)
        for (int a = 0; a < nalias; a++) out[(size_t)alias[a].y * nt + j] += out[(size_t)alias[a].x * nt + j];
}

}  // namespace swd
