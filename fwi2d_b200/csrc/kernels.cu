// Fused per-time-step propagation kernels for sm_100a.
//
// One launch advances every shot of a batch by one time step.  Each CTA owns
// a TZ x TX tile of one shot grid and performs, for every cell of the tile,
// the whole step of the reference time loop (src/cpp/we_op.cpp:667-871 for the
// elastic propagator, :1640-1840 for VTI):
//   second-derivative and mixed-derivative SBP terms, source injection, the
//   SAT free-surface / absorbing closures, the leapfrog update, the implicit
//   absorbing-boundary scaling and the cos^2 taper of curr and next,
// plus receiver extraction, snapshot storage (forward) or the zero-lag imaging
// condition (adjoint), so each field sample is read from HBM/L2 once per step.
//
// Tiling.  Tile k of an axis of length n covers the window
// [min(kT, n-T), +T) and owns the cells up to the next window: the last
// window is flush with the far boundary, so every SBP boundary band (6 cells)
// and the halo its closures read lie inside one window.
//
// Memory per step: curr is read with a 4-cell halo into shared memory; prev
// is read and overwritten in place by next (it is only ever read at its own
// cell).  The second application of the taper that the reference makes to
// curr at the end of each step is applied when that buffer is read back as
// prev one step later.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdio>
#include "engine.h"
#include "sbp.cuh"

namespace fwi2d {

enum StepFlags { F_STORE = 1, F_EXTRACT = 2, F_AMAX = 4, F_GRAD = 8 };

// ---------------------------------------------------------------------------
// Snapshot storage: fp32, or bf16/fp16 scaled by a per-snapshot power of two
// chosen from the snapshot's max |u| (so |u*scale| < 2^14).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float snap_scale(const unsigned *amax, int slot)
{
    float m = __uint_as_float(amax[slot]);
    if (!(m > 0.f)) return 1.f;
    int e = ilogbf(m) + 1;                 // m < 2^e
    return ldexpf(1.f, 14 - e);
}

__device__ __forceinline__ void snap_store(void *base, long long idx, int prec, float v, float scale)
{
    if (prec == SNAP_FP32) ((float *)base)[idx] = v;
    else if (prec == SNAP_BF16) ((__nv_bfloat16 *)base)[idx] = __float2bfloat16_rn(v * scale);
    else ((__half *)base)[idx] = __float2half_rn(v * scale);
}

__device__ __forceinline__ float snap_load(const void *base, long long idx, int prec, float inv)
{
    if (prec == SNAP_FP32) return ((const float *)base)[idx];
    if (prec == SNAP_BF16) return __bfloat162float(((const __nv_bfloat16 *)base)[idx]) * inv;
    return __half2float(((const __half *)base)[idx]) * inv;
}

__device__ __forceinline__ void tile_window(int k, int ntile, int n, int T, int &w0, int &own_hi)
{
    w0 = min(k * T, n - T);
    own_hi = (k == ntile - 1) ? n : min((k + 1) * T, n - T);
}

// ---------------------------------------------------------------------------
// Elastic isotropic / VTI step.
// ---------------------------------------------------------------------------
template <bool VTI, int TZ, int TX, bool GRAD>
__global__ void __launch_bounds__(TZ *TX)
elastic_step(const ShotDev *__restrict__ shots, const TileRef *__restrict__ tiles, ModelDev M, StepConst C,
             int it, int flags, float dtg)
{
    constexpr int UZ = TZ + 8, UX = TX + 8;
    constexpr int WZ = TZ + 4, WX = TX + 4;
    constexpr int NT = TZ * TX;
    __shared__ float U0[UX * UZ], U1[UX * UZ];
    __shared__ float MU[WX * WZ], Q[WX * WZ];          // mu; lambda (iso) or (1+2eps)2mu (VTI)
    __shared__ float T0[WX * WZ], T1[WX * WZ];         // iso: ux_x+uz_z ; VTI: tmp_x, tmp_z
    __shared__ float BX[WX * WZ], CZ[WX * WZ];         // uz_x, ux_z
    __shared__ float F0[GRAD ? WX * WZ : 1], F1[GRAD ? WX * WZ : 1];
    __shared__ float red[NT / 32];

    const TileRef tr = tiles[blockIdx.x];
    const ShotDev &S = shots[tr.shot];
    const int nt = S.nt;
    if (it >= nt - 1) return;
    const int nx = S.nx, nz = S.nz, ldz = S.ldz;
    const long long nxz = (long long)nx * ldz;
    int wx0, ownx, wz0, ownz;
    tile_window(tr.tx, S.tiles_x, nx, TX, wx0, ownx);
    tile_window(tr.tz, S.tiles_z, nz, TZ, wz0, ownz);

    const float *curr = S.u[(it + 1) & 1];
    float *pn = S.u[it & 1];                 // prev in, next out
    const long long mofs = (long long)S.x0 * M.ldz;

    // ---- phase 1: curr with a 4-cell halo, coefficients with a 2-cell halo
    for (int i = threadIdx.x; i < UX * UZ; i += NT) {
        const int sx = i / UZ, sz = i - sx * UZ;
        const int gx = wx0 - 4 + sx, gz = wz0 - 4 + sz;
        float a = 0.f, b = 0.f;
        if (gx >= 0 && gx < nx && gz >= 0 && gz < nz) {
            const long long o = (long long)gx * ldz + gz;
            a = curr[o];
            b = curr[nxz + o];
        }
        U0[i] = a;
        U1[i] = b;
    }
    const int itf = GRAD ? (nt - 1 - (it + 1)) / C.sub : 0;
    const bool do_grad = GRAD && (flags & F_GRAD) && ((nt - 1 - (it + 1)) % C.sub == 0);
    float finv = 1.f;
    if (GRAD && do_grad && C.snap_prec != SNAP_FP32) finv = 1.f / snap_scale(S.snap_amax, itf);
    for (int i = threadIdx.x; i < WX * WZ; i += NT) {
        const int sx = i / WZ, sz = i - sx * WZ;
        const int gx = wx0 - 2 + sx, gz = wz0 - 2 + sz;
        float m = 0.f, q = 0.f;
        if (gx >= 0 && gx < nx && gz >= 0 && gz < nz) {
            const long long o = mofs + (long long)gx * M.ldz + gz;
            m = M.p1[o];
            q = VTI ? M.fxx[o] : M.p0[o];
        }
        MU[i] = m;
        Q[i] = q;
        if (GRAD) {
            float f0 = 0.f, f1 = 0.f;
            if (do_grad && gx >= 0 && gx < nx && gz >= 0 && gz < nz) {
                const long long o = (long long)itf * S.snap_slot + (long long)gx * ldz + gz;
                f0 = snap_load(S.snap, o, C.snap_prec, finv);
                f1 = snap_load(S.snap, o + nxz, C.snap_prec, finv);
            }
            F0[i] = f0;
            F1[i] = f1;
        }
    }
    __syncthreads();

    // ---- phase 2: first derivatives of curr on the tile plus a 2-cell halo
    for (int i = threadIdx.x; i < WX * WZ; i += NT) {
        const int sx = i / WZ, sz = i - sx * WZ;
        const int gx = wx0 - 2 + sx, gz = wz0 - 2 + sz;
        float t0 = 0.f, t1 = 0.f, bx = 0.f, cz = 0.f;
        // a closure reads up to 5 samples from its boundary: evaluate only
        // where the loaded window holds them (other points are never used)
        const bool okx = (gx >= 4 && gx < nx - 4) || (gx < 4 ? wx0 <= 4 : wx0 + TX + 4 >= nx);
        const bool okz = (gz >= 4 && gz < nz - 4) || (gz < 4 ? wz0 <= 4 : wz0 + TZ + 4 >= nz);
        if (gx >= 0 && gx < nx && gz >= 0 && gz < nz && okx && okz) {
            const int ui = (sx + 2) * UZ + (sz + 2);
            const float ux_x = d1(U0 + ui, UZ, gx, nx, C.dx, C.sdx);
            const float uz_z = d1(U1 + ui, 1, gz, nz, C.dz, C.sdz);
            bx = d1(U1 + ui, UZ, gx, nx, C.dx, C.sdx);
            cz = d1(U0 + ui, 1, gz, nz, C.dz, C.sdz);
            if (!VTI) {
                t0 = ux_x + uz_z;
            } else {
                const long long o = mofs + (long long)gx * M.ldz + gz;
                const float lb = M.lbis[o], c13 = M.c13[o], lam = M.p0[o];
                t0 = lb * ux_x + c13 * uz_z;
                t1 = lam * uz_z + c13 * ux_x;
            }
        }
        T0[i] = t0;
        T1[i] = t1;
        BX[i] = bx;
        CZ[i] = cz;
    }
    __syncthreads();

    // ---- phase 3: the cell of this thread
    const int tz = threadIdx.x % TZ, tx = threadIdx.x / TZ;
    const int gx = wx0 + tx, gz = wz0 + tz;
    const bool owned = (gx < ownx) && (gz < ownz);
    const int ui = (tx + 4) * UZ + (tz + 4);
    const int wi = (tx + 2) * WZ + (tz + 2);
    const long long cell = (long long)gx * ldz + gz;
    const long long mcell = mofs + (long long)gx * M.ldz + gz;

    // snapshot of curr (forward), before anything else as the reference does
    if ((flags & F_STORE) && (it % C.sub == 0) && owned) {
        const int slot = it / C.sub;
        const float sc = C.snap_prec == SNAP_FP32 ? 1.f : snap_scale(S.snap_amax, slot);
        const long long o = (long long)slot * S.snap_slot + cell;
        snap_store(S.snap, o, C.snap_prec, U0[ui], sc);
        snap_store(S.snap, o + nxz, C.snap_prec, U1[ui], sc);
    }

    // receivers (forward): one thread per receiver of this tile
    if (flags & F_EXTRACT) {
        const int tile_id = tr.tz * S.tiles_x + tr.tx;
        const int e0 = S.ext_off[tile_id], e1 = S.ext_off[tile_id + 1];
        for (int e = e0 + threadIdx.x; e < e1; e += NT) {
            const ExtEntry E = S.ext[e];
            const float *U = E.comp == 0 ? U0 : U1;
            float o = 0.f;
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++)
                    o += E.w[a * 3 + b] * U[(E.gx0 + a - wx0 + 4) * UZ + (E.gz0 + b - wz0 + 4)];
            S.rcv[(long long)it * S.nrcv + E.row] = o;
        }
    }

    float n0 = 0.f, n1 = 0.f;
    if (owned) {
        // interior operators, in the reference's order of accumulation
        const float mu = MU[wi];
        if (!VTI) {
            d2acc(n0, U0 + ui, UZ, MU + wi, WZ, 2.f, gx, nx, C.inv_d2x, C.d2x);   // Dxx_var<2mu>(ux)
            d2acc(n1, U1 + ui, 1, MU + wi, 1, 2.f, gz, nz, C.inv_d2z, C.d2z);     // Dzz_var<2mu>(uz)
        } else {
            d2acc(n0, U0 + ui, UZ, Q + wi, WZ, 1.f, gx, nx, C.inv_d2x, C.d2x);    // Dxx_var<(1+2eps)2mu>(ux)
            d2acc(n1, U1 + ui, 1, MU + wi, 1, 2.f, gz, nz, C.inv_d2z, C.d2z);     // Dzz_var<2mu>(uz)
        }
        d2acc(n1, U1 + ui, UZ, MU + wi, WZ, 1.f, gx, nx, C.inv_d2x, C.d2x);       // Dxx_var<mu>(uz)
        d2acc(n0, U0 + ui, 1, MU + wi, 1, 1.f, gz, nz, C.inv_d2z, C.d2z);         // Dzz_var<mu>(ux)
        if (!VTI) {
            n0 += md1(T0 + wi, Q + wi, WZ, gx, nx, C.adx);                        // mult_Dx(lambda, tmp)
            n1 += md1(T0 + wi, Q + wi, 1, gz, nz, C.adz);                         // mult_Dz(lambda, tmp)
        } else {
            n0 += d1(T0 + wi, WZ, gx, nx, C.dx, C.sdx);                           // Dx(tmp_x)
            n1 += d1(T1 + wi, 1, gz, nz, C.dz, C.sdz);                            // Dz(tmp_z)
        }
        n1 += md1(CZ + wi, MU + wi, WZ, gx, nx, C.adx);                           // mult_Dx(mu, ux_z)
        n0 += md1(BX + wi, MU + wi, 1, gz, nz, C.adz);                            // mult_Dz(mu, uz_x)

        // sources
        {
            const int tile_id = tr.tz * S.tiles_x + tr.tx;
            const int e0 = S.inj_off[tile_id], e1 = S.inj_off[tile_id + 1];
            const float *src = S.src + (long long)it * S.nsrc;
            for (int e = e0; e < e1; e++) {
                const InjEntry E = S.inj[e];
                if (E.gx == gx && E.gz == gz) {
                    const float c = E.mt ? (E.wa * src[E.ia] - E.wb * src[E.ib]) : E.wa * src[E.ia];
                    if (E.comp == 0) n0 += c;
                    else n1 += c;
                }
            }
        }

        // previous field, with the taper it received at the end of the last step
        const float tzv = S.tz[gz], txv = S.tx[gx];
        float p0 = pn[cell], p1 = pn[nxz + cell];
        if (it > 0) {
            p0 = p0 * tzv * txv;
            p1 = p1 * tzv * txv;
        }

        // SAT closures (spatial_operators.hpp:160-822), in the reference's side order
        const bool edge = gz == 0 || gz == nz - 1 || gx == 0 || gx == nx - 1;
        if (edge) {
            const float lam = VTI ? M.p0[mcell] : Q[wi];
            const float rho = M.p2[mcell];
            const float c13 = VTI ? M.c13[mcell] : lam;
            const float fxx = VTI ? Q[wi] : 2 * mu;
            const float lamx = VTI ? M.lbis[mcell] : lam;
            const float eps = VTI ? M.eps[mcell] : 0.f;
            const float imp_s = 0.5f * sqrtf(mu * rho);
            const float imp_p = 0.5f * sqrtf((lam + 2 * mu) * rho);
            const float imp_px = VTI ? 0.5f * sqrtf((1 + 2 * eps) * (lam + 2 * mu) * rho) : imp_p;
            for (int side = 0; side < 4; side++) {
                const int bc = C.bc[side];
                if (bc != 1 && bc != 2) continue;
                const bool ab = bc == 2;
                if (side < 2) {
                    if (gz != (side == 0 ? 0 : nz - 1)) continue;
                    const int in = side == 0 ? 1 : -1;
                    const float sg = side == 0 ? -1.f : 1.f;
                    // next0: f1 = f2 = mu, in1 = uz (along x), in2 = ux (outward)
                    {
                        float t = (sg * mu) * tsum(U1 + ui, UZ, gx, nx) / C.dx + mu * nsum(U0 + ui, in) / C.dz;
                        if (ab) t = t - imp_s * p0 / C.dt;
                        n0 = n0 - C.sat_z * t;
                    }
                    // next1: f1 = lambda (c13), f2 = 2mu, in1 = ux, in2 = uz ; then -H^-1(lambda Dz uz)_0
                    {
                        float t = (sg * c13) * tsum(U0 + ui, UZ, gx, nx) / C.dx + (2 * mu) * nsum(U1 + ui, in) / C.dz;
                        if (ab) t = t - imp_p * p1 / C.dt;
                        n1 = n1 - C.sat_z * t;
                        n1 = n1 - C.nsat_z * lam * ndsum(U1 + ui, in);
                    }
                } else {
                    if (gx != (side == 2 ? 0 : nx - 1)) continue;
                    const int in = side == 2 ? UZ : -UZ;
                    const float sg = side == 2 ? -1.f : 1.f;
                    // next0: f1 = lambda (c13), f2 = 2mu ((1+2eps)2mu), in1 = uz (along z), in2 = ux
                    {
                        float t = (sg * c13) * tsum(U1 + ui, 1, gz, nz) / C.dz + fxx * nsum(U0 + ui, in) / C.dx;
                        if (ab) t = t - imp_px * p0 / C.dt;
                        n0 = n0 - C.sat_x * t;
                        n0 = n0 - C.nsat_x * lamx * ndsum(U0 + ui, in);
                    }
                    // next1: f1 = f2 = mu, in1 = ux, in2 = uz
                    {
                        float t = (sg * mu) * tsum(U0 + ui, 1, gz, nz) / C.dz + mu * nsum(U1 + ui, in) / C.dx;
                        if (ab) t = t - imp_s * p1 / C.dt;
                        n1 = n1 - C.sat_x * t;
                    }
                }
            }
        }

        // leapfrog (we_op.cpp:825-830)
        const float rho = M.p2[mcell];
        n0 = C.dt2 * n0 / rho + 2 * U0[ui] - p0;
        n1 = C.dt2 * n1 / rho + 2 * U1[ui] - p1;

        // implicit absorbing scaling (esat_scale_boundaries)
        if (edge) {
            const int per = 2 * nx + 2 * nz;
            int k = -1;
            if (gz == 0) k = gx;
            else if (gz == nz - 1) k = nx + gx;
            else if (gx == 0) k = 2 * nx + gz;
            else if (gx == nx - 1) k = 2 * nx + nz + gz;
            n0 = n0 / S.den[k];
            n1 = n1 / S.den[per + k];
        }

        // taper of next
        n0 = n0 * tzv * txv;
        n1 = n1 * tzv * txv;

        pn[cell] = n0;
        pn[nxz + cell] = n1;

        // imaging condition for the next adjoint sample (we_op.cpp:505-562)
        if (GRAD && do_grad) {
            const float ax0 = d1(U0 + ui, UZ, gx, nx, C.dx, C.sdx);
            const float az1 = d1(U1 + ui, 1, gz, nz, C.dz, C.sdz);
            const float az0 = CZ[wi], ax1 = BX[wi];
            const float t0 = d1(F0 + wi, WZ, gx, nx, C.dx, C.sdx);
            const float t1 = d1(F1 + wi, 1, gz, nz, C.dz, C.sdz);
            const float t2 = d1(F1 + wi, WZ, gx, nx, C.dx, C.sdx);
            const float t3 = d1(F0 + wi, 1, gz, nz, C.dz, C.sdz);
            const int last = nt / C.sub;
            const float f0 = F0[wi], f1 = F1[wi];
            float fp0 = 0.f, fp1 = 0.f, fm0 = 0.f, fm1 = 0.f;
            if (itf + 1 <= last) {
                const float inv = C.snap_prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(S.snap_amax, itf + 1);
                const long long o = (long long)(itf + 1) * S.snap_slot + cell;
                fp0 = snap_load(S.snap, o, C.snap_prec, inv);
                fp1 = snap_load(S.snap, o + nxz, C.snap_prec, inv);
            }
            if (itf > 0) {
                const float inv = C.snap_prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(S.snap_amax, itf - 1);
                const long long o = (long long)(itf - 1) * S.snap_slot + cell;
                fm0 = snap_load(S.snap, o, C.snap_prec, inv);
                fm1 = snap_load(S.snap, o + nxz, C.snap_prec, inv);
            }
            float dl, dm;
            if (!VTI) {
                dl = 0.f;
                dm = (az0 + ax1) * (t2 + t3) + 2 * ax0 * t0 + 2 * az1 * t1;
            } else {
                const float e2 = 1 + 2 * M.eps[mcell];
                const float v2 = M.gv2[mcell], v3 = M.gv3[mcell];
                dl = e2 * ax0 * t0 + az1 * t1 + v2 * (ax0 * t1 + az1 * t0);
                dm = (az0 + ax1) * (t2 + t3) + 2 * e2 * ax0 * t0 + 2 * az1 * t1 + v3 * (ax0 * t1 + az1 * t0);
            }
            float *g0 = S.grad + cell, *g1 = g0 + nxz, *g2 = g1 + nxz;
            const float gw = S.gwt[itf];
            const double wdt = (double)gw * 1.0 / (double)dtg;
            if (itf > 0 && itf < last) {
                if (!VTI) *g0 = *g0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                else *g0 = *g0 + gw * dtg * dl;
                *g1 = *g1 + gw * dtg * dm;
                *g2 = (float)((double)*g2 + wdt * (double)(n0 * (fp0 - 2 * f0 + fm0) + n1 * (fp1 - 2 * f1 + fm1)));
            } else if (itf == 0) {
                const double wh = (double)gw * 0.5 * (double)dtg;
                if (!VTI) *g0 = (float)((double)*g0 + wh * (double)(ax0 + az1) * (double)(t0 + t1));
                else *g0 = (float)((double)*g0 + wh * (double)dl);
                *g1 = (float)((double)*g1 + wh * (double)dm);
                *g2 = (float)((double)*g2 + wdt * (double)(n0 * (fp0 - f0) + n1 * (fp1 - f1)));
            } else {
                if (!VTI) *g0 = *g0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                else *g0 = *g0 + gw * dtg * dl;
                *g1 = *g1 + gw * dtg * dm;
                *g2 = (float)((double)*g2 + wdt * (double)(n0 * (-f0 + fm0) + n1 * (-f1 + fm1)));
            }
        }
    }

    // max |next| for the scale of the next 16-bit snapshot
    if ((flags & F_AMAX) && ((it + 1) % C.sub == 0)) {
        float m = owned ? fmaxf(fabsf(n0), fabsf(n1)) : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32) {
            m = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (threadIdx.x == 0 && m > 0.f) atomicMax(S.snap_amax + (it + 1) / C.sub, __float_as_uint(m));
        }
    }
}

// ---------------------------------------------------------------------------
// Initial state: zero both buffers' touched cells is done by memset; this
// scatters the precomputed first "prev" samples (we_op.cpp:657-663).
// ---------------------------------------------------------------------------
__global__ void scatter_init(const ShotDev *__restrict__ shots, int nshots, const InitEntry *__restrict__ ent,
                             const int *__restrict__ off)
{
    const int s = blockIdx.x;
    if (s >= nshots) return;
    const ShotDev &S = shots[s];
    const long long nxz = (long long)S.nx * S.ldz;
    for (int e = off[s] + threadIdx.x; e < off[s + 1]; e += blockDim.x) {
        const InitEntry E = ent[e];
        S.u[0][E.comp * nxz + (long long)E.gx * S.ldz + E.gz] = E.val;
    }
}

// ---------------------------------------------------------------------------
// Last sample: receivers and the final snapshot (we_op.cpp:874-881).
// One CTA per shot.
// ---------------------------------------------------------------------------
__global__ void finalize_shots(const ShotDev *__restrict__ shots, int nshots, StepConst C, int ncomp, int flags)
{
    const int s = blockIdx.y;
    if (s >= nshots) return;
    const ShotDev &S = shots[s];
    const int it = S.nt - 1;
    const float *curr = S.u[(it + 1) & 1];
    const long long nxz = (long long)S.nx * S.ldz;
    if (flags & F_EXTRACT) {
        const int tiles = S.tiles_x * S.tiles_z;
        const int e1 = S.ext_off[tiles];
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < e1; e += gridDim.x * blockDim.x) {
            const ExtEntry E = S.ext[e];
            const float *U = curr + E.comp * nxz;
            float o = 0.f;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) o += E.w[a * 3 + b] * U[(long long)(E.gx0 + a) * S.ldz + E.gz0 + b];
            S.rcv[(long long)it * S.nrcv + E.row] = o;
        }
    }
    if ((flags & F_STORE) && (it % C.sub == 0)) {
        const int slot = it / C.sub;
        const float sc = C.snap_prec == SNAP_FP32 ? 1.f : snap_scale(S.snap_amax, slot);
        const long long n = (long long)ncomp * nxz;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
            const long long rem = i % S.ldz;
            if (rem < S.nz) snap_store(S.snap, (long long)slot * S.snap_slot + i, C.snap_prec, curr[i], sc);
        }
    }
}

// ---------------------------------------------------------------------------
// VTI gradient coefficients dC13/dlambda, dC13/dmu (we_op.cpp:1499-1504),
// evaluated once per model in the reference's float order.
// ---------------------------------------------------------------------------
__global__ void vti_grad_coefs(int n, const float *lam, const float *mu, const float *c13, float *v2, float *v3)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float l = lam[i], m = mu[i], c = c13[i];
        const float d = ((c + m) * (c + m) - (l + m) * (l + m)) / (2 * (l + m) * (l + 2 * m));
        const float val1 = sqrtf(2 * (l + 2 * m) * (l + m) * d + (l + m) * (l + m));
        v2[i] = ((1 + 2 * d) * l + (1 + 3 * d) * m) / val1;
        v3[i] = ((1 + 3 * d) * l + (1 + 4 * d) * m) / val1 - 1;
    }
}

// ---------------------------------------------------------------------------
// Host-side launch helpers
// ---------------------------------------------------------------------------
void upload_sbp_tables(const float *b1, const float *b2, const float *c2, const float *c1, const float *sc, const float *hc)
{
    cudaMemcpyToSymbol(kB1, b1, sizeof(float) * 24);
    cudaMemcpyToSymbol(kB2, b2, sizeof(float) * 384);
    cudaMemcpyToSymbol(kC2, c2, sizeof(float) * 10);
    cudaMemcpyToSymbol(kC1, c1, sizeof(float) * 2);
    cudaMemcpyToSymbol(kSC, sc, sizeof(float) * 4);
    cudaMemcpyToSymbol(kHC, hc, sizeof(float) * 4);
}

template <bool VTI, int TZ, int TX>
static void launch_elastic_t(const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M, const StepConst &C,
                             int it, int flags, float dtg, cudaStream_t st)
{
    if (flags & F_GRAD)
        elastic_step<VTI, TZ, TX, true><<<ntiles, TZ * TX, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
    else
        elastic_step<VTI, TZ, TX, false><<<ntiles, TZ * TX, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
}

// tile shapes offered to the autotuner: (TZ, TX)
int elastic_tile_count() { return 3; }
void elastic_tile_shape(int i, int *tz, int *tx)
{
    static const int s[3][2] = {{32, 16}, {32, 8}, {64, 8}};
    *tz = s[i][0];
    *tx = s[i][1];
}

void launch_elastic_step(int shape, bool vti, const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                         const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    switch (shape) {
    case 0: vti ? launch_elastic_t<true, 32, 16>(shots, tiles, ntiles, M, C, it, flags, dtg, st)
                : launch_elastic_t<false, 32, 16>(shots, tiles, ntiles, M, C, it, flags, dtg, st); break;
    case 1: vti ? launch_elastic_t<true, 32, 8>(shots, tiles, ntiles, M, C, it, flags, dtg, st)
                : launch_elastic_t<false, 32, 8>(shots, tiles, ntiles, M, C, it, flags, dtg, st); break;
    default: vti ? launch_elastic_t<true, 64, 8>(shots, tiles, ntiles, M, C, it, flags, dtg, st)
                 : launch_elastic_t<false, 64, 8>(shots, tiles, ntiles, M, C, it, flags, dtg, st); break;
    }
}

void launch_scatter_init(const ShotDev *shots, int nshots, const InitEntry *ent, const int *off, cudaStream_t st)
{
    scatter_init<<<nshots, 128, 0, st>>>(shots, nshots, ent, off);
}

void launch_finalize(const ShotDev *shots, int nshots, const StepConst &C, int ncomp, int flags, cudaStream_t st)
{
    dim3 grid(148, nshots);
    finalize_shots<<<grid, 256, 0, st>>>(shots, nshots, C, ncomp, flags);
}

void launch_vti_grad_coefs(int n, const float *lam, const float *mu, const float *c13, float *v2, float *v3, cudaStream_t st)
{
    vti_grad_coefs<<<296, 256, 0, st>>>(n, lam, mu, c13, v2, v3);
}

}  // namespace fwi2d
