// Left / right band kernel: the cells within 6 of the left or right edge,
// over the full height, in framed and marching plans.
//
// One CTA takes one 32 x 8 window of a band (a TileRef from the tile plans'
// full-height band windows: 32 z cells, the band's 6 columns and the 2
// columns next to them, owned cells [ox0, ox1) x [oz0, oz1)).  The window is
// staged and differentiated as in the tile kernel's general path.  The two
// field components of a cell are then updated by two different warps: warps
// 0-5 take ux of columns 0-5 of the band, warps 6-11 take uz; in the adjoint,
// warps 12-17 take the lambda and mu terms of the imaging condition, which
// need first derivatives only.  Every one of these cells sits in the x
// closure of the SBP operators, so the arithmetic of one cell is long and
// serial; spreading it over warps shortens the instruction chain that sets
// the band's time, and the band sets the time of a step on a single shot.
// Each component keeps the reference's own operation order (the terms of ux
// and of uz never mix until the density term of the imaging condition,
// whose float sum the ux warp forms from the uz warp's product, passed
// through shared memory behind a barrier of those two warp groups only).
// Elastic isotropic and VTI, not the acoustic-elastic propagator (which runs
// on tile plans).
//
// The arithmetic is the tile kernel's general path (src/cpp/we_op.cpp:667-871
// elastic, :1640-1840 VTI, closures of src/include/spatial_operators.hpp,
// imaging condition we_op.cpp:505-562, 1478-1557), through the same sbp.cuh
// routines.
#pragma once

namespace fwi2d {

// threads per CTA: 2 components (and, in the adjoint, the imaging terms) x 6 band columns x 32 z cells
template <bool GRAD>
__host__ __device__ constexpr int xband_threads() { return GRAD ? 576 : 384; }

template <bool VTI, bool GRAD>
__global__ void __launch_bounds__(xband_threads<GRAD>(), 1)
elastic_xband(const ShotDev *__restrict__ shots, const TileRef *__restrict__ tiles, ModelDev M, StepConst C, int it,
              int flags, float dtg)
{
    constexpr int TZ = 32, TX = 8;
    constexpr int UZ = TZ + 8, UX = TX + 8, WZ = TZ + 4, WX = TX + 4;
    constexpr int NT = xband_threads<GRAD>();
    __shared__ __align__(16) float U0[UX * UZ];
    __shared__ __align__(16) float U1[UX * UZ];
    __shared__ float MU[WX * WZ], Q[WX * WZ];   // mu; lambda (iso) or (1+2eps)2mu (VTI)
    __shared__ float T0[WX * WZ];               // iso: ux_x+uz_z ; VTI: tmp_x
    __shared__ float BX[WX * WZ], CZ[WX * WZ];  // uz_x, ux_z
    __shared__ float T1[VTI ? WX * WZ : 1];     // VTI: tmp_z
    __shared__ float F0[GRAD ? WX * WZ : 1], F1[GRAD ? WX * WZ : 1];
    __shared__ float XP[GRAD ? 6 * TZ : 1];     // uz warp's density-term product per cell
    __shared__ float red[NT / 32];

    const TileRef tr = tiles[blockIdx.x];
    const ShotDev *__restrict__ Sp = shots + tr.shot;
    const int nt = Sp->nt;
    if (it >= nt - 1) return;
    const int nx = Sp->nx, nz = Sp->nz, ldz = Sp->ldz;
    const int nxz = nx * ldz;
    const int wx0 = tr.wx0, wz0 = tr.wz0;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int comp = warp / 6, c = warp - 6 * comp;   // comp 0: ux, 1: uz, 2: imaging terms (adjoint)
    const bool stencil = comp < 2;

    const float *__restrict__ curr = Sp->u[(it + 1) & 1];
    float *__restrict__ pn = Sp->u[it & 1];   // prev in, next out
    const int mld = M.ldz;
    const long long mofs = (long long)Sp->x0 * mld;
    const float *__restrict__ mp0 = M.p0 + mofs;
    const float *__restrict__ mp1 = M.p1 + mofs;
    const float *__restrict__ mp2 = M.p2 + mofs;
    const float *__restrict__ qsrc = VTI ? M.fxx + mofs : mp0;

    const int itf = GRAD ? (nt - 1 - (it + 1)) / C.sub : 0;
    const bool do_grad = GRAD && (flags & F_GRAD) && ((nt - 1 - (it + 1)) % C.sub == 0);
    const int prec = C.snap_prec;
    const long long slot_elems = Sp->snap_slot;
    const void *snap = Sp->snap;
    const int last = nt / C.sub;

    // this thread's cell and component; its own operands are loaded first so
    // that their latency overlaps the staging and the first derivatives
    const int gx = tr.ox0 + c, gz = wz0 + lane;
    const int tx = gx - wx0;
    const bool owned = gz >= tr.oz0 && gz < tr.oz1;
    const int cell = gx * ldz + gz, mcell = gx * mld + gz;
    float p = 0.f, rho = 1.f, tzv = 0.f, txv = 0.f;
    float hfp = 0.f, hfm = 0.f, hg0 = 0.f, hg1 = 0.f, hg2 = 0.f;
    if (owned && stencil) {
        p = pn[comp * nxz + cell];
        rho = mp2[mcell];
        tzv = Sp->tz[gz];
        txv = Sp->tx[gx];
        if (GRAD && do_grad) {
            if (itf + 1 <= last) {
                const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf + 1);
                hfp = snap_load(snap, (long long)(itf + 1) * slot_elems + comp * nxz + cell, prec, inv);
            }
            if (itf > 0) {
                const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf - 1);
                hfm = snap_load(snap, (long long)(itf - 1) * slot_elems + comp * nxz + cell, prec, inv);
            }
            if (comp == 0) hg2 = Sp->grad[cell + 2 * (long long)nxz];
        }
    }
    if (GRAD && do_grad && owned && comp == 2) {
        hg0 = Sp->grad[cell];
        hg1 = Sp->grad[cell + (long long)nxz];
    }
    float finv = 1.f;
    if (GRAD && do_grad && prec != SNAP_FP32) finv = 1.f / snap_scale(Sp->snap_amax, itf);

    // ---- curr with a 4-cell halo, coefficients and snapshot with a 2-cell halo
    for (int i = t; i < UX * UZ; i += NT) {
        const int sx = i / UZ, sz = i - sx * UZ;
        const int x = wx0 - 4 + sx, z = wz0 - 4 + sz;
        float a = 0.f, b = 0.f;
        if (x >= 0 && x < nx && z >= 0 && z < nz) {
            const int o = x * ldz + z;
            a = curr[o];
            b = curr[nxz + o];
        }
        U0[i] = a;
        U1[i] = b;
    }
    for (int i = t; i < WX * WZ; i += NT) {
        const int sx = i / WZ, sz = i - sx * WZ;
        const int x = wx0 - 2 + sx, z = wz0 - 2 + sz;
        float m = 0.f, q = 0.f;
        const bool in = x >= 0 && x < nx && z >= 0 && z < nz;
        if (in) {
            const int o = x * mld + z;
            m = mp1[o];
            q = qsrc[o];
        }
        MU[i] = m;
        Q[i] = q;
        if (GRAD) {
            float f0 = 0.f, f1 = 0.f;
            if (do_grad && in) {
                const long long o = (long long)itf * slot_elems + x * ldz + z;
                f0 = snap_load(snap, o, prec, finv);
                f1 = snap_load(snap, o + nxz, prec, finv);
            }
            F0[i] = f0;
            F1[i] = f1;
        }
    }
    __syncthreads();

    // ---- first derivatives of curr on the window plus a 2-cell halo
    for (int i = t; i < WX * WZ; i += NT) {
        const int sx = i / WZ, sz = i - sx * WZ;
        const int x = wx0 - 2 + sx, z = wz0 - 2 + sz;
        const int ui = (sx + 2) * UZ + (sz + 2);
        // a closure reads up to 5 samples from its boundary: evaluate only
        // where the loaded window holds them (other points are never used)
        const bool okx = (x >= 4 && x < nx - 4) || (x < 4 ? wx0 <= 4 : wx0 + TX + 4 >= nx);
        const bool okz = (z >= 4 && z < nz - 4) || (z < 4 ? wz0 <= 4 : wz0 + TZ + 4 >= nz);
        const bool ok = x >= 0 && x < nx && z >= 0 && z < nz && okx && okz;
        float t0 = 0.f, t1 = 0.f, bx = 0.f, cz = 0.f;
        if (ok) {
            const float ux_x = d1(U0 + ui, UZ, x, nx, C.dx, C.sdx);
            const float uz_z = d1(U1 + ui, 1, z, nz, C.dz, C.sdz);
            bx = d1(U1 + ui, UZ, x, nx, C.dx, C.sdx);
            cz = d1(U0 + ui, 1, z, nz, C.dz, C.sdz);
            if (!VTI) {
                t0 = ux_x + uz_z;
            } else {
                const long long o = mofs + (long long)x * mld + z;
                const float lb = M.lbis[o], c13 = M.c13[o], lam = M.p0[o];
                t0 = lb * ux_x + c13 * uz_z;
                t1 = lam * uz_z + c13 * ux_x;
            }
        }
        T0[i] = t0;
        if (VTI) T1[i] = t1;
        BX[i] = bx;
        CZ[i] = cz;
    }
    __syncthreads();

    // receivers (forward): one thread per receiver of this window
    if (flags & F_EXTRACT) {
        const int e0 = Sp->ext_off[tr.unit], e1 = Sp->ext_off[tr.unit + 1];
        for (int e = e0 + t; e < e1; e += NT) {
            const ExtEntry &E = Sp->ext[e];
            const float *U = E.comp == 0 ? U0 : U1;
            const int base = (E.gx0 - wx0 + 4) * UZ + (E.gz0 - wz0 + 4);
            float o = 0.f;
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) o += E.w[a * 3 + b] * U[base + a * UZ + b];
            Sp->rcv[(long long)it * Sp->nrcv + E.row] = o;
        }
    }

    // ---- one component of one cell
    const int ui = (tx + 4) * UZ + (lane + 4);
    const int wi = (tx + 2) * WZ + (lane + 2);
    const float *Uc = comp == 0 ? U0 : U1;
    float n = 0.f, amax = 0.f;
    if (owned && stencil) {
        const bool store = (flags & F_STORE) && (it % C.sub == 0);
        if (store) {
            const int slot = it / C.sub;
            const float sc = prec == SNAP_FP32 ? 1.f : snap_scale(Sp->snap_amax, slot);
            snap_store(Sp->snap, (long long)slot * slot_elems + comp * nxz + cell, prec, Uc[ui], sc);
        }
        if (comp == 0) {
            if (!VTI) d2acc(n, U0 + ui, UZ, MU + wi, WZ, 2.f, gx, nx, C.inv_d2x, C.d2x);
            else d2acc(n, U0 + ui, UZ, Q + wi, WZ, 1.f, gx, nx, C.inv_d2x, C.d2x);
            d2acc(n, U0 + ui, 1, MU + wi, 1, 1.f, gz, nz, C.inv_d2z, C.d2z);
            if (!VTI) n += md1(T0 + wi, Q + wi, WZ, gx, nx, C.adx);
            else n += d1(T0 + wi, WZ, gx, nx, C.dx, C.sdx);
            n += md1(BX + wi, MU + wi, 1, gz, nz, C.adz);
        } else {
            d2acc(n, U1 + ui, 1, MU + wi, 1, 2.f, gz, nz, C.inv_d2z, C.d2z);
            d2acc(n, U1 + ui, UZ, MU + wi, WZ, 1.f, gx, nx, C.inv_d2x, C.d2x);
            if (!VTI) n += md1(T0 + wi, Q + wi, 1, gz, nz, C.adz);
            else n += d1(T1 + wi, 1, gz, nz, C.dz, C.sdz);
            n += md1(CZ + wi, MU + wi, WZ, gx, nx, C.adx);
        }
        const int e0 = Sp->inj_off[tr.unit], e1 = Sp->inj_off[tr.unit + 1];
        if (e0 < e1) {
            const float *srcrow = Sp->src + (long long)it * Sp->nsrc;
            for (int e = e0; e < e1; e++) {
                const InjEntry &E = Sp->inj[e];
                if (E.gx == gx && E.gz == gz && E.comp == comp)
                    n += E.mt ? (E.wa * srcrow[E.ia] - E.wb * srcrow[E.ib]) : E.wa * srcrow[E.ia];
            }
        }
        if (it > 0) p = p * tzv * txv;

        // SAT closures (spatial_operators.hpp:160-822), this component's terms in the reference's side order
        const bool edge = gz == 0 || gz == nz - 1 || gx == 0 || gx == nx - 1;
        if (edge) {
            const float mu = MU[wi];
            const float lam = VTI ? mp0[mcell] : Q[wi];
            const float c13 = VTI ? M.c13[mofs + mcell] : lam;
            const float fxx = VTI ? Q[wi] : 2 * mu;
            const float lamx = VTI ? M.lbis[mofs + mcell] : lam;
            const float eps = VTI ? M.eps[mofs + mcell] : 0.f;
            const float imp_s = 0.5f * sqrtf(mu * rho);
            const float imp_p = 0.5f * sqrtf((lam + 2 * mu) * rho);
            const float imp_px = VTI ? 0.5f * sqrtf((1 + 2 * eps) * (lam + 2 * mu) * rho) : imp_p;
#pragma unroll 1
            for (int side = 0; side < 4; side++) {
                // a select, not an indexed read: an indexed kernel parameter would be copied to the stack
                const int bc = side == 0 ? C.bc[0] : side == 1 ? C.bc[1] : side == 2 ? C.bc[2] : C.bc[3];
                if (bc != 1 && bc != 2) continue;
                const bool ab = bc == 2;
                if (side < 2) {
                    if (gz != (side == 0 ? 0 : nz - 1)) continue;
                    const int in = side == 0 ? 1 : -1;
                    const float sg = side == 0 ? -1.f : 1.f;
                    if (comp == 0) {
                        float tt = (sg * mu) * tsum(U1 + ui, UZ, gx, nx) / C.dx + mu * nsum(U0 + ui, in) / C.dz;
                        if (ab) tt = tt - imp_s * p / C.dt;
                        n = n - C.sat_z * tt;
                    } else {
                        float tt = (sg * c13) * tsum(U0 + ui, UZ, gx, nx) / C.dx + (2 * mu) * nsum(U1 + ui, in) / C.dz;
                        if (ab) tt = tt - imp_p * p / C.dt;
                        n = n - C.sat_z * tt;
                        n = n - C.nsat_z * lam * ndsum(U1 + ui, in);
                    }
                } else {
                    if (gx != (side == 2 ? 0 : nx - 1)) continue;
                    const int in = side == 2 ? UZ : -UZ;
                    const float sg = side == 2 ? -1.f : 1.f;
                    if (comp == 0) {
                        float tt = (sg * c13) * tsum(U1 + ui, 1, gz, nz) / C.dz + fxx * nsum(U0 + ui, in) / C.dx;
                        if (ab) tt = tt - imp_px * p / C.dt;
                        n = n - C.sat_x * tt;
                        n = n - C.nsat_x * lamx * ndsum(U0 + ui, in);
                    } else {
                        float tt = (sg * mu) * tsum(U0 + ui, 1, gz, nz) / C.dz + mu * nsum(U1 + ui, in) / C.dx;
                        if (ab) tt = tt - imp_s * p / C.dt;
                        n = n - C.sat_x * tt;
                    }
                }
            }
        }

        n = C.dt2 * n / rho + 2 * Uc[ui] - p;
        if (edge) {
            const int per = 2 * nx + 2 * nz;
            int k;
            if (gz == 0) k = gx;
            else if (gz == nz - 1) k = nx + gx;
            else if (gx == 0) k = 2 * nx + gz;
            else k = 2 * nx + nz + gz;
            n = n / Sp->den[comp * per + k];
        }
        n = n * tzv * txv;
        pn[comp * nxz + cell] = n;
        amax = fabsf(n);
    }

    if (GRAD && do_grad) {
        float *g0 = Sp->grad + cell, *g1 = g0 + nxz, *g2 = g1 + nxz;
        const float gw = Sp->gwt[itf];
        if (comp == 2) {
            // lambda and mu terms: first derivatives of curr and of the snapshot
            if (owned) {
                const float ax0 = d1(U0 + ui, UZ, gx, nx, C.dx, C.sdx);
                const float az1 = d1(U1 + ui, 1, gz, nz, C.dz, C.sdz);
                const float t0 = d1(F0 + wi, WZ, gx, nx, C.dx, C.sdx);
                const float t1 = d1(F1 + wi, 1, gz, nz, C.dz, C.sdz);
                const float t2 = d1(F1 + wi, WZ, gx, nx, C.dx, C.sdx);
                const float t3 = d1(F0 + wi, 1, gz, nz, C.dz, C.sdz);
                const float az0 = CZ[wi], ax1 = BX[wi];
                float dl, dm;
                if (!VTI) {
                    dl = 0.f;
                    dm = (az0 + ax1) * (t2 + t3) + 2 * ax0 * t0 + 2 * az1 * t1;
                } else {
                    const long long mo = mofs + mcell;
                    const float e2 = 1 + 2 * M.eps[mo];
                    const float v2 = M.gv2[mo], v3 = M.gv3[mo];
                    dl = e2 * ax0 * t0 + az1 * t1 + v2 * (ax0 * t1 + az1 * t0);
                    dm = (az0 + ax1) * (t2 + t3) + 2 * e2 * ax0 * t0 + 2 * az1 * t1 + v3 * (ax0 * t1 + az1 * t0);
                }
                if (itf == 0) {
                    const double wh = (double)gw * 0.5 * (double)dtg;
                    if (!VTI) *g0 = (float)((double)hg0 + wh * (double)(ax0 + az1) * (double)(t0 + t1));
                    else *g0 = (float)((double)hg0 + wh * (double)dl);
                    *g1 = (float)((double)hg1 + wh * (double)dm);
                } else {
                    if (!VTI) *g0 = hg0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                    else *g0 = hg0 + gw * dtg * dl;
                    *g1 = hg1 + gw * dtg * dm;
                }
            }
        } else {
            // density term: each component's product; the ux warp forms their
            // float sum in the reference's order, behind a barrier of the 12
            // stencil warps only (named barrier 1)
            float prod = 0.f;
            if (owned) {
                const float f = comp == 0 ? F0[wi] : F1[wi];
                if (itf > 0 && itf < last) prod = n * (hfp - 2 * f + hfm);
                else if (itf == 0) prod = n * (hfp - f);
                else prod = n * (-f + hfm);
            }
            const int xi = c * TZ + lane;
            if (comp == 1) XP[xi] = prod;
            asm volatile("bar.sync 1, 384;" ::: "memory");
            if (owned && comp == 0) {
                const double wdt = (double)gw * 1.0 / (double)dtg;
                *g2 = (float)((double)hg2 + wdt * (double)(prod + XP[xi]));
            }
        }
    }

    // max |next| for the scale of the next 16-bit snapshot
    if ((flags & F_AMAX) && ((it + 1) % C.sub == 0)) {
        float m = amax;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) red[warp] = m;
        __syncthreads();
        if (t == 0) {
            m = red[0];
            for (int w = 1; w < NT / 32; w++) m = fmaxf(m, red[w]);
            if (m > 0.f) atomicMax(Sp->snap_amax + (it + 1) / C.sub, __float_as_uint(m));
        }
    }
}

}  // namespace fwi2d
