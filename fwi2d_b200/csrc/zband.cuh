// Top / bottom band kernel: the cells within 6 of the top or bottom edge, for
// the rows clear of the x boundary bands (6 <= x < nx-6), in plans whose
// interior runs on the marching kernel.
//
// One CTA takes XB consecutive rows of one band on 384 threads.  The rows
// (with a 4-row halo) and the 10 z-samples next to the edge are staged in
// shared memory and the first derivatives are formed there.  Then:
//   - SPLIT = false (XB = 64): thread k XB + r updates cell k (k-th cell from
//     the edge) of row xb + r, both components;
//   - SPLIT = true (XB = 32): thread (comp 6 + k) XB + r updates component
//     comp (0: ux, 1: uz) of that cell.  The two components of a cell go to
//     two warps, which halves the serial closure chain of a thread; plans
//     whose few band CTAs set the time of a step (one shot) take it.  The
//     larger CTAs cost the interior kernel registers on their SMs, so plans
//     of many shots keep SPLIT = false.  Each component keeps the
//     reference's operation order; the density term of the imaging
//     condition, which sums one product of each component, is formed by the
//     ux warp from the uz warp's product passed through shared memory, and
//     the ux warp takes the lambda term and the uz warp the mu term.
// Every lane of a warp sits on the same closure row (the same k) and the
// same component, so the SBP closure coefficients are uniform reads and no
// lane diverges.  The arithmetic is the tile kernel's general path
// (src/cpp/we_op.cpp:667-871 elastic, :1640-1840 VTI, closures of
// src/include/spatial_operators.hpp), through the same sbp.cuh routines.
#pragma once

namespace fwi2d {

constexpr int kZbRows = 64;        // rows per band CTA, both components per thread
constexpr int kZbSplitRows = 32;   // rows per band CTA, one component per thread
constexpr int kZbCols = 10;        // z-samples staged next to the edge
constexpr int kZbThreads = 384;    // 6 cells x 64 rows, or 2 components x 6 cells x 32 rows

template <bool VTI, bool GRAD, bool SPLIT>
__global__ void __launch_bounds__(kZbThreads)
elastic_zband(const ShotDev *__restrict__ shots, const BandRef *__restrict__ units, ModelDev M, StepConst C, int it,
              int flags, float dtg)
{
    constexpr int XB = SPLIT ? kZbSplitRows : kZbRows, ZW = kZbCols, NT = kZbThreads;
    static_assert(NT == (SPLIT ? 12 : 6) * XB, "one thread per cell (and component)");
    constexpr int NR4 = XB + 8, NR2 = XB + 4;
    __shared__ float U0[NR4 * ZW], U1[NR4 * ZW];            // curr, rows xb-4 ..
    __shared__ float MU[NR2 * ZW], Q[NR2 * ZW];             // mu; lambda (iso) or (1+2eps)(lambda+2mu) (VTI), rows xb-2 ..
    __shared__ float T0[NR2 * ZW], CZ[NR2 * ZW];            // iso: ux_x+uz_z, VTI: lbis ux_x + c13 uz_z; ux_z
    __shared__ float BX[XB * ZW], T1[VTI ? XB * ZW : 1];    // uz_x; VTI: lambda uz_z + c13 ux_x (own rows)
    __shared__ float F0[GRAD ? NR2 * ZW : 1], F1[GRAD ? NR2 * ZW : 1];
    __shared__ float XP[GRAD && SPLIT ? 6 * XB : 1];        // uz warp's density-term product per cell
    __shared__ float GD[4][GRAD && SPLIT ? 6 * XB : 1];     // ux warp's first derivatives of the lambda term
    __shared__ float red[NT / 32];

    const BandRef U = units[blockIdx.x];
    const ShotDev *__restrict__ Sp = shots + U.shot;
    const int nt = Sp->nt;
    if (it >= nt - 1) return;
    const int nx = Sp->nx, nz = Sp->nz, ldz = Sp->ldz, nxz = nx * ldz, mld = M.ldz;
    const int xb = U.xb, xe = U.xe, t = threadIdx.x;
    const bool top = U.side == 0;
    const int zb = top ? 0 : nz - ZW;            // z of staged column 0
    const int c0 = top ? 0 : ZW - 6;             // first owned column
    const int d0 = top ? 0 : 2, d1c = top ? 8 : ZW;   // derivative columns [d0, d1c)
    const float *__restrict__ curr = Sp->u[(it + 1) & 1];
    float *__restrict__ pn = Sp->u[it & 1];
    const long long mofs = (long long)Sp->x0 * mld;
    const float *__restrict__ qsrc = (VTI ? M.fxx : M.p0) + mofs;
    const int prec = C.snap_prec;
    const int itf = GRAD ? (nt - 1 - (it + 1)) / C.sub : 0;
    const bool do_grad = GRAD && (flags & F_GRAD) && ((nt - 1 - (it + 1)) % C.sub == 0);
    float finv = 1.f;
    if (GRAD && do_grad && prec != SNAP_FP32) finv = 1.f / snap_scale(Sp->snap_amax, itf);

    // ---- stage curr (rows xb-4 .. xe+3), coefficients and snapshot (rows xb-2 .. xe+1)
    for (int i = t; i < NR4 * ZW; i += NT) {
        const int r = i / ZW, c = i - r * ZW, gx = xb - 4 + r;
        float a = 0.f, b = 0.f;
        if (gx < xe + 4) {
            const long long o = (long long)gx * ldz + zb + c;
            a = curr[o];
            b = curr[nxz + o];
        }
        U0[i] = a;
        U1[i] = b;
    }
    for (int i = t; i < NR2 * ZW; i += NT) {
        const int r = i / ZW, c = i - r * ZW, gx = xb - 2 + r;
        float m = 0.f, q = 0.f, f0 = 0.f, f1 = 0.f;
        if (gx < xe + 2) {
            const long long o = mofs + (long long)gx * mld + zb + c;
            m = M.p1[o];
            q = qsrc[(long long)gx * mld + zb + c];
            if (GRAD && do_grad) {
                const long long so = (long long)itf * Sp->snap_slot + (long long)gx * ldz + zb + c;
                f0 = snap_load(Sp->snap, so, prec, finv);
                f1 = snap_load(Sp->snap, so + nxz, prec, finv);
            }
        }
        MU[i] = m;
        Q[i] = q;
        if (GRAD) {
            F0[i] = f0;
            F1[i] = f1;
        }
    }
    __syncthreads();

    // ---- first derivatives (the tile kernel's phase 2)
    for (int i = t; i < NR2 * ZW; i += NT) {
        const int r = i / ZW, c = i - r * ZW, gx = xb - 2 + r;
        float t0 = 0.f, cz = 0.f;
        if (gx < xe + 2 && c >= d0 && c < d1c) {
            const int gz = zb + c;
            const int ui = (r + 2) * ZW + c;
            const float ux_x = d1(U0 + ui, ZW, gx, nx, C.dx, C.sdx);
            const float uz_z = d1(U1 + ui, 1, gz, nz, C.dz, C.sdz);
            cz = d1(U0 + ui, 1, gz, nz, C.dz, C.sdz);
            if (!VTI) {
                t0 = ux_x + uz_z;
            } else {
                const long long o = mofs + (long long)gx * mld + gz;
                const float lb = M.lbis[o], c13 = M.c13[o], lam = M.p0[o];
                t0 = lb * ux_x + c13 * uz_z;
                if (r >= 2 && r < XB + 2) T1[(r - 2) * ZW + c] = lam * uz_z + c13 * ux_x;
            }
        }
        T0[i] = t0;
        CZ[i] = cz;
    }
    for (int i = t; i < XB * ZW; i += NT) {
        const int r = i / ZW, c = i - r * ZW, gx = xb + r;
        float bx = 0.f;
        if (gx < xe && c >= d0 && c < d1c) bx = d1(U1 + (r + 4) * ZW + c, ZW, gx, nx, C.dx, C.sdx);
        BX[i] = bx;
    }
    __syncthreads();

    float amax = 0.f;
    if constexpr (SPLIT) {
        // ---- component comp of cell k of row gx
        const int comp = t / (6 * XB), k = (t / XB) % 6, tr = t % XB;   // comp and k are uniform across a warp
        const int gx = xb + tr;
        const bool owned = gx < xe;
        const int c = c0 + k, gz = zb + c;
        const int ui = (tr + 4) * ZW + c, wi = (tr + 2) * ZW + c, bi = tr * ZW + c;
        const long long cell = (long long)gx * ldz + gz;
        const long long mcell = mofs + (long long)gx * mld + gz;
        const int last = nt / C.sub;
        float n = 0.f;
        if (owned) {
            const MarchRow R = Sp->mrow[U.roff + tr];
            const float txv = R.tx;
            if (comp == 0) {
                if (!VTI) d2acc(n, U0 + ui, ZW, MU + wi, ZW, 2.f, gx, nx, C.inv_d2x, C.d2x);
                else d2acc(n, U0 + ui, ZW, Q + wi, ZW, 1.f, gx, nx, C.inv_d2x, C.d2x);
                d2acc(n, U0 + ui, 1, MU + wi, 1, 1.f, gz, nz, C.inv_d2z, C.d2z);
                if (!VTI) n += md1(T0 + wi, Q + wi, ZW, gx, nx, C.adx);
                else n += d1(T0 + wi, ZW, gx, nx, C.dx, C.sdx);
                n += md1(BX + bi, MU + wi, 1, gz, nz, C.adz);
            } else {
                d2acc(n, U1 + ui, 1, MU + wi, 1, 2.f, gz, nz, C.inv_d2z, C.d2z);
                d2acc(n, U1 + ui, ZW, MU + wi, ZW, 1.f, gx, nx, C.inv_d2x, C.d2x);
                if (!VTI) n += md1(T0 + wi, Q + wi, 1, gz, nz, C.adz);
                else n += d1(T1 + bi, 1, gz, nz, C.dz, C.sdz);
                n += md1(CZ + wi, MU + wi, ZW, gx, nx, C.adx);
            }
            // sources of this cell and component, in the reference's order
            if (R.e0 < R.e1) {
                const float *srcrow = Sp->src + (long long)it * Sp->nsrc;
                for (int e = R.e0; e < R.e1; e++) {
                    const InjEntry &E = Sp->inj[e];
                    if (E.gz != gz || E.comp != comp) continue;
                    n += E.mt ? (E.wa * srcrow[E.ia] - E.wb * srcrow[E.ib]) : E.wa * srcrow[E.ia];
                }
            }
            const bool store = (flags & F_STORE) && (it % C.sub == 0);
            const int slot = it / C.sub;
            const float tzv = Sp->tz[gz];
            float p = pn[comp * nxz + cell];
            if (it > 0) p = p * tzv * txv;
            const float rho = M.p2[mcell];
            const bool edge = gz == 0 || gz == nz - 1;
            const int side = gz == 0 ? 0 : 1;
            const int bc = side == 0 ? C.bc[0] : C.bc[1];   // a select: an indexed parameter would be copied to the stack
            if (edge && (bc == 1 || bc == 2)) {
                // esat_neumann / esat_absorbing top or bottom (spatial_operators.hpp:160-727), esat_Dz (:732-776)
                const float mu = MU[wi];
                const float lam = VTI ? M.p0[mcell] : Q[wi];
                const float c13 = VTI ? M.c13[mcell] : lam;
                const bool ab = bc == 2;
                const int in = side == 0 ? 1 : -1;
                const float sg = side == 0 ? -1.f : 1.f;
                if (comp == 0) {
                    const float imp_s = 0.5f * sqrtf(mu * rho);
                    float tt = (sg * mu) * tsum(U1 + ui, ZW, gx, nx) / C.dx + mu * nsum(U0 + ui, in) / C.dz;
                    if (ab) tt = tt - imp_s * p / C.dt;
                    n = n - C.sat_z * tt;
                } else {
                    const float imp_p = 0.5f * sqrtf((lam + 2 * mu) * rho);
                    float tt = (sg * c13) * tsum(U0 + ui, ZW, gx, nx) / C.dx + (2 * mu) * nsum(U1 + ui, in) / C.dz;
                    if (ab) tt = tt - imp_p * p / C.dt;
                    n = n - C.sat_z * tt;
                    n = n - C.nsat_z * lam * ndsum(U1 + ui, in);
                }
            }
            const float *Uc = comp == 0 ? U0 : U1;
            n = C.dt2 * n / rho + 2 * Uc[ui] - p;
            if (edge) {
                const int per = 2 * nx + 2 * nz;
                const int kk = side == 0 ? gx : nx + gx;
                n = n / Sp->den[comp * per + kk];
            }
            n = n * tzv * txv;
            pn[comp * nxz + cell] = n;
            amax = fabsf(n);
            if (store) {
                const float sc = prec != SNAP_FP32 ? snap_scale(Sp->snap_amax, slot) : 1.f;
                const long long o = (long long)slot * Sp->snap_slot + comp * nxz + cell;
                snap_store(Sp->snap, o, prec, Uc[ui], sc);
            }
            // receivers whose pivot lies on this row (one thread per row)
            if ((flags & F_EXTRACT) && k == 0 && comp == 0) {
                for (int e = R.r0; e < R.r1; e++) {
                    const ExtEntry &E = Sp->ext[e];
                    const float *Ub = E.comp == 0 ? U0 : U1;
                    const int base = (E.gx0 - xb + 4) * ZW + (E.gz0 - zb);
                    float o = 0.f;
    #pragma unroll
                    for (int aa = 0; aa < 3; aa++)
    #pragma unroll
                        for (int bb = 0; bb < 3; bb++) o += E.w[aa * 3 + bb] * Ub[base + aa * ZW + bb];
                    Sp->rcv[(long long)it * Sp->nrcv + E.row] = o;
                }
            }
        }
        if (GRAD && do_grad) {
            // The ux warp takes the lambda term, whose four first derivatives
            // it passes to the uz warp for the mu term, and the density term,
            // whose float sum of one product per component it forms in the
            // reference's order from the uz warp's product; the uz warp adds
            // the two further derivatives of the mu term.
            const float gw = Sp->gwt[itf];
            const double wdt = (double)gw * 1.0 / (double)dtg;
            const double wh = (double)gw * 0.5 * (double)dtg;
            const int xi = k * XB + tr;
            float *g0 = Sp->grad + cell, *g1 = g0 + nxz, *g2 = g1 + nxz;
            float prod = 0.f, t2 = 0.f, t3 = 0.f;
            if (owned) {
                const float f = comp == 0 ? F0[wi] : F1[wi];
                float fp = 0.f, fm = 0.f;
                if (itf + 1 <= last) {
                    const float finvp = prec != SNAP_FP32 ? 1.f / snap_scale(Sp->snap_amax, itf + 1) : 1.f;
                    fp = snap_load(Sp->snap, (long long)(itf + 1) * Sp->snap_slot + comp * nxz + cell, prec, finvp);
                }
                if (itf > 0) {
                    const float finvm = prec != SNAP_FP32 ? 1.f / snap_scale(Sp->snap_amax, itf - 1) : 1.f;
                    fm = snap_load(Sp->snap, (long long)(itf - 1) * Sp->snap_slot + comp * nxz + cell, prec, finvm);
                }
                if (itf > 0 && itf < last) prod = n * (fp - 2 * f + fm);
                else if (itf == 0) prod = n * (fp - f);
                else prod = n * (-f + fm);
                if (comp == 0) {
                    const float ax0 = d1(U0 + ui, ZW, gx, nx, C.dx, C.sdx);
                    const float az1 = d1(U1 + ui, 1, gz, nz, C.dz, C.sdz);
                    const float t0 = d1(F0 + wi, ZW, gx, nx, C.dx, C.sdx);
                    const float t1 = d1(F1 + wi, 1, gz, nz, C.dz, C.sdz);
                    GD[0][xi] = ax0;
                    GD[1][xi] = az1;
                    GD[2][xi] = t0;
                    GD[3][xi] = t1;
                    float dl = 0.f;
                    if (VTI) {
                        const float e2 = 1 + 2 * M.eps[mcell];
                        const float v2 = M.gv2[mcell];
                        dl = e2 * ax0 * t0 + az1 * t1 + v2 * (ax0 * t1 + az1 * t0);
                    }
                    if (itf == 0) {
                        if (!VTI) *g0 = (float)((double)*g0 + wh * (double)(ax0 + az1) * (double)(t0 + t1));
                        else *g0 = (float)((double)*g0 + wh * (double)dl);
                    } else {
                        if (!VTI) *g0 = *g0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                        else *g0 = *g0 + gw * dtg * dl;
                    }
                } else {
                    XP[xi] = prod;
                    t2 = d1(F1 + wi, ZW, gx, nx, C.dx, C.sdx);
                    t3 = d1(F0 + wi, 1, gz, nz, C.dz, C.sdz);
                }
            }
            __syncthreads();
            if (owned) {
                if (comp == 0) {
                    *g2 = (float)((double)*g2 + wdt * (double)(prod + XP[xi]));
                } else {
                    const float ax0 = GD[0][xi], az1 = GD[1][xi], t0 = GD[2][xi], t1 = GD[3][xi];
                    const float az0 = CZ[wi], ax1 = BX[bi];
                    float dm;
                    if (!VTI) {
                        dm = (az0 + ax1) * (t2 + t3) + 2 * ax0 * t0 + 2 * az1 * t1;
                    } else {
                        const float e2 = 1 + 2 * M.eps[mcell];
                        const float v3 = M.gv3[mcell];
                        dm = (az0 + ax1) * (t2 + t3) + 2 * e2 * ax0 * t0 + 2 * az1 * t1 + v3 * (ax0 * t1 + az1 * t0);
                    }
                    if (itf == 0) *g1 = (float)((double)*g1 + wh * (double)dm);
                    else *g1 = *g1 + gw * dtg * dm;
                }
            }
        }
    } else {
        // ---- cell k of row gx
        const int k = t / XB, tr = t - k * XB;   // k is uniform across a warp
        const int gx = xb + tr;
        if (gx < xe) {
            const MarchRow R = Sp->mrow[U.roff + tr];
            const float txv = R.tx;
            const int c = c0 + k, gz = zb + c;
            const int ui = (tr + 4) * ZW + c, wi = (tr + 2) * ZW + c, bi = tr * ZW + c;
            float a = 0.f, b = 0.f;
            if (!VTI) {
                d2acc(a, U0 + ui, ZW, MU + wi, ZW, 2.f, gx, nx, C.inv_d2x, C.d2x);
                d2acc(b, U1 + ui, 1, MU + wi, 1, 2.f, gz, nz, C.inv_d2z, C.d2z);
            } else {
                d2acc(a, U0 + ui, ZW, Q + wi, ZW, 1.f, gx, nx, C.inv_d2x, C.d2x);
                d2acc(b, U1 + ui, 1, MU + wi, 1, 2.f, gz, nz, C.inv_d2z, C.d2z);
            }
            d2acc(b, U1 + ui, ZW, MU + wi, ZW, 1.f, gx, nx, C.inv_d2x, C.d2x);
            d2acc(a, U0 + ui, 1, MU + wi, 1, 1.f, gz, nz, C.inv_d2z, C.d2z);
            if (!VTI) {
                a += md1(T0 + wi, Q + wi, ZW, gx, nx, C.adx);
                b += md1(T0 + wi, Q + wi, 1, gz, nz, C.adz);
            } else {
                a += d1(T0 + wi, ZW, gx, nx, C.dx, C.sdx);
                b += d1(T1 + bi, 1, gz, nz, C.dz, C.sdz);
            }
            b += md1(CZ + wi, MU + wi, ZW, gx, nx, C.adx);
            a += md1(BX + bi, MU + wi, 1, gz, nz, C.adz);
            // sources of this cell, in the reference's order
            if (R.e0 < R.e1) {
                const float *srcrow = Sp->src + (long long)it * Sp->nsrc;
                for (int e = R.e0; e < R.e1; e++) {
                    const InjEntry &E = Sp->inj[e];
                    if (E.gz != gz) continue;
                    const float v = E.mt ? (E.wa * srcrow[E.ia] - E.wb * srcrow[E.ib]) : E.wa * srcrow[E.ia];
                    if (E.comp == 0) a += v;
                    else b += v;
                }
            }
            const long long cell = (long long)gx * ldz + gz;
            const long long mcell = mofs + (long long)gx * mld + gz;
            const bool store = (flags & F_STORE) && (it % C.sub == 0);
            const int slot = it / C.sub;
            const int last = nt / C.sub;
            const float tzv = Sp->tz[gz];
            float p0 = pn[cell], p1 = pn[nxz + cell];
            if (it > 0) {
                p0 = p0 * tzv * txv;
                p1 = p1 * tzv * txv;
            }
            const float rho = M.p2[mcell];
            const bool edge = gz == 0 || gz == nz - 1;
            const int side = gz == 0 ? 0 : 1;
            const int bc = side == 0 ? C.bc[0] : C.bc[1];   // a select: an indexed parameter would be copied to the stack
            if (edge && (bc == 1 || bc == 2)) {
                // esat_neumann / esat_absorbing top or bottom (spatial_operators.hpp:160-727), esat_Dz (:732-776)
                const float mu = MU[wi];
                const float lam = VTI ? M.p0[mcell] : Q[wi];
                const float c13 = VTI ? M.c13[mcell] : lam;
                const float imp_s = 0.5f * sqrtf(mu * rho);
                const float imp_p = 0.5f * sqrtf((lam + 2 * mu) * rho);
                const bool ab = bc == 2;
                const int in = side == 0 ? 1 : -1;
                const float sg = side == 0 ? -1.f : 1.f;
                {
                    float tt = (sg * mu) * tsum(U1 + ui, ZW, gx, nx) / C.dx + mu * nsum(U0 + ui, in) / C.dz;
                    if (ab) tt = tt - imp_s * p0 / C.dt;
                    a = a - C.sat_z * tt;
                }
                {
                    float tt = (sg * c13) * tsum(U0 + ui, ZW, gx, nx) / C.dx + (2 * mu) * nsum(U1 + ui, in) / C.dz;
                    if (ab) tt = tt - imp_p * p1 / C.dt;
                    b = b - C.sat_z * tt;
                    b = b - C.nsat_z * lam * ndsum(U1 + ui, in);
                }
            }
            a = C.dt2 * a / rho + 2 * U0[ui] - p0;
            b = C.dt2 * b / rho + 2 * U1[ui] - p1;
            if (edge) {
                const int per = 2 * nx + 2 * nz;
                const int kk = side == 0 ? gx : nx + gx;
                a = a / Sp->den[kk];
                b = b / Sp->den[per + kk];
            }
            a = a * tzv * txv;
            b = b * tzv * txv;
            pn[cell] = a;
            pn[nxz + cell] = b;
            amax = fmaxf(fabsf(a), fabsf(b));
            if (store) {
                const float sc = prec != SNAP_FP32 ? snap_scale(Sp->snap_amax, slot) : 1.f;
                const long long o = (long long)slot * Sp->snap_slot + cell;
                snap_store(Sp->snap, o, prec, U0[ui], sc);
                snap_store(Sp->snap, o + nxz, prec, U1[ui], sc);
            }
            if (GRAD && do_grad) {
                const float gw = Sp->gwt[itf];
                const double wdt = (double)gw * 1.0 / (double)dtg;
                const double wh = (double)gw * 0.5 * (double)dtg;
                const float ax0 = d1(U0 + ui, ZW, gx, nx, C.dx, C.sdx);
                const float az1 = d1(U1 + ui, 1, gz, nz, C.dz, C.sdz);
                const float t0 = d1(F0 + wi, ZW, gx, nx, C.dx, C.sdx);
                const float t1 = d1(F1 + wi, 1, gz, nz, C.dz, C.sdz);
                const float t2 = d1(F1 + wi, ZW, gx, nx, C.dx, C.sdx);
                const float t3 = d1(F0 + wi, 1, gz, nz, C.dz, C.sdz);
                const float az0 = CZ[wi], ax1 = BX[bi];
                const float f0 = F0[wi], f1 = F1[wi];
                float fp0 = 0.f, fp1 = 0.f, fm0 = 0.f, fm1 = 0.f;
                if (itf + 1 <= last) {
                    const float finvp = prec != SNAP_FP32 ? 1.f / snap_scale(Sp->snap_amax, itf + 1) : 1.f;
                    const long long o = (long long)(itf + 1) * Sp->snap_slot + cell;
                    fp0 = snap_load(Sp->snap, o, prec, finvp);
                    fp1 = snap_load(Sp->snap, o + nxz, prec, finvp);
                }
                if (itf > 0) {
                    const float finvm = prec != SNAP_FP32 ? 1.f / snap_scale(Sp->snap_amax, itf - 1) : 1.f;
                    const long long o = (long long)(itf - 1) * Sp->snap_slot + cell;
                    fm0 = snap_load(Sp->snap, o, prec, finvm);
                    fm1 = snap_load(Sp->snap, o + nxz, prec, finvm);
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
                float *g0 = Sp->grad + cell, *g1 = g0 + nxz, *g2 = g1 + nxz;
                if (itf > 0 && itf < last) {
                    if (!VTI) *g0 = *g0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                    else *g0 = *g0 + gw * dtg * dl;
                    *g1 = *g1 + gw * dtg * dm;
                    *g2 = (float)((double)*g2 + wdt * (double)(a * (fp0 - 2 * f0 + fm0) + b * (fp1 - 2 * f1 + fm1)));
                } else if (itf == 0) {
                    if (!VTI) *g0 = (float)((double)*g0 + wh * (double)(ax0 + az1) * (double)(t0 + t1));
                    else *g0 = (float)((double)*g0 + wh * (double)dl);
                    *g1 = (float)((double)*g1 + wh * (double)dm);
                    *g2 = (float)((double)*g2 + wdt * (double)(a * (fp0 - f0) + b * (fp1 - f1)));
                } else {
                    if (!VTI) *g0 = *g0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                    else *g0 = *g0 + gw * dtg * dl;
                    *g1 = *g1 + gw * dtg * dm;
                    *g2 = (float)((double)*g2 + wdt * (double)(a * (-f0 + fm0) + b * (-f1 + fm1)));
                }
            }
            // receivers whose pivot lies on this row (one thread per row)
            if ((flags & F_EXTRACT) && k == 0) {
                for (int e = R.r0; e < R.r1; e++) {
                    const ExtEntry &E = Sp->ext[e];
                    const float *Ub = E.comp == 0 ? U0 : U1;
                    const int base = (E.gx0 - xb + 4) * ZW + (E.gz0 - zb);
                    float o = 0.f;
    #pragma unroll
                    for (int aa = 0; aa < 3; aa++)
    #pragma unroll
                        for (int bb = 0; bb < 3; bb++) o += E.w[aa * 3 + bb] * Ub[base + aa * ZW + bb];
                    Sp->rcv[(long long)it * Sp->nrcv + E.row] = o;
                }
            }
        }
    }

    if ((flags & F_AMAX) && ((it + 1) % C.sub == 0)) {
        const int lane = t & 31, warp = t >> 5;
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
