// x-marching elastic / VTI step kernel for the rows of a shot grid that lie
// clear of the left and right SBP boundary bands (6 <= x < nx-6).
//
// One CTA owns a strip of z (a window of W = NTH cells, one per thread) and
// marches along x over a run of rows [xb, xe).  Rows are contiguous in memory
// (z fastest), so every row of every field is read from HBM once per step with
// coalesced loads.  Along x the stencil samples
// live in per-thread register queues; along z they come from shared-memory
// ring buffers holding the last few rows.  Everything a step reads from
// shared memory was written at an earlier row, so one barrier per row
// suffices.  The arithmetic per cell is the same single-precision sequence
// as the tile kernel's (src/cpp/we_op.cpp:667-871 elastic, :1640-1840 VTI);
// z-boundary cells use the closure forms of sbp.cuh on the ring rows.
//
// Row schedule of step j (output row j):
//   loads       curr row j+5, coefficient and snapshot rows j+3, prev / rho
//               of row j+1 (held in registers until the end of the step, or
//               the next step, so that their latency overlaps the arithmetic);
//   derivatives ux_x, uz_z, ux_z and T0 / T1 of row j+2, uz_x of row j+1
//               (from rows loaded at earlier steps);
//   output      row j: SBP terms, sources, SAT (z edges), leapfrog, taper,
//               receivers, snapshot store or imaging condition;
//   queues      the rows loaded at this step enter the queues and rings.
// The first output row is preceded by 9 steps that only fill the queues.
//
// Shared-memory rings (RW = NTH + 4 floats per row, cell z at index z - za + 2):
//   ux, uz         8 rows (curr, with a 2-cell z halo on each side); register
//                  queues of 8 rows (j-2 .. j+5)
//   mu             4 rows
//   q              4 rows: lambda (isotropic) or T1 (VTI)
//   t              4 rows: T0 = ux_x + uz_z (isotropic only)
//   bx             4 rows: uz_x
//   f0, f1         4 rows: forward snapshot (imaging condition only)
#pragma once

namespace fwi2d {


// Per-thread state that stays fixed during one launch.
struct MarchCtx {
    float *u;                 // curr base (component stride nxz); prev/next at u + pn_off
    long long pn_off;
    long long mofs;           // model offset of the shot's first column + this thread's z
    int ldz, mld, nx, nz, nxz;
    int xb, xe, z, li;
    bool zin, zb4, zb6, own;
    bool hlo, hhi;            // thread loads the low / high 2-cell z halo of curr
    int hz;                   // first halo cell (hlo: za-2, hhi: za+NTH)
    float tzv;
    bool extract, store, do_grad;
    int it, itf, last, prec, slot;
    float sc, finv, finvp, finvm, dtg, gw;
    double wdt, wh;
    int roff, zw0, zw1;
    float amax;
};

template <bool GRAD>
struct MarchQ {
    float ux[8], uz[8], mu[8], q[8], t0[8], cz[8];
    float ax[8], az[8], bx[8], f0[8], f1[8];
    float pv0[2], pv1[2], rh[2];
    float vlb[2], vc13[2], vlam[2];   // VTI coefficients of the next derivative row
};

template <bool VTI, bool GRAD, int NTH>
struct MarchLayout {
    static constexpr int RW = NTH + 4;
    static constexpr int UX = 0, UZ = 8 * RW, MU = 16 * RW, Q = 20 * RW, T = 24 * RW;
    static constexpr int BX = T + (VTI ? 0 : 4 * RW);
    static constexpr int F0 = BX + 4 * RW, F1 = F0 + (GRAD ? 4 * RW : 0);
    static constexpr int RED = F1 + (GRAD ? 4 * RW : 0);
    static constexpr int FLOATS = RED + 32;
};

__device__ __forceinline__ float ldz_pred(const float *p, bool ok) { return ok ? *p : 0.f; }

__device__ __forceinline__ void add_sources(const InjEntry *__restrict__ inj, const float *__restrict__ srcrow, int e0,
                                            int e1, int gz, float &n0, float &n1)
{
    for (int e = e0; e < e1; e++) {
        const InjEntry &E = inj[e];
        if (E.gz == gz) {
            const float v = E.mt ? (E.wa * srcrow[E.ia] - E.wb * srcrow[E.ib]) : E.wa * srcrow[E.ia];
            if (E.comp == 0) n0 += v;
            else n1 += v;
        }
    }
}

template <bool VTI, bool GRAD, int NTH, int P>
__device__ __forceinline__ void march_step(MarchQ<GRAD> &Q, MarchCtx &X, float *sm, const ShotDev *__restrict__ Sp,
                                           const ModelDev &M, const StepConst &C, int j)
{
    using L = MarchLayout<VTI, GRAD, NTH>;
    constexpr int RW = L::RW;
    constexpr int S0 = P & 7, SM1 = (P + 7) & 7, SM2 = (P + 6) & 7, SP1 = (P + 1) & 7, SP2 = (P + 2) & 7,
                  SP3 = (P + 3) & 7, SP4 = (P + 4) & 7, SP5 = (P + 5) & 7;
    constexpr int R0 = P & 3, RP1 = (P + 1) & 3, RP2 = (P + 2) & 3, RP3 = (P + 3) & 3;
    const int li = X.li;
    const float *cur = X.u;

    __syncthreads();

    // ---- loads: curr row j+5 (+ z halo), coefficient and snapshot rows j+3, prev/rho of row j+1
    const long long c4 = (long long)(j + 5) * X.ldz;
    const float nux = ldz_pred(cur + c4 + X.z, X.zin);
    const float nuz = ldz_pred(cur + X.nxz + c4 + X.z, X.zin);
    float h0a = 0.f, h0b = 0.f, h1a = 0.f, h1b = 0.f;
    if (X.hlo || X.hhi) {
        const bool ia = X.hz >= 0 && X.hz < X.nz, ib = X.hz + 1 >= 0 && X.hz + 1 < X.nz;
        h0a = ldz_pred(cur + c4 + X.hz, ia);
        h0b = ldz_pred(cur + c4 + X.hz + 1, ib);
        h1a = ldz_pred(cur + X.nxz + c4 + X.hz, ia);
        h1b = ldz_pred(cur + X.nxz + c4 + X.hz + 1, ib);
    }
    const long long m2 = X.mofs + (long long)(j + 3) * X.mld;
    const float nmu = ldz_pred(M.p1 + m2, X.zin);
    const float nq = ldz_pred((VTI ? M.fxx : M.p0) + m2, X.zin);
    float nlb = 0.f, nc13 = 0.f, nlam = 0.f;
    if (VTI) {
        nlb = ldz_pred(M.lbis + m2, X.zin);
        nc13 = ldz_pred(M.c13 + m2, X.zin);
        nlam = ldz_pred(M.p0 + m2, X.zin);
    }
    float nf0 = 0.f, nf1 = 0.f;
    if (GRAD && X.do_grad && X.zin) {
        const long long so = (long long)X.itf * Sp->snap_slot + (long long)(j + 3) * X.ldz + X.z;
        nf0 = snap_load(Sp->snap, so, X.prec, X.finv);
        nf1 = snap_load(Sp->snap, so + X.nxz, X.prec, X.finv);
    }
    if (j + 1 >= X.xb && j + 1 < X.xe) {
        const float *pn = X.u + X.pn_off;
        const long long o1 = (long long)(j + 1) * X.ldz + X.z;
        Q.pv0[(P + 1) & 1] = ldz_pred(pn + o1, X.zin);
        Q.pv1[(P + 1) & 1] = ldz_pred(pn + X.nxz + o1, X.zin);
        Q.rh[(P + 1) & 1] = ldz_pred(M.p2 + X.mofs + (long long)(j + 1) * X.mld, X.zin);
    }

    // ---- derivatives of row j+2 (its curr ring row was written three steps ago)
    {
        const float *ux2 = sm + L::UX + SP2 * RW + li, *uz2 = sm + L::UZ + SP2 * RW + li;
        const float uxx = d1s(Q.ux[S0], Q.ux[SP1], Q.ux[SP3], Q.ux[SP4], C.sdx);
        float uzz, czz;
        if (!X.zb4) {
            uzz = d1s(uz2[-2], uz2[-1], uz2[1], uz2[2], C.sdz);
            czz = d1s(ux2[-2], ux2[-1], ux2[1], ux2[2], C.sdz);
        } else if (X.zin) {
            uzz = d1(uz2, 1, X.z, X.nz, C.dz, C.sdz);
            czz = d1(ux2, 1, X.z, X.nz, C.dz, C.sdz);
        } else {
            uzz = czz = 0.f;
        }
        float t0;
        if (!VTI) {
            t0 = uxx + uzz;
            sm[L::T + RP2 * RW + li] = t0;
        } else {
            const float vlb = Q.vlb[P & 1], vc13 = Q.vc13[P & 1], vlam = Q.vlam[P & 1];
            t0 = vlb * uxx + vc13 * uzz;
            sm[L::Q + RP2 * RW + li] = vlam * uzz + vc13 * uxx;
        }
        Q.t0[SP2] = t0;
        Q.cz[SP2] = czz;
        if (GRAD) {
            Q.ax[SP2] = uxx;
            Q.az[SP2] = uzz;
        }
    }
    // uz_x of row j+1 from rows j-1 .. j+3
    {
        const float bx = d1s(Q.uz[SM1], Q.uz[S0], Q.uz[SP2], Q.uz[SP3], C.sdx);
        sm[L::BX + RP1 * RW + li] = bx;
        if (GRAD) Q.bx[SP1] = bx;
    }

    // ---- output row j
    if (j >= X.xb) {
        const float *ruxj = sm + L::UX + S0 * RW + li, *ruzj = sm + L::UZ + S0 * RW + li;
        const float *rmuj = sm + L::MU + R0 * RW + li, *rqj = sm + L::Q + R0 * RW + li;
        const float *rtj = sm + L::T + R0 * RW + li, *rbxj = sm + L::BX + R0 * RW + li;
        const float am2 = Q.ux[SM2], am1 = Q.ux[SM1], a00 = Q.ux[S0], ap1 = Q.ux[SP1], ap2 = Q.ux[SP2];
        const float bm2 = Q.uz[SM2], bm1 = Q.uz[SM1], b00 = Q.uz[S0], bp1 = Q.uz[SP1], bp2 = Q.uz[SP2];
        const float mm2 = Q.mu[SM2], mm1 = Q.mu[SM1], m00 = Q.mu[S0], mp1 = Q.mu[SP1], mp2 = Q.mu[SP2];
        const float qm2 = Q.q[SM2], qm1 = Q.q[SM1], q00 = Q.q[S0], qp1 = Q.q[SP1], qp2 = Q.q[SP2];
        const float tm2 = Q.t0[SM2], tm1 = Q.t0[SM1], tp1 = Q.t0[SP1], tp2 = Q.t0[SP2];
        const float cm2 = Q.cz[SM2], cm1 = Q.cz[SM1], cp1 = Q.cz[SP1], cp2 = Q.cz[SP2];
        const float txv = Sp->tx[j];
        const long long cell = (long long)j * X.ldz + X.z;
        const int gz = X.z;

        // sources of this row (entries sorted by z); warps clear of them skip
        const int *inj_roff = Sp->inj_roff;
        const int e0 = inj_roff[X.roff + j - X.xb], e1 = inj_roff[X.roff + j - X.xb + 1];
        bool src_here = false;
        if (e0 < e1) src_here = Sp->inj[e0].gz < X.zw1 && Sp->inj[e1 - 1].gz >= X.zw0;
        const float *srcrow = Sp->src + (long long)X.it * Sp->nsrc;

        const Brk bkx = brk5(mm2, mm1, m00, mp1, mp2);
        float n0, n1;
        if (!VTI) n0 = d2s(0.f, twice(bkx), am2, am1, a00, ap1, ap2, C.inv_d2x);
        else n0 = d2s(0.f, brk5(qm2, qm1, q00, qp1, qp2), am2, am1, a00, ap1, ap2, C.inv_d2x);
        float p0 = Q.pv0[P & 1], p1 = Q.pv1[P & 1];
        const float rho = Q.rh[P & 1];
        if (X.it > 0) {
            p0 = p0 * X.tzv * txv;
            p1 = p1 * X.tzv * txv;
        }
        if (!X.zb6) {
            const float mzm2 = rmuj[-2], mzm1 = rmuj[-1], mzp1 = rmuj[1], mzp2 = rmuj[2];
            const Brk bkz = brk5(mzm2, mzm1, m00, mzp1, mzp2);
            n1 = d2s(0.f, twice(bkz), ruzj[-2], ruzj[-1], b00, ruzj[1], ruzj[2], C.inv_d2z);
            n1 = d2s(n1, bkx, bm2, bm1, b00, bp1, bp2, C.inv_d2x);
            n0 = d2s(n0, bkz, ruxj[-2], ruxj[-1], a00, ruxj[1], ruxj[2], C.inv_d2z);
            if (!VTI) {
                n0 += md1s(tm2, qm2, tm1, qm1, tp1, qp1, tp2, qp2, C.adx);
                n1 += md1s(rtj[-2], rqj[-2], rtj[-1], rqj[-1], rtj[1], rqj[1], rtj[2], rqj[2], C.adz);
            } else {
                n0 += d1s(tm2, tm1, tp1, tp2, C.sdx);
                n1 += d1s(rqj[-2], rqj[-1], rqj[1], rqj[2], C.sdz);
            }
            n1 += md1s(cm2, mm2, cm1, mm1, cp1, mp1, cp2, mp2, C.adx);
            n0 += md1s(rbxj[-2], mzm2, rbxj[-1], mzm1, rbxj[1], mzp1, rbxj[2], mzp2, C.adz);
            if (src_here) add_sources(Sp->inj, srcrow, e0, e1, gz, n0, n1);
            n0 = C.dt2 * n0 / rho + 2 * a00 - p0;
            n1 = C.dt2 * n1 / rho + 2 * b00 - p1;
        } else if (X.own) {
            n1 = 0.f;
            d2acc(n1, ruzj, 1, rmuj, 1, 2.f, gz, X.nz, C.inv_d2z, C.d2z);
            n1 = d2s(n1, bkx, bm2, bm1, b00, bp1, bp2, C.inv_d2x);
            d2acc(n0, ruxj, 1, rmuj, 1, 1.f, gz, X.nz, C.inv_d2z, C.d2z);
            if (!VTI) {
                n0 += md1s(tm2, qm2, tm1, qm1, tp1, qp1, tp2, qp2, C.adx);
                n1 += md1(rtj, rqj, 1, gz, X.nz, C.adz);
            } else {
                n0 += d1s(tm2, tm1, tp1, tp2, C.sdx);
                n1 += d1(rqj, 1, gz, X.nz, C.dz, C.sdz);
            }
            n1 += md1s(cm2, mm2, cm1, mm1, cp1, mp1, cp2, mp2, C.adx);
            n0 += md1(rbxj, rmuj, 1, gz, X.nz, C.adz);
            if (src_here) add_sources(Sp->inj, srcrow, e0, e1, gz, n0, n1);
            const bool top = gz == 0, bot = gz == X.nz - 1;
            const int bc = top ? C.bc[0] : C.bc[1];
            if ((top || bot) && (bc == 1 || bc == 2)) {
                // esat_neumann / esat_absorbing top or bottom (spatial_operators.hpp:160-727) and
                // esat_Dz (:732-776); x is interior here, so the tangential sums take the interior form
                const float mu = m00;
                const long long mcell = X.mofs + (long long)j * X.mld;
                const float lam = VTI ? M.p0[mcell] : q00;
                const float c13 = VTI ? M.c13[mcell] : lam;
                const float imp_s = 0.5f * sqrtf(mu * rho);
                const float imp_p = 0.5f * sqrtf((lam + 2 * mu) * rho);
                const int in = top ? 1 : -1;
                const float sg = top ? -1.f : 1.f;
                float tsz = 0.f, tsx = 0.f;
                tsz += kC1[0] * (bp1 - bm1);
                tsz += kC1[1] * (bp2 - bm2);
                tsx += kC1[0] * (ap1 - am1);
                tsx += kC1[1] * (ap2 - am2);
                {
                    float t = (sg * mu) * tsz / C.dx + mu * nsum(ruxj, in) / C.dz;
                    if (bc == 2) t = t - imp_s * p0 / C.dt;
                    n0 = n0 - C.sat_z * t;
                }
                {
                    float t = (sg * c13) * tsx / C.dx + (2 * mu) * nsum(ruzj, in) / C.dz;
                    if (bc == 2) t = t - imp_p * p1 / C.dt;
                    n1 = n1 - C.sat_z * t;
                    n1 = n1 - C.nsat_z * lam * ndsum(ruzj, in);
                }
            }
            n0 = C.dt2 * n0 / rho + 2 * a00 - p0;
            n1 = C.dt2 * n1 / rho + 2 * b00 - p1;
            if (top || bot) {
                const int k = top ? j : X.nx + j;
                n0 = n0 / Sp->den[k];
                n1 = n1 / Sp->den[2 * X.nx + 2 * X.nz + k];
            }
        } else {
            n0 = n1 = 0.f;
        }
        n0 = n0 * X.tzv * txv;
        n1 = n1 * X.tzv * txv;
        float *pn = X.u + X.pn_off;
        if (X.own) {
            pn[cell] = n0;
            pn[X.nxz + cell] = n1;
            X.amax = fmaxf(X.amax, fmaxf(fabsf(n0), fabsf(n1)));
            if (X.store) {
                const long long o = (long long)X.slot * Sp->snap_slot + cell;
                snap_store(Sp->snap, o, X.prec, a00, X.sc);
                snap_store(Sp->snap, o + X.nxz, X.prec, b00, X.sc);
            }
        }

        // receivers whose pivot lies on this row: curr rows j-1 .. j+1 are in the rings
        if (X.extract) {
            const int r0 = Sp->ext_roff[X.roff + j - X.xb], r1 = Sp->ext_roff[X.roff + j - X.xb + 1];
            for (int e = r0 + (int)threadIdx.x; e < r1; e += NTH) {
                const ExtEntry &E = Sp->ext[e];
                const float *Rb = sm + (E.comp == 0 ? L::UX : L::UZ);
                const int zi = E.gz0 - (X.z - li);
                float o = 0.f;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const float *row = Rb + ((P + 7 + a) & 7) * RW + zi;
#pragma unroll
                    for (int b = 0; b < 3; b++) o += E.w[a * 3 + b] * row[b];
                }
                Sp->rcv[(long long)X.it * Sp->nrcv + E.row] = o;
            }
        }

        // zero-lag imaging condition (we_op.cpp:505-562, VTI :1478-1557)
        if (GRAD && X.do_grad && X.own) {
            const float *rf0 = sm + L::F0 + R0 * RW + li, *rf1 = sm + L::F1 + R0 * RW + li;
            float fp0 = 0.f, fp1 = 0.f, fm0 = 0.f, fm1 = 0.f;
            if (X.itf + 1 <= X.last) {
                const long long o = (long long)(X.itf + 1) * Sp->snap_slot + cell;
                fp0 = snap_load(Sp->snap, o, X.prec, X.finvp);
                fp1 = snap_load(Sp->snap, o + X.nxz, X.prec, X.finvp);
            }
            if (X.itf > 0) {
                const long long o = (long long)(X.itf - 1) * Sp->snap_slot + cell;
                fm0 = snap_load(Sp->snap, o, X.prec, X.finvm);
                fm1 = snap_load(Sp->snap, o + X.nxz, X.prec, X.finvm);
            }
            float *g0 = Sp->grad + cell, *g1 = g0 + X.nxz, *g2 = g1 + X.nxz;
            float g0v = *g0, g1v = *g1, g2v = *g2;
            const float ax0 = Q.ax[S0], az1 = Q.az[S0], az0 = Q.cz[S0], ax1 = Q.bx[S0];
            const float t0 = d1s(Q.f0[SM2], Q.f0[SM1], Q.f0[SP1], Q.f0[SP2], C.sdx);
            const float t2 = d1s(Q.f1[SM2], Q.f1[SM1], Q.f1[SP1], Q.f1[SP2], C.sdx);
            float t1, t3;
            if (!X.zb6) {
                t1 = d1s(rf1[-2], rf1[-1], rf1[1], rf1[2], C.sdz);
                t3 = d1s(rf0[-2], rf0[-1], rf0[1], rf0[2], C.sdz);
            } else {
                t1 = d1(rf1, 1, gz, X.nz, C.dz, C.sdz);
                t3 = d1(rf0, 1, gz, X.nz, C.dz, C.sdz);
            }
            const float f0 = Q.f0[S0], f1 = Q.f1[S0];
            const float a0 = n0, a1 = n1;
            const float gw = X.gw, dtg = X.dtg;
            float dl, dm;
            if (!VTI) {
                dl = 0.f;
                dm = (az0 + ax1) * (t2 + t3) + 2 * ax0 * t0 + 2 * az1 * t1;
            } else {
                const long long mo = X.mofs + (long long)j * X.mld;
                const float e2 = 1 + 2 * M.eps[mo];
                const float v2 = M.gv2[mo], v3 = M.gv3[mo];
                dl = e2 * ax0 * t0 + az1 * t1 + v2 * (ax0 * t1 + az1 * t0);
                dm = (az0 + ax1) * (t2 + t3) + 2 * e2 * ax0 * t0 + 2 * az1 * t1 + v3 * (ax0 * t1 + az1 * t0);
            }
            if (X.itf > 0 && X.itf < X.last) {
                if (!VTI) g0v = g0v + gw * dtg * (ax0 + az1) * (t0 + t1);
                else g0v = g0v + gw * dtg * dl;
                g1v = g1v + gw * dtg * dm;
                g2v = (float)((double)g2v + X.wdt * (double)(a0 * (fp0 - 2 * f0 + fm0) + a1 * (fp1 - 2 * f1 + fm1)));
            } else if (X.itf == 0) {
                if (!VTI) g0v = (float)((double)g0v + X.wh * (double)(ax0 + az1) * (double)(t0 + t1));
                else g0v = (float)((double)g0v + X.wh * (double)dl);
                g1v = (float)((double)g1v + X.wh * (double)dm);
                g2v = (float)((double)g2v + X.wdt * (double)(a0 * (fp0 - f0) + a1 * (fp1 - f1)));
            } else {
                if (!VTI) g0v = g0v + gw * dtg * (ax0 + az1) * (t0 + t1);
                else g0v = g0v + gw * dtg * dl;
                g1v = g1v + gw * dtg * dm;
                g2v = (float)((double)g2v + X.wdt * (double)(a0 * (-f0 + fm0) + a1 * (-f1 + fm1)));
            }
            *g0 = g0v;
            *g1 = g1v;
            *g2 = g2v;
        }
    }

    // ---- queues and rings: curr row j+5, coefficient and snapshot rows j+3
    Q.ux[SP5] = nux;
    Q.uz[SP5] = nuz;
    sm[L::UX + SP5 * RW + li] = nux;
    sm[L::UZ + SP5 * RW + li] = nuz;
    if (X.hlo || X.hhi) {
        const int hi = X.hlo ? 0 : RW - 2;
        sm[L::UX + SP5 * RW + hi] = h0a;
        sm[L::UX + SP5 * RW + hi + 1] = h0b;
        sm[L::UZ + SP5 * RW + hi] = h1a;
        sm[L::UZ + SP5 * RW + hi + 1] = h1b;
    }
    Q.mu[SP3] = nmu;
    Q.q[SP3] = nq;
    sm[L::MU + RP3 * RW + li] = nmu;
    if (!VTI) sm[L::Q + RP3 * RW + li] = nq;
    if (VTI) {
        Q.vlb[(P + 1) & 1] = nlb;
        Q.vc13[(P + 1) & 1] = nc13;
        Q.vlam[(P + 1) & 1] = nlam;
    }
    if (GRAD) {
        Q.f0[SP3] = nf0;
        Q.f1[SP3] = nf1;
        sm[L::F0 + RP3 * RW + li] = nf0;
        sm[L::F1 + RP3 * RW + li] = nf1;
    }
}

template <bool VTI, bool GRAD, int NTH>
__global__ void __launch_bounds__(NTH, 2)
elastic_march(const ShotDev *__restrict__ shots, const MarchRef *__restrict__ units, ModelDev M, StepConst C, int it,
              int flags, float dtg)
{
    using L = MarchLayout<VTI, GRAD, NTH>;
    const MarchRef U = units[blockIdx.x];
    const ShotDev *__restrict__ Sp = shots + U.shot;
    const int nt = Sp->nt;
    if (it >= nt - 1) return;
    extern __shared__ __align__(16) float smem[];

    const int t = threadIdx.x;
    MarchCtx X;
    X.nx = Sp->nx;
    X.nz = Sp->nz;
    X.ldz = Sp->ldz;
    X.nxz = X.nx * X.ldz;
    X.mld = M.ldz;
    X.xb = U.xb;
    X.xe = U.xe;
    X.z = U.za + t;
    X.li = 2 + t;
    X.zin = X.z >= 0 && X.z < X.nz;
    X.own = X.z >= U.oz0 && X.z < U.oz1;
    X.zb4 = !(X.z >= 4 && X.z < X.nz - 4);
    X.zb6 = !(X.z >= 6 && X.z < X.nz - 6);
    X.hlo = t == 0;
    X.hhi = t == NTH - 1;
    X.hz = X.hlo ? U.za - 2 : U.za + NTH;
    X.tzv = X.zin ? Sp->tz[X.z] : 0.f;
    X.zw0 = U.za + 32 * (t >> 5);
    X.zw1 = X.zw0 + 32;
    X.u = Sp->u[(it + 1) & 1];
    X.pn_off = Sp->u[it & 1] - X.u;
    X.mofs = (long long)Sp->x0 * X.mld + X.z;

    X.it = it;
    X.prec = C.snap_prec;
    X.extract = (flags & F_EXTRACT) != 0;
    X.store = (flags & F_STORE) && (it % C.sub == 0);
    X.slot = it / C.sub;
    X.sc = 1.f;
    if (X.store && X.prec != SNAP_FP32) X.sc = snap_scale(Sp->snap_amax, X.slot);
    X.do_grad = GRAD && (flags & F_GRAD) && ((nt - 1 - (it + 1)) % C.sub == 0);
    X.itf = GRAD ? (nt - 1 - (it + 1)) / C.sub : 0;
    X.last = nt / C.sub;
    X.finv = X.finvp = X.finvm = 1.f;
    X.gw = 1.f;
    X.dtg = dtg;
    X.wdt = X.wh = 0.0;
    if (GRAD && X.do_grad) {
        if (X.prec != SNAP_FP32) {
            X.finv = 1.f / snap_scale(Sp->snap_amax, X.itf);
            if (X.itf + 1 <= X.last) X.finvp = 1.f / snap_scale(Sp->snap_amax, X.itf + 1);
            if (X.itf > 0) X.finvm = 1.f / snap_scale(Sp->snap_amax, X.itf - 1);
        }
        X.gw = Sp->gwt[X.itf];
        X.wdt = (double)X.gw * 1.0 / (double)dtg;
        X.wh = (double)X.gw * 0.5 * (double)dtg;
    }
    X.roff = U.roff;
    X.amax = 0.f;

    MarchQ<GRAD> Q;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        Q.ux[k] = Q.uz[k] = Q.mu[k] = Q.q[k] = Q.t0[k] = Q.cz[k] = 0.f;
        Q.ax[k] = Q.az[k] = Q.bx[k] = Q.f0[k] = Q.f1[k] = 0.f;
    }
    Q.pv0[0] = Q.pv1[0] = Q.rh[0] = Q.pv0[1] = Q.pv1[1] = Q.rh[1] = 0.f;
    Q.vlb[0] = Q.vc13[0] = Q.vlam[0] = Q.vlb[1] = Q.vc13[1] = Q.vlam[1] = 0.f;

    for (int jb = U.xb - 9; jb < U.xe; jb += 8) {
        march_step<VTI, GRAD, NTH, 0>(Q, X, smem, Sp, M, C, jb);
        if (jb + 1 >= U.xe) break;
        march_step<VTI, GRAD, NTH, 1>(Q, X, smem, Sp, M, C, jb + 1);
        if (jb + 2 >= U.xe) break;
        march_step<VTI, GRAD, NTH, 2>(Q, X, smem, Sp, M, C, jb + 2);
        if (jb + 3 >= U.xe) break;
        march_step<VTI, GRAD, NTH, 3>(Q, X, smem, Sp, M, C, jb + 3);
        if (jb + 4 >= U.xe) break;
        march_step<VTI, GRAD, NTH, 4>(Q, X, smem, Sp, M, C, jb + 4);
        if (jb + 5 >= U.xe) break;
        march_step<VTI, GRAD, NTH, 5>(Q, X, smem, Sp, M, C, jb + 5);
        if (jb + 6 >= U.xe) break;
        march_step<VTI, GRAD, NTH, 6>(Q, X, smem, Sp, M, C, jb + 6);
        if (jb + 7 >= U.xe) break;
        march_step<VTI, GRAD, NTH, 7>(Q, X, smem, Sp, M, C, jb + 7);
    }

    if ((flags & F_AMAX) && ((it + 1) % C.sub == 0)) {
        float *red = smem + L::RED;
        const int lane = t & 31, warp = t >> 5;
        float m = X.amax;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        __syncthreads();
        if (lane == 0) red[warp] = m;
        __syncthreads();
        if (t < 32) {
            m = t < NTH / 32 ? red[t] : 0.f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (t == 0 && m > 0.f) atomicMax(Sp->snap_amax + (it + 1) / C.sub, __float_as_uint(m));
        }
    }
}

}  // namespace fwi2d
