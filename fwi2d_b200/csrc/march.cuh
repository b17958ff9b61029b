// x-marching elastic / VTI step kernel for the rows of a shot grid that lie
// clear of the left and right SBP boundary bands (6 <= x < nx-6).
//
// One CTA owns a strip of z (a window of NTH cells, one per thread) and
// marches along x over a run of rows [xb, xe).  Units own cells of
// 6 <= z < nz-6 only, where every stencil takes its interior form, so the
// kernel carries no closure code and its warps stay in step; the boundary
// frame (x or z within 6 cells of an edge) is computed by the tile kernel.  Rows are contiguous in memory
// (z fastest).  Every row a step needs is fetched one step ahead by 1-D bulk
// copies (cp.async.bulk, no multicast) into shared-memory rings, completion
// tracked by a two-stage mbarrier pipeline, so HBM latency overlaps a whole
// row of arithmetic and no register staging is needed.  Along x the stencil
// samples live in per-thread register queues filled from the rings; along z
// they are read from the rings directly.  Everything a step reads from shared
// memory was written at an earlier step, so one barrier per row suffices.
// The arithmetic per cell is the same single-precision sequence as the tile
// kernel's (src/cpp/we_op.cpp:667-871 elastic, :1640-1840 VTI); z-boundary
// cells use the closure forms of sbp.cuh on the ring rows.
//
// Step j (output row j), after the barrier:
//   issue       bulk copies of curr row j+6, coefficient and snapshot rows
//               j+4, and the own-cell rows of row j+1 (prev, rho, gradient,
//               neighbouring snapshots) plus its row record;
//   derivatives ux_x, uz_z, ux_z and T0 / T1 of row j+2, uz_x of row j+1;
//   output      row j: SBP terms, sources, SAT (z edges), leapfrog, taper,
//               receivers, snapshot store or imaging condition;
//   queues      curr row j+5 and coefficient / snapshot rows j+3 (copied at
//               step j-1) enter the register queues.
// The first output row is preceded by 10 steps that only fill the pipeline.
// The step body is unrolled over groups of UNR phases (MARCH_FWD_UNROLL,
// MARCH_GRAD_UNROLL; 2 measured best on B200 for both): register-queue slots
// are compile-time constants within a group and the queues shift down by UNR
// rows once per group.  Unrolling all 8 ring phases removes the shifts but
// overflows the instruction cache.
//
// Shared memory, rows of RB = NTH + 16 floats; cell z of a row buffer sits
// at index z - s0 with s0 = (za - 2) rounded down to a multiple of 8, so that
// every copy starts and ends on a 16-byte boundary (and 16-bit snapshot rows
// on 16-byte boundaries too).  za is even, so a row spans at most NTH + 16
// cells (s0 at most 6 below za - 2, the end at most 6 above za + NTH + 2):
//   ux, uz, mu, q, f0, f1   8-row rings (q: lambda, or (1+2eps)(lambda+2mu) for VTI)
//   t, bx                   4-row rings of T0 (VTI: T1) and uz_x
//   vl, vc, va              4-row rings of the VTI coefficients lbis, c13, lambda
//   own[2][..]              per step: prev, rho, gradient, snapshot rows of row j+1
#pragma once

namespace fwi2d {

// Set (to the row where it happened + 1) when a wait of the marching kernel
// reaches its limit.  After every forward or adjoint pass the engine moves it
// into the plan's status word and clears it (launch_take_timeout); the host
// then returns FWI2D_ERR_TIMEOUT for that pass.
__device__ int g_march_timeout;

// Each per-row wait has two bounds.  Past the first (StepConst::spin polls,
// FWI2D_SPIN_LIMIT) the row is recorded in g_march_timeout and the CTA keeps
// waiting for the same phase, so that no copy is left in flight in its shared
// memory; past the second (MARCH_HARD_LIMIT more polls) the copies are taken
// to be lost and the CTA leaves.
#define MARCH_HARD_LIMIT (1 << 22)

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// 1-D bulk copy global -> shared of `bytes` (a multiple of 16; both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_row(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for a phase of an mbarrier; false when `limit` polls found it
// still incomplete.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, int limit)
{
    for (int k = 0; k < limit; k++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

template <bool VTI, bool GRAD, int NTH>
struct MarchLayout {
    static constexpr int RB = NTH + 16;
    static constexpr int UX = 0, UZ = UX + 8 * RB, MU = UZ + 8 * RB, Q = MU + 8 * RB;
    static constexpr int F0 = Q + 8 * RB, F1 = F0 + (GRAD ? 8 : 0) * RB;
    static constexpr int T = F1 + (GRAD ? 8 : 0) * RB, BX = T + 4 * RB;
    static constexpr int VL = BX + 4 * RB, VC = VL + (VTI ? 4 : 0) * RB, VA = VC + (VTI ? 4 : 0) * RB;
    // own-cell rows of one step: prev ux, prev uz, rho, g0, g1, g2, fp0, fp1, fm0, fm1, eps, v2, v3
    static constexpr int NOWN = 3 + (GRAD ? 7 : 0) + (VTI && GRAD ? 3 : 0);
    static constexpr int OWN = VA + (VTI ? 4 : 0) * RB;
    static constexpr int ROWREC = OWN + 2 * NOWN * RB;    // 2 x 8 ints
    static constexpr int RED = ROWREC + 16;
    static constexpr int MBAR = RED + 32;                 // 2 x u64, 8-byte aligned (MBAR even)
    static constexpr int FLOATS = MBAR + 4;
    static_assert(RB % 8 == 0, "row buffers must keep 32-byte alignment");
    static_assert(MBAR % 2 == 0, "mbarrier alignment");
};

enum OwnRow { O_PV0 = 0, O_PV1, O_RHO, O_G0, O_G1, O_G2, O_FP0, O_FP1, O_FM0, O_FM1, O_EPS, O_V2, O_V3 };

// Per-thread state that stays fixed during one launch.
struct MarchCtx {
    float *u;                 // curr base (component stride nxz); prev/next at u + pn_off
    long long pn_off;
    long long mofs;           // model offset of the shot's first column
    int ldz, mld, nx, nz, nxz;
    int xb, xe, z, li, s0, s0c, s1c;
    bool zin, own;
    float tzv;
    bool extract, store, do_grad, has_fp, has_fm;
    int it, itf, last, prec, slot;
    float sc, finv, finvp, finvm, dtg, gw;
    double wdt, wh;
    int roff, zw0, zw1;
    float amax;
    const float *srcrow;      // this time sample's injection row
    void *snap;
    long long slot_elems;
    float *grad;
    unsigned ph[2];           // mbarrier phase parity per stage
    int spin;                 // poll limit of the per-step wait before the row is reported
};

// Register queues along x.  UNR = 8: ring of 8 slots, row j+d of phase PH at
// (PH + d) & 7, nothing moves.  UNR < 8: row j+d of phase PH at d + 2 + PH
// (QL = 7 + UNR slots), and the queues shift down by UNR after the last phase.
template <bool GRAD, int UNR>
struct MarchQ {
    static constexpr int QL = UNR == 8 ? 8 : 7 + UNR;
    float ux[QL], uz[QL], mu[QL], q[QL], t0[QL], cz[QL];
    float ax[QL], az[QL], bx[QL], f0[QL], f1[QL];
};

// sample of a snapshot row buffer (fp32, or 16-bit scaled by inv)
__device__ __forceinline__ float srow(const float *buf, int idx, int prec, float inv)
{
    if (prec == SNAP_FP32) return buf[idx];
    if (prec == SNAP_BF16) return __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(buf)[idx]) * inv;
    return __half2float(reinterpret_cast<const __half *>(buf)[idx]) * inv;
}

// Rare per-row paths (rows holding a source or a receiver pivot) are kept
// out of line, so that the unrolled step bodies stay small.
#ifndef MARCH_RARE_INLINE
#define MARCH_RARE __noinline__
#else
#define MARCH_RARE __forceinline__
#endif
__device__ MARCH_RARE void add_sources(const InjEntry *__restrict__ inj, const float *__restrict__ srcrow, int e0,
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

// Receivers of one row: entries [r0, r1), 3x3 weights over the curr rows
// j-1 .. j+1 of the rings (slots P+7, P, P+1).
__device__ MARCH_RARE void march_extract(const ExtEntry *__restrict__ ext, float *__restrict__ rcvrow,
                                           const float *rux, const float *ruz, int RB, int P, int s0, int r0, int r1,
                                           int nth)
{
    for (int e = r0 + (int)threadIdx.x; e < r1; e += nth) {
        const ExtEntry &E = ext[e];
        const float *Rb = E.comp == 0 ? rux : ruz;
        const int zi = E.gz0 - s0;
        float o = 0.f;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float *row = Rb + ((P + 7 + a) & 7) * RB + zi;
#pragma unroll
            for (int b = 0; b < 3; b++) o += E.w[a * 3 + b] * row[b];
        }
        rcvrow[E.row] = o;
    }
}

// Bulk copies issued at step j (by thread 0) for consumption at step j+1.
template <bool VTI, bool GRAD, int NTH>
__device__ __forceinline__ void march_issue(const MarchCtx &X, float *sm, const ShotDev &S, const ModelDev &M, int j,
                                            int P)
{
    using L = MarchLayout<VTI, GRAD, NTH>;
    constexpr int RB = L::RB;
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm + L::MBAR) + ((P + 1) & 1);
    const int n = X.s1c - X.s0c, dofs = X.s0c - X.s0;
    const unsigned nf = 4u * n, nh = (X.prec == SNAP_FP32 ? 4u : 2u) * n;
    const bool own_next = j + 1 >= X.xb;
    unsigned bytes = 2 * nf + (VTI ? 5 : 2) * nf;
    if (GRAD && X.do_grad) bytes += 2 * nh;
    if (own_next) {
        bytes += 3 * nf + 32;
        if (GRAD && X.do_grad) {
            bytes += 3 * nf + (X.has_fp ? 2 * nh : 0) + (X.has_fm ? 2 * nh : 0);
            if (VTI) bytes += 3 * nf;
        }
    }
    mbar_expect_tx(bar, bytes);
    // curr row j+6
    const long long c6 = (long long)(j + 6) * X.ldz + X.s0c;
    bulk_row(sm + L::UX + ((P + 6) & 7) * RB + dofs, X.u + c6, nf, bar);
    bulk_row(sm + L::UZ + ((P + 6) & 7) * RB + dofs, X.u + X.nxz + c6, nf, bar);
    // coefficient rows j+4
    const long long m4 = X.mofs + (long long)(j + 4) * X.mld + X.s0c;
    bulk_row(sm + L::MU + ((P + 4) & 7) * RB + dofs, M.p1 + m4, nf, bar);
    bulk_row(sm + L::Q + ((P + 4) & 7) * RB + dofs, (VTI ? M.fxx : M.p0) + m4, nf, bar);
    if (VTI) {
        bulk_row(sm + L::VL + ((P + 4) & 3) * RB + dofs, M.lbis + m4, nf, bar);
        bulk_row(sm + L::VC + ((P + 4) & 3) * RB + dofs, M.c13 + m4, nf, bar);
        bulk_row(sm + L::VA + ((P + 4) & 3) * RB + dofs, M.p0 + m4, nf, bar);
    }
    const int esz = X.prec == SNAP_FP32 ? 4 : 2;
    const char *snap = (const char *)S.snap;
    if (GRAD && X.do_grad) {
        const long long so = (long long)X.itf * S.snap_slot + (long long)(j + 4) * X.ldz + X.s0c;
        bulk_row((char *)(sm + L::F0 + ((P + 4) & 7) * RB) + dofs * esz, snap + so * esz, nh, bar);
        bulk_row((char *)(sm + L::F1 + ((P + 4) & 7) * RB) + dofs * esz, snap + (so + X.nxz) * esz, nh, bar);
    }
    if (own_next) {
        float *own = sm + L::OWN + ((P + 1) & 1) * L::NOWN * RB;
        const long long o1 = (long long)(j + 1) * X.ldz + X.s0c;
        const float *pn = X.u + X.pn_off;
        bulk_row(own + O_PV0 * RB + dofs, pn + o1, nf, bar);
        bulk_row(own + O_PV1 * RB + dofs, pn + X.nxz + o1, nf, bar);
        const long long m1 = X.mofs + (long long)(j + 1) * X.mld + X.s0c;
        bulk_row(own + O_RHO * RB + dofs, M.p2 + m1, nf, bar);
        bulk_row(sm + L::ROWREC + ((P + 1) & 1) * 8, S.mrow + X.roff + (j + 1 - X.xb), 32, bar);
        if (GRAD && X.do_grad) {
            bulk_row(own + O_G0 * RB + dofs, S.grad + o1, nf, bar);
            bulk_row(own + O_G1 * RB + dofs, S.grad + X.nxz + o1, nf, bar);
            bulk_row(own + O_G2 * RB + dofs, S.grad + 2 * (long long)X.nxz + o1, nf, bar);
            if (X.has_fp) {
                const long long o = (long long)(X.itf + 1) * S.snap_slot + o1;
                bulk_row((char *)(own + O_FP0 * RB) + dofs * esz, snap + o * esz, nh, bar);
                bulk_row((char *)(own + O_FP1 * RB) + dofs * esz, snap + (o + X.nxz) * esz, nh, bar);
            }
            if (X.has_fm) {
                const long long o = (long long)(X.itf - 1) * S.snap_slot + o1;
                bulk_row((char *)(own + O_FM0 * RB) + dofs * esz, snap + o * esz, nh, bar);
                bulk_row((char *)(own + O_FM1 * RB) + dofs * esz, snap + (o + X.nxz) * esz, nh, bar);
            }
            if (VTI) {
                bulk_row(own + O_EPS * RB + dofs, M.eps + m1, nf, bar);
                bulk_row(own + O_V2 * RB + dofs, M.gv2 + m1, nf, bar);
                bulk_row(own + O_V3 * RB + dofs, M.gv3 + m1, nf, bar);
            }
        }
    }
}

// Returns false when the CTA must stop (a wait reached its second bound).
// Register queues of 8 rows.  Unrolled (PH >= 0): row j+d sits at index
// (PH + d) & 7.  Rolled (PH < 0): row j+d sits at index d + 2 and the queues
// shift by one row at the end of each step.
template <bool GRAD, int UNR>
__device__ __forceinline__ void shift_queues(MarchQ<GRAD, UNR> &Q)
{
#pragma unroll
    for (int k = 0; k < 7; k++) {
        Q.ux[k] = Q.ux[k + UNR];
        Q.uz[k] = Q.uz[k + UNR];
        Q.mu[k] = Q.mu[k + UNR];
        Q.q[k] = Q.q[k + UNR];
        Q.t0[k] = Q.t0[k + UNR];
        Q.cz[k] = Q.cz[k + UNR];
        if (GRAD) {
            Q.ax[k] = Q.ax[k + UNR];
            Q.az[k] = Q.az[k + UNR];
            Q.bx[k] = Q.bx[k + UNR];
            Q.f0[k] = Q.f0[k + UNR];
            Q.f1[k] = Q.f1[k + UNR];
        }
    }
}

template <bool VTI, bool GRAD, int NTH, int PH, int UNR>
__device__ __forceinline__ bool march_step(MarchQ<GRAD, UNR> &Q, MarchCtx &X, float *sm, const ShotDev &S,
                                           const ModelDev &M, const StepConst &C, int j, int j0)
{
    using L = MarchLayout<VTI, GRAD, NTH>;
    constexpr int RB = L::RB;
    constexpr bool RING = UNR == 8;   // queue slots rotate with the 8 phases
    const int P = RING ? PH : ((j - j0) & 7);
#define MQ(d) (RING ? ((PH + (d) + 8) & 7) : (PH + (d) + 2))
    constexpr int QM2 = MQ(-2), QM1 = MQ(-1), Q00 = MQ(0), QP1 = MQ(1), QP2 = MQ(2), QP3 = MQ(3), QP4 = MQ(4);
    // register-queue slots of the rows arriving at the end of this step (j+5, j+3)
    constexpr int QN5 = MQ(5), QN3 = MQ(3);
#undef MQ
    // ring slots of rows j+d (8-row rings) and (4-row rings)
    const int S0 = P, SP2 = (P + 2) & 7, SP3 = (P + 3) & 7, SP5 = (P + 5) & 7;
    const int R0 = P & 3, RP1 = (P + 1) & 3, RP2 = (P + 2) & 3;
    const int li = X.li;
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(sm + L::MBAR);

    // ---- wait for the copies issued at the previous step, then the step barrier
    bool lost = false;
    if (j > j0) {
        const unsigned par = X.ph[P & 1];
        if (!mbar_wait(bars + (P & 1), par, X.spin)) {
            // first bound reached: report the row, keep waiting for the phase
            if (g_march_timeout == 0) atomicCAS(&g_march_timeout, 0, j + 1);
            lost = !mbar_wait(bars + (P & 1), par, MARCH_HARD_LIMIT);
        }
        X.ph[P & 1] ^= 1u;
    }
    if (__syncthreads_or(lost)) {
        if (threadIdx.x == 0) atomicCAS(&g_march_timeout, 0, j + 1);
        return false;
    }
    if (threadIdx.x == 0 && j + 1 < X.xe) march_issue<VTI, GRAD, NTH>(X, sm, S, M, j, P);

    // ---- derivatives of row j+2 (its curr ring row arrived three steps ago)
    {
        const float *ux2 = sm + L::UX + SP2 * RB + li, *uz2 = sm + L::UZ + SP2 * RB + li;
        const float uxx = d1s(Q.ux[Q00], Q.ux[QP1], Q.ux[QP3], Q.ux[QP4], C.sdx);
        const float uzz = d1s(uz2[-2], uz2[-1], uz2[1], uz2[2], C.sdz);
        const float czz = d1s(ux2[-2], ux2[-1], ux2[1], ux2[2], C.sdz);
        float t0;
        if (!VTI) {
            t0 = uxx + uzz;
            sm[L::T + RP2 * RB + li] = t0;
        } else {
            const float vlb = sm[L::VL + RP2 * RB + li], vc13 = sm[L::VC + RP2 * RB + li];
            const float vlam = sm[L::VA + RP2 * RB + li];
            t0 = vlb * uxx + vc13 * uzz;
            sm[L::T + RP2 * RB + li] = vlam * uzz + vc13 * uxx;
        }
        Q.t0[QP2] = t0;
        Q.cz[QP2] = czz;
        if (GRAD) {
            Q.ax[QP2] = uxx;
            Q.az[QP2] = uzz;
        }
    }
    // uz_x of row j+1 from rows j-1 .. j+3
    {
        const float bx = d1s(Q.uz[QM1], Q.uz[Q00], Q.uz[QP2], Q.uz[QP3], C.sdx);
        sm[L::BX + RP1 * RB + li] = bx;
        if (GRAD) Q.bx[QP1] = bx;
    }

    // ---- output row j
    if (j >= X.xb) {
        const float *ruxj = sm + L::UX + S0 * RB + li, *ruzj = sm + L::UZ + S0 * RB + li;
        const float *rmuj = sm + L::MU + S0 * RB + li, *rqj = sm + L::Q + S0 * RB + li;
        const float *rtj = sm + L::T + R0 * RB + li, *rbxj = sm + L::BX + R0 * RB + li;
        const float *own = sm + L::OWN + (P & 1) * L::NOWN * RB + li;
        const MarchRow R = *reinterpret_cast<const MarchRow *>(sm + L::ROWREC + (P & 1) * 8);
        const float am2 = Q.ux[QM2], am1 = Q.ux[QM1], a00 = Q.ux[Q00], ap1 = Q.ux[QP1], ap2 = Q.ux[QP2];
        const float bm2 = Q.uz[QM2], bm1 = Q.uz[QM1], b00 = Q.uz[Q00], bp1 = Q.uz[QP1], bp2 = Q.uz[QP2];
        const float mm2 = Q.mu[QM2], mm1 = Q.mu[QM1], m00 = Q.mu[Q00], mp1 = Q.mu[QP1], mp2 = Q.mu[QP2];
        const float qm2 = Q.q[QM2], qm1 = Q.q[QM1], q00 = Q.q[Q00], qp1 = Q.q[QP1], qp2 = Q.q[QP2];
        const float tm2 = Q.t0[QM2], tm1 = Q.t0[QM1], tp1 = Q.t0[QP1], tp2 = Q.t0[QP2];
        const float cm2 = Q.cz[QM2], cm1 = Q.cz[QM1], cp1 = Q.cz[QP1], cp2 = Q.cz[QP2];
        const float txv = R.tx;
        const long long cell = (long long)j * X.ldz + X.z;
        const int gz = X.z;
        const bool src_here = R.e0 < R.e1 && R.zlo < X.zw1 && R.zhi >= X.zw0;
        const float *srcrow = X.srcrow;

        const Brk bkx = brk5(mm2, mm1, m00, mp1, mp2);
        float n0, n1;
        if (!VTI) n0 = d2s(0.f, twice(bkx), am2, am1, a00, ap1, ap2, C.inv_d2x);
        else n0 = d2s(0.f, brk5(qm2, qm1, q00, qp1, qp2), am2, am1, a00, ap1, ap2, C.inv_d2x);
        float p0 = own[O_PV0 * RB], p1 = own[O_PV1 * RB];
        const float rho = own[O_RHO * RB];
        if (X.it > 0) {
            p0 = p0 * X.tzv * txv;
            p1 = p1 * X.tzv * txv;
        }
        {
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
                n1 += d1s(rtj[-2], rtj[-1], rtj[1], rtj[2], C.sdz);
            }
            n1 += md1s(cm2, mm2, cm1, mm1, cp1, mp1, cp2, mp2, C.adx);
            n0 += md1s(rbxj[-2], mzm2, rbxj[-1], mzm1, rbxj[1], mzp1, rbxj[2], mzp2, C.adz);
            if (src_here) add_sources(S.inj, srcrow, R.e0, R.e1, gz, n0, n1);
            n0 = C.dt2 * n0 / rho + 2 * a00 - p0;
            n1 = C.dt2 * n1 / rho + 2 * b00 - p1;
        }
        n0 = n0 * X.tzv * txv;
        n1 = n1 * X.tzv * txv;
        float *pn = X.u + X.pn_off;
        if (X.own) {
            pn[cell] = n0;
            pn[X.nxz + cell] = n1;
            X.amax = fmaxf(X.amax, fmaxf(fabsf(n0), fabsf(n1)));
            if (X.store) {
                const long long o = (long long)X.slot * X.slot_elems + cell;
                snap_store(X.snap, o, X.prec, a00, X.sc);
                snap_store(X.snap, o + X.nxz, X.prec, b00, X.sc);
            }
        }

        // receivers whose pivot lies on this row: curr rows j-1 .. j+1 are in the rings
        if (X.extract && R.r0 < R.r1)
            march_extract(S.ext, S.rcv + (long long)X.it * S.nrcv, sm + L::UX, sm + L::UZ, RB, P, X.s0, R.r0, R.r1,
                          NTH);

        // zero-lag imaging condition (we_op.cpp:505-562, VTI :1478-1557)
        if (GRAD && X.do_grad && X.own) {
            const float *rf0 = sm + L::F0 + S0 * RB, *rf1 = sm + L::F1 + S0 * RB;
            float fp0 = 0.f, fp1 = 0.f, fm0 = 0.f, fm1 = 0.f;
            if (X.has_fp) {
                fp0 = srow(own - li + O_FP0 * RB, li, X.prec, X.finvp);
                fp1 = srow(own - li + O_FP1 * RB, li, X.prec, X.finvp);
            }
            if (X.has_fm) {
                fm0 = srow(own - li + O_FM0 * RB, li, X.prec, X.finvm);
                fm1 = srow(own - li + O_FM1 * RB, li, X.prec, X.finvm);
            }
            float g0v = own[O_G0 * RB], g1v = own[O_G1 * RB], g2v = own[O_G2 * RB];
            const float ax0 = Q.ax[Q00], az1 = Q.az[Q00], az0 = Q.cz[Q00], ax1 = Q.bx[Q00];
            const float t0 = d1s(Q.f0[QM2], Q.f0[QM1], Q.f0[QP1], Q.f0[QP2], C.sdx);
            const float t2 = d1s(Q.f1[QM2], Q.f1[QM1], Q.f1[QP1], Q.f1[QP2], C.sdx);
            float t1, t3;
            if (X.prec == SNAP_FP32) {
                t1 = d1s(rf1[li - 2], rf1[li - 1], rf1[li + 1], rf1[li + 2], C.sdz);
                t3 = d1s(rf0[li - 2], rf0[li - 1], rf0[li + 1], rf0[li + 2], C.sdz);
            } else {
                t1 = d1s(srow(rf1, li - 2, X.prec, X.finv), srow(rf1, li - 1, X.prec, X.finv),
                         srow(rf1, li + 1, X.prec, X.finv), srow(rf1, li + 2, X.prec, X.finv), C.sdz);
                t3 = d1s(srow(rf0, li - 2, X.prec, X.finv), srow(rf0, li - 1, X.prec, X.finv),
                         srow(rf0, li + 1, X.prec, X.finv), srow(rf0, li + 2, X.prec, X.finv), C.sdz);
            }
            const float f0 = Q.f0[Q00], f1 = Q.f1[Q00];
            const float a0 = n0, a1 = n1;
            const float gw = X.gw, dtg = X.dtg;
            float dl, dm;
            if (!VTI) {
                dl = 0.f;
                dm = (az0 + ax1) * (t2 + t3) + 2 * ax0 * t0 + 2 * az1 * t1;
            } else {
                const float e2 = 1 + 2 * own[O_EPS * RB];
                const float v2 = own[O_V2 * RB], v3 = own[O_V3 * RB];
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
            float *g0 = X.grad + cell;
            g0[0] = g0v;
            g0[X.nxz] = g1v;
            g0[2 * (long long)X.nxz] = g2v;
        }
    }

    // ---- queues: curr row j+5 and coefficient / snapshot rows j+3 (copied
    // at step j-1) take the slots the next step reads as j+4 and j+2
    if (j > j0) {
        Q.ux[QN5] = sm[L::UX + SP5 * RB + li];
        Q.uz[QN5] = sm[L::UZ + SP5 * RB + li];
        Q.mu[QN3] = sm[L::MU + SP3 * RB + li];
        Q.q[QN3] = sm[L::Q + SP3 * RB + li];
        if (GRAD && X.do_grad) {
            Q.f0[QN3] = srow(sm + L::F0 + SP3 * RB, li, X.prec, X.finv);
            Q.f1[QN3] = srow(sm + L::F1 + SP3 * RB, li, X.prec, X.finv);
        }
    }
    if (!RING && PH == UNR - 1) shift_queues<GRAD, UNR>(Q);
    return true;
}

// Phases per unrolled group (1, 2, 4 or 8) of the imaging-condition and of the
// forward kernels: fewer phases keep the step body within the instruction
// cache at the cost of shifting the register queues every group.
#ifndef MARCH_GRAD_UNROLL
#define MARCH_GRAD_UNROLL 2
#endif
#ifndef MARCH_FWD_UNROLL
#define MARCH_FWD_UNROLL 2
#endif

#ifndef MARCH_FWD_MIN_BLOCKS
#define MARCH_FWD_MIN_BLOCKS 3
#endif
#ifndef MARCH_GRAD_MIN_BLOCKS
#define MARCH_GRAD_MIN_BLOCKS 2
#endif
template <bool VTI, bool GRAD, int NTH>
__global__ void __launch_bounds__(NTH, NTH > 224 ? 2 : (GRAD ? MARCH_GRAD_MIN_BLOCKS : MARCH_FWD_MIN_BLOCKS))
elastic_march(const ShotDev *__restrict__ shots, const MarchRef *__restrict__ units, ModelDev M, StepConst C, int it,
              int flags, float dtg)
{
    using L = MarchLayout<VTI, GRAD, NTH>;
    __shared__ ShotDev S;
    extern __shared__ __align__(16) float smem[];
    const MarchRef U = units[blockIdx.x];
    const int t = threadIdx.x;
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem + L::MBAR);
    if (t == 0) {
        S = shots[U.shot];
        mbar_init(bars, 1);
        mbar_init(bars + 1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int nt = S.nt;
    if (it >= nt - 1) return;

    MarchCtx X;
    X.nx = S.nx;
    X.nz = S.nz;
    X.ldz = S.ldz;
    X.nxz = X.nx * X.ldz;
    X.mld = M.ldz;
    X.xb = U.xb;
    X.xe = U.xe;
    X.z = U.za + t;
    X.s0 = (U.za - 2) & ~7;
    X.s0c = X.s0 > 0 ? X.s0 : 0;
    const int s1 = (U.za + NTH + 2 + 7) & ~7;
    X.s1c = s1 < X.ldz ? s1 : X.ldz;
    X.li = X.z - X.s0;
    X.zin = X.z >= 0 && X.z < X.nz;
    X.own = X.z >= U.oz0 && X.z < U.oz1;
    X.tzv = X.zin ? S.tz[X.z] : 0.f;
    X.zw0 = U.za + 32 * (t >> 5);
    X.zw1 = X.zw0 + 32;
    X.u = S.u[(it + 1) & 1];
    X.pn_off = S.u[it & 1] - X.u;
    X.mofs = (long long)S.x0 * X.mld;

    X.it = it;
    X.prec = C.snap_prec;
    X.extract = (flags & F_EXTRACT) != 0;
    X.store = (flags & F_STORE) && (it % C.sub == 0);
    X.slot = it / C.sub;
    X.sc = 1.f;
    if (X.store && X.prec != SNAP_FP32) X.sc = snap_scale(S.snap_amax, X.slot);
    X.do_grad = GRAD && (flags & F_GRAD) && ((nt - 1 - (it + 1)) % C.sub == 0);
    X.itf = GRAD ? (nt - 1 - (it + 1)) / C.sub : 0;
    X.last = nt / C.sub;
    X.has_fp = X.itf + 1 <= X.last;
    X.has_fm = X.itf > 0;
    X.finv = X.finvp = X.finvm = 1.f;
    X.gw = 1.f;
    X.dtg = dtg;
    X.wdt = X.wh = 0.0;
    if (GRAD && X.do_grad) {
        if (X.prec != SNAP_FP32) {
            X.finv = 1.f / snap_scale(S.snap_amax, X.itf);
            if (X.has_fp) X.finvp = 1.f / snap_scale(S.snap_amax, X.itf + 1);
            if (X.has_fm) X.finvm = 1.f / snap_scale(S.snap_amax, X.itf - 1);
        }
        X.gw = S.gwt[X.itf];
        X.wdt = (double)X.gw * 1.0 / (double)dtg;
        X.wh = (double)X.gw * 0.5 * (double)dtg;
    }
    X.roff = U.roff;
    X.amax = 0.f;
    X.srcrow = S.src + (long long)it * S.nsrc;
    X.snap = S.snap;
    X.slot_elems = S.snap_slot;
    X.grad = S.grad;
    X.ph[0] = X.ph[1] = 0u;
    X.spin = C.spin;

    constexpr int UNR = GRAD ? MARCH_GRAD_UNROLL : MARCH_FWD_UNROLL;
    MarchQ<GRAD, UNR> Q;
#pragma unroll
    for (int k = 0; k < MarchQ<GRAD, UNR>::QL; k++) {
        Q.ux[k] = Q.uz[k] = Q.mu[k] = Q.q[k] = Q.t0[k] = Q.cz[k] = 0.f;
        Q.ax[k] = Q.az[k] = Q.bx[k] = Q.f0[k] = Q.f1[k] = 0.f;
    }

    const int j0 = U.xb - 10;
    bool ok = true;
    for (int jb = j0; jb < U.xe; jb += UNR) {
#define MARCH_PHASE(k)                                                                              \
    if (k < UNR) {                                                                                  \
        if (jb + k >= U.xe) break;                                                                  \
        ok = march_step<VTI, GRAD, NTH, (k < UNR ? k : 0), UNR>(Q, X, smem, S, M, C, jb + k, j0);   \
        if (!ok) break;                                                                             \
    }
        MARCH_PHASE(0) MARCH_PHASE(1) MARCH_PHASE(2) MARCH_PHASE(3)
        MARCH_PHASE(4) MARCH_PHASE(5) MARCH_PHASE(6) MARCH_PHASE(7)
#undef MARCH_PHASE
    }
    if (!ok) return;   // a wait reached its second bound: the copies did not arrive

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
            if (t == 0 && m > 0.f) atomicMax(S.snap_amax + (it + 1) / C.sub, __float_as_uint(m));
        }
    }
}

}  // namespace fwi2d
