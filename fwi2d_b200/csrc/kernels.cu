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
#include "launch.h"

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


// 4-byte asynchronous copy global -> shared (cp.async, no register staging)
__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The 4-byte word holding snapshot sample idx: the sample itself (FP32), or
// the pair of 16-bit samples that contains it.
__device__ __forceinline__ const void *snap_word(const void *base, long long idx, int prec)
{
    if (prec == SNAP_FP32) return (const float *)base + idx;
    return (const unsigned short *)base + (idx & ~1LL);
}
// snap_load on a word copied by snap_word
__device__ __forceinline__ float snap_from_word(float w, long long idx, int prec, float inv)
{
    if (prec == SNAP_FP32) return w;
    const unsigned u = __float_as_uint(w);
    const unsigned short h = (unsigned short)((idx & 1) ? (u >> 16) : (u & 0xffffu));
    if (prec == SNAP_BF16) return __bfloat162float(__ushort_as_bfloat16(h)) * inv;
    return __half2float(__ushort_as_half(h)) * inv;
}

// Per-thread slots of the scalar interior path: the operands of the thread's
// own cell, copied into shared memory at the start of the step.
enum OwnSlot { OS_P0 = 0, OS_P1, OS_RHO, OS_FP0, OS_FP1, OS_FM0, OS_FM1, OS_G0, OS_G1, OS_G2, OS_EPS, OS_V2, OS_V3 };
template <bool VTI, bool GRAD>
constexpr int own_slots() { return GRAD ? (VTI ? 13 : 10) : 3; }

// ---------------------------------------------------------------------------
// Elastic isotropic / VTI step.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 ld2(const float *base, int idx)
{
    return *reinterpret_cast<const float2 *>(base + idx);
}
__device__ __forceinline__ float pick(const float2 v, int c) { return c ? v.y : v.x; }
// the five z-samples around cell c of a z-pair from the pairs (z-2,z-1) (z,z+1) (z+2,z+3)
struct Z5 {
    float m2, m1, c, p1, p2;
};
__device__ __forceinline__ Z5 zsel(const float2 lo, const float2 mid, const float2 hi, int c)
{
    Z5 r;
    if (c == 0) {
        r.m2 = lo.x; r.m1 = lo.y; r.c = mid.x; r.p1 = mid.y; r.p2 = hi.x;
    } else {
        r.m2 = lo.y; r.m1 = mid.x; r.c = mid.y; r.p1 = hi.x; r.p2 = hi.y;
    }
    return r;
}

// Two-sample snapshot loads for the lean path (even index).
__device__ __forceinline__ float2 snap_load2(const void *base, long long idx, int prec, float inv)
{
    if (prec == SNAP_FP32) return *reinterpret_cast<const float2 *>((const float *)base + idx);
    if (prec == SNAP_BF16) {
        const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>((const __nv_bfloat16 *)base + idx));
        return make_float2(v.x * inv, v.y * inv);
    }
    const float2 v = __half22float2(*reinterpret_cast<const __half2 *>((const __half *)base + idx));
    return make_float2(v.x * inv, v.y * inv);
}

// ---------------------------------------------------------------------------
// Elastic isotropic / VTI step.  Tiles are TZ = 32*RZ (z) by TX (x) cells on
// 32*TX threads.  Tiles whose every evaluated point is clear of the SBP
// boundary bands take the lean path (RZ == 2): each thread owns a z-pair of
// one column, loads are vectorised, all offsets are compile-time and the
// pair is evaluated with packed FP32x2 arithmetic (sbp.cuh add2 / mul2:
// FADD2 / FMUL2, each lane rounded as the scalar operation); a lane whose
// cell the tile does not own is computed but not stored.  Other tiles take
// the general path, which carries the boundary closures, the SAT terms and
// the absorbing scaling.  All paths perform the same arithmetic.
// ---------------------------------------------------------------------------
// AE: the elastic part of the acoustic-elastic propagator
// (nl_we_op_ae::propagate, we_op.cpp:2137-2577): isotropic, version-1 split of
// the lambda terms (Dx(lambda ux_x) + Dx(lambda uz_z), Dz(lambda uz_z) +
// Dz(lambda ux_x)), the top edge is the fluid interface (traction-free SAT,
// applied after the other sides), and the interface row of uz is left
// untapered, with its prev saved in halo_save, for ae_couple.  No imaging
// term at snapshot 0.  Windows clear of the bands take the scalar interior
// path with the same split; the others, the interface row among them, the
// general path.
// Resident CTAs per SM asked of the compiler for the 32 x 8 tiles (a cap of
// 51 registers a thread): the kernel is latency-bound, and five resident
// tiles instead of four cut its single-shot time by about 20 % on B200.
#ifndef TILE_MIN_BLOCKS
#define TILE_MIN_BLOCKS 5
#endif
// CORE: the interior-only instantiation for the interior windows of framed
// plans, which the engine places clear of the boundary bands (owned cells at
// least 6 cells from every edge, window and halo inside the grid, even first
// row); it compiles the lean paths only, without the general path's
// registers.
#ifndef CORE_MIN_BLOCKS
#define CORE_MIN_BLOCKS 2
#endif
// resident CTAs per SM asked for the scalar (RZ = 1) 32 x 8 interior windows:
// six (40 registers) instead of five took batched gradients 4-5 % faster on
// B200 and left the single shot unchanged
#ifndef CORE1_MIN_BLOCKS
#define CORE1_MIN_BLOCKS 6
#endif
// resident CTAs per SM asked for the scalar (RZ = 1) 32 x 16 interior windows:
// two (64 registers).  Three (40 registers) took the single-shot adjoint 8 %
// slower on B200, and on 8-shot plans the 32 x 8 windows stayed ahead.
#ifndef CORE16_MIN_BLOCKS
#define CORE16_MIN_BLOCKS 2
#endif
// BAND: the instantiation for the full-height x-band windows of framed and
// marching plans with many band windows (one thread per cell; plans with few
// take elastic_xband, which splits a cell's components over two warps).  It
// runs on few CTAs beside the interior, so it is compiled without the
// occupancy bound (no register spills) and, in
// the imaging condition, loads its snapshot and gradient operands before the
// stencil arithmetic so that their latency overlaps it.
template <bool VTI, int RZ, int TX, bool GRAD, bool AE, bool CORE = false, bool BAND = false>
__global__ void __launch_bounds__(32 * TX, BAND ? 1
                                               : (TX == 8 ? (RZ == 1 ? (CORE ? CORE1_MIN_BLOCKS : TILE_MIN_BLOCKS)
                                                                     : (CORE ? CORE_MIN_BLOCKS : 1))
                                                          : (CORE && RZ == 1 ? CORE16_MIN_BLOCKS : 1)))
elastic_step(const ShotDev *__restrict__ shots, const TileRef *__restrict__ tiles, ModelDev M, StepConst C,
             int it, int flags, float dtg)
{
    constexpr int TZ = 32 * RZ;
    constexpr int UZ = TZ + 8, UX = TX + 8;
    constexpr int WZ = TZ + 4, WX = TX + 4;
    constexpr int NT = 32 * TX;
    // dynamic shared memory: see elastic_smem_bytes()
    extern __shared__ __align__(16) float smem[];
    float *U0 = smem;
    float *U1 = U0 + UX * UZ;
    float *MU = U1 + UX * UZ;
    float *Q = MU + WX * WZ;       // lambda (iso) or (1+2eps)2mu (VTI)
    float *T0 = Q + WX * WZ;       // iso: ux_x+uz_z ; VTI: tmp_x
    float *BX = T0 + WX * WZ;      // uz_x
    float *CZ = BX + WX * WZ;      // ux_z
    float *T1 = CZ + WX * WZ;      // VTI: tmp_z
    float *F0 = T1 + ((VTI || AE) ? WX * WZ : 0);
    float *F1 = F0 + (GRAD ? WX * WZ : 0);
    float *red = F1 + (GRAD ? WX * WZ : 0);
    float *OWN = red + TX;         // scalar interior path: own_slots() x NT per-thread slots

    const TileRef tr = tiles[blockIdx.x];
    const ShotDev *__restrict__ Sp = shots + tr.shot;
    const int nt = Sp->nt;
    if (it >= nt - 1) return;
    const int nx = Sp->nx, nz = Sp->nz, ldz = Sp->ldz;
    const int nxz = nx * ldz;
    const int wx0 = tr.wx0, wz0 = tr.wz0;
    // every point this tile evaluates is clear of the SBP boundary bands
    const bool interior = wx0 >= 6 && wx0 + TX + 6 <= nx && wz0 >= 6 && wz0 + TZ + 6 <= nz;
    const bool lean = CORE ? RZ == 2 : (!AE && RZ == 2 && interior && (wz0 & 1) == 0);
    // one cell per thread: tiles clear of the boundary bands take the scalar
    // interior forms (no closure code, which keeps the hot loop small); a
    // thread whose cell the tile does not own computes nothing in phase 3
    const bool lean1 = CORE ? RZ == 1 : (RZ == 1 && interior);

    const float *__restrict__ curr = Sp->u[(it + 1) & 1];
    float *__restrict__ pn = Sp->u[it & 1];              // prev in, next out
    const int mld = M.ldz;
    const long long mofs = (long long)Sp->x0 * mld;
    const float *__restrict__ mp0 = M.p0 + mofs;
    const float *__restrict__ mp1 = M.p1 + mofs;
    const float *__restrict__ mp2 = M.p2 + mofs;
    const float *__restrict__ qsrc = VTI ? M.fxx + mofs : mp0;

    const int itf = GRAD ? (nt - 1 - (it + 1)) / C.sub : 0;
    const bool do_grad = GRAD && (flags & F_GRAD) && ((nt - 1 - (it + 1)) % C.sub == 0) &&
                         (!AE || (nt - 1 - (it + 1)) / C.sub != 0);
    const int prec = C.snap_prec;
    float finv = 1.f;
    if (GRAD && do_grad && prec != SNAP_FP32) finv = 1.f / snap_scale(Sp->snap_amax, itf);
    const long long slot_elems = Sp->snap_slot;
    const void *snap = Sp->snap;

    // scalar interior path: start the copies of the own cell's operands (prev,
    // rho; for the imaging condition the neighbouring snapshots, the gradient
    // and the VTI coefficients) so that their latency overlaps phases 1 and 2;
    // each thread waits for its own copies in phase 3
    if (RZ == 1 && lean1) {
        const int gx = wx0 + (int)(threadIdx.x >> 5), gz = wz0 + (int)(threadIdx.x & 31);
        if (gx >= tr.ox0 && gx < tr.ox1 && gz >= tr.oz0 && gz < tr.oz1) {
            float *own = OWN + threadIdx.x;
            const long long cell = (long long)gx * ldz + gz, mcell = (long long)gx * mld + gz;
            cp_async4(own + OS_P0 * NT, pn + cell);
            cp_async4(own + OS_P1 * NT, pn + nxz + cell);
            cp_async4(own + OS_RHO * NT, mp2 + mcell);
            if (GRAD && do_grad) {
                const int last = nt / C.sub;
                if (itf + 1 <= last) {
                    const long long o = (long long)(itf + 1) * slot_elems + cell;
                    cp_async4(own + OS_FP0 * NT, snap_word(snap, o, prec));
                    cp_async4(own + OS_FP1 * NT, snap_word(snap, o + nxz, prec));
                }
                if (itf > 0) {
                    const long long o = (long long)(itf - 1) * slot_elems + cell;
                    cp_async4(own + OS_FM0 * NT, snap_word(snap, o, prec));
                    cp_async4(own + OS_FM1 * NT, snap_word(snap, o + nxz, prec));
                }
                const float *g = Sp->grad + cell;
                cp_async4(own + OS_G0 * NT, g);
                cp_async4(own + OS_G1 * NT, g + nxz);
                cp_async4(own + OS_G2 * NT, g + 2 * (long long)nxz);
                if (VTI) {
                    cp_async4(own + OS_EPS * NT, M.eps + mofs + mcell);
                    cp_async4(own + OS_V2 * NT, M.gv2 + mofs + mcell);
                    cp_async4(own + OS_V3 * NT, M.gv3 + mofs + mcell);
                }
            }
        }
    }

    // ---- phase 1: curr with a 4-cell halo, coefficients (and snapshot) with a 2-cell halo
    // (vector loads for interior tiles that start on a multiple of 4 cells)
    if ((lean || lean1) && (wz0 & 3) == 0) {
        constexpr int Q4 = UZ / 4;   // float4 per window row
        for (int f = threadIdx.x; f < UX * Q4; f += NT) {
            const int r = f / Q4, q = f - r * Q4;
            const int o = (wx0 - 4 + r) * ldz + wz0 - 4 + 4 * q;
            const float4 a = *reinterpret_cast<const float4 *>(curr + o);
            const float4 b = *reinterpret_cast<const float4 *>(curr + nxz + o);
            *reinterpret_cast<float4 *>(U0 + r * UZ + 4 * q) = a;
            *reinterpret_cast<float4 *>(U1 + r * UZ + 4 * q) = b;
        }
        constexpr int Q2 = WZ / 2;
        for (int f = threadIdx.x; f < WX * Q2; f += NT) {
            const int r = f / Q2, q = f - r * Q2;
            const int o = (wx0 - 2 + r) * mld + wz0 - 2 + 2 * q;
            *reinterpret_cast<float2 *>(MU + r * WZ + 2 * q) = *reinterpret_cast<const float2 *>(mp1 + o);
            *reinterpret_cast<float2 *>(Q + r * WZ + 2 * q) = *reinterpret_cast<const float2 *>(qsrc + o);
            if (GRAD) {
                float2 f0 = make_float2(0.f, 0.f), f1 = f0;
                if (do_grad) {
                    const long long so = (long long)itf * slot_elems + (wx0 - 2 + r) * ldz + wz0 - 2 + 2 * q;
                    f0 = snap_load2(snap, so, prec, finv);
                    f1 = snap_load2(snap, so + nxz, prec, finv);
                }
                *reinterpret_cast<float2 *>(F0 + r * WZ + 2 * q) = f0;
                *reinterpret_cast<float2 *>(F1 + r * WZ + 2 * q) = f1;
            }
        }
    } else if ((lean || lean1) && (wz0 & 1) == 0) {
        // interior window on an even row: pairs of samples, no bounds checks
        // (the window and its 4-cell halo lie inside the grid)
        constexpr int Q2U = UZ / 2;
        for (int f = threadIdx.x; f < UX * Q2U; f += NT) {
            const int r = f / Q2U, q = f - r * Q2U;
            const int o = (wx0 - 4 + r) * ldz + wz0 - 4 + 2 * q;
            *reinterpret_cast<float2 *>(U0 + r * UZ + 2 * q) = *reinterpret_cast<const float2 *>(curr + o);
            *reinterpret_cast<float2 *>(U1 + r * UZ + 2 * q) = *reinterpret_cast<const float2 *>(curr + nxz + o);
        }
        constexpr int Q2 = WZ / 2;
        for (int f = threadIdx.x; f < WX * Q2; f += NT) {
            const int r = f / Q2, q = f - r * Q2;
            const int o = (wx0 - 2 + r) * mld + wz0 - 2 + 2 * q;
            *reinterpret_cast<float2 *>(MU + r * WZ + 2 * q) = *reinterpret_cast<const float2 *>(mp1 + o);
            *reinterpret_cast<float2 *>(Q + r * WZ + 2 * q) = *reinterpret_cast<const float2 *>(qsrc + o);
            if (GRAD) {
                float2 f0 = make_float2(0.f, 0.f), f1 = f0;
                if (do_grad) {
                    const long long so = (long long)itf * slot_elems + (wx0 - 2 + r) * ldz + wz0 - 2 + 2 * q;
                    f0 = snap_load2(snap, so, prec, finv);
                    f1 = snap_load2(snap, so + nxz, prec, finv);
                }
                *reinterpret_cast<float2 *>(F0 + r * WZ + 2 * q) = f0;
                *reinterpret_cast<float2 *>(F1 + r * WZ + 2 * q) = f1;
            }
        }
    } else {
        for (int i = threadIdx.x; i < UX * UZ; i += NT) {
            const int sx = i / UZ, sz = i - sx * UZ;
            const int gx = wx0 - 4 + sx, gz = wz0 - 4 + sz;
            float a = 0.f, b = 0.f;
            if (gx >= 0 && gx < nx && gz >= 0 && gz < nz) {
                const int o = gx * ldz + gz;
                a = curr[o];
                b = curr[nxz + o];
            }
            U0[i] = a;
            U1[i] = b;
        }
        for (int i = threadIdx.x; i < WX * WZ; i += NT) {
            const int sx = i / WZ, sz = i - sx * WZ;
            const int gx = wx0 - 2 + sx, gz = wz0 - 2 + sz;
            float m = 0.f, q = 0.f;
            const bool in = gx >= 0 && gx < nx && gz >= 0 && gz < nz;
            if (in) {
                const int o = gx * mld + gz;
                m = mp1[o];
                q = qsrc[o];
            }
            MU[i] = m;
            Q[i] = q;
            if (GRAD) {
                float f0 = 0.f, f1 = 0.f;
                if (do_grad && in) {
                    const long long o = (long long)itf * slot_elems + gx * ldz + gz;
                    f0 = snap_load(snap, o, prec, finv);
                    f1 = snap_load(snap, o + nxz, prec, finv);
                }
                F0[i] = f0;
                F1[i] = f1;
            }
        }
    }
    __syncthreads();

    // ---- phase 2: first derivatives of curr on the tile plus a 2-cell halo
    if (lean) {
        constexpr int Q2 = WZ / 2;
        for (int f = threadIdx.x; f < WX * Q2; f += NT) {
            const int sx = f / Q2, pz = 2 * (f - sx * Q2);
            const int ui = (sx + 2) * UZ + pz + 2;
            const float2 am2 = ld2(U0, ui - 2 * UZ), am1 = ld2(U0, ui - UZ), ap1 = ld2(U0, ui + UZ), ap2 = ld2(U0, ui + 2 * UZ);
            const float2 bm2 = ld2(U1, ui - 2 * UZ), bm1 = ld2(U1, ui - UZ), bp1 = ld2(U1, ui + UZ), bp2 = ld2(U1, ui + 2 * UZ);
            const float2 alo = ld2(U0, ui - 2), amid = ld2(U0, ui), ahi = ld2(U0, ui + 2);
            const float2 blo = ld2(U1, ui - 2), bmid = ld2(U1, ui), bhi = ld2(U1, ui + 2);
            // the pair's z-neighbours: (m2, m1, p1, p2) = (lo, lo|mid, mid|hi, hi)
            const float2 ux_x = d1s2(am2, am1, ap1, ap2, C.sdx);
            const float2 uz_z = d1s2(blo, zsh(blo, bmid), zsh(bmid, bhi), bhi, C.sdz);
            const float2 bx = d1s2(bm2, bm1, bp1, bp2, C.sdx);
            const float2 cz = d1s2(alo, zsh(alo, amid), zsh(amid, ahi), ahi, C.sdz);
            float2 t0, t1 = make_float2(0.f, 0.f);
            if (!VTI) {
                t0 = add2(ux_x, uz_z);
            } else {
                const long long o = mofs + (long long)(wx0 - 2 + sx) * mld + wz0 - 2 + pz;
                const float2 lb = *reinterpret_cast<const float2 *>(M.lbis + o);
                const float2 cc = *reinterpret_cast<const float2 *>(M.c13 + o);
                const float2 ll = *reinterpret_cast<const float2 *>(M.p0 + o);
                t0 = add2(mul2(lb, ux_x), mul2(cc, uz_z));
                t1 = add2(mul2(ll, uz_z), mul2(cc, ux_x));
            }
            const int wo = sx * WZ + pz;
            *reinterpret_cast<float2 *>(T0 + wo) = t0;
            if (VTI) *reinterpret_cast<float2 *>(T1 + wo) = t1;
            *reinterpret_cast<float2 *>(BX + wo) = bx;
            *reinterpret_cast<float2 *>(CZ + wo) = cz;
        }
    } else if (lean1) {
        for (int i = threadIdx.x; i < WX * WZ; i += NT) {
            const int sx = i / WZ, sz = i - sx * WZ;
            const int ui = (sx + 2) * UZ + (sz + 2);
            const float ux_x = d1i(U0 + ui, UZ, C.sdx);
            const float uz_z = d1i(U1 + ui, 1, C.sdz);
            float t0, t1 = 0.f;
            if (AE) {
                t0 = ux_x;
                t1 = uz_z;
            } else if (!VTI) {
                t0 = ux_x + uz_z;
            } else {
                const long long o = mofs + (long long)(wx0 - 2 + sx) * mld + wz0 - 2 + sz;
                const float lb = M.lbis[o], c13 = M.c13[o], lam = M.p0[o];
                t0 = lb * ux_x + c13 * uz_z;
                t1 = lam * uz_z + c13 * ux_x;
            }
            T0[i] = t0;
            if (VTI || AE) T1[i] = t1;
            BX[i] = d1i(U1 + ui, UZ, C.sdx);
            CZ[i] = d1i(U0 + ui, 1, C.sdz);
        }
    } else {
        for (int i = threadIdx.x; i < WX * WZ; i += NT) {
            const int sx = i / WZ, sz = i - sx * WZ;
            const int gx = wx0 - 2 + sx, gz = wz0 - 2 + sz;
            const int ui = (sx + 2) * UZ + (sz + 2);
            // a closure reads up to 5 samples from its boundary: evaluate only
            // where the loaded window holds them (other points are never used)
            const bool okx = (gx >= 4 && gx < nx - 4) || (gx < 4 ? wx0 <= 4 : wx0 + TX + 4 >= nx);
            const bool okz = (gz >= 4 && gz < nz - 4) || (gz < 4 ? wz0 <= 4 : wz0 + TZ + 4 >= nz);
            const bool ok = gx >= 0 && gx < nx && gz >= 0 && gz < nz && okx && okz;
            float t0 = 0.f, t1 = 0.f, bx = 0.f, cz = 0.f;
            if (ok) {
                const float ux_x = d1(U0 + ui, UZ, gx, nx, C.dx, C.sdx);
                const float uz_z = d1(U1 + ui, 1, gz, nz, C.dz, C.sdz);
                bx = d1(U1 + ui, UZ, gx, nx, C.dx, C.sdx);
                cz = d1(U0 + ui, 1, gz, nz, C.dz, C.sdz);
                if (AE) {
                    t0 = ux_x;
                    t1 = uz_z;
                } else if (!VTI) {
                    t0 = ux_x + uz_z;
                } else {
                    const long long o = mofs + (long long)gx * mld + gz;
                    const float lb = M.lbis[o], c13 = M.c13[o], lam = M.p0[o];
                    t0 = lb * ux_x + c13 * uz_z;
                    t1 = lam * uz_z + c13 * ux_x;
                }
            }
            T0[i] = t0;
            if (VTI || AE) T1[i] = t1;
            BX[i] = bx;
            CZ[i] = cz;
        }
    }
    __syncthreads();

    // ---- phase 3
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile_id = tr.unit;

    // receivers (forward): one thread per receiver of this tile
    if (flags & F_EXTRACT) {
        const int e0 = Sp->ext_off[tile_id], e1 = Sp->ext_off[tile_id + 1];
        for (int e = e0 + threadIdx.x; e < e1; e += NT) {
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
    const int e0 = Sp->inj_off[tile_id], e1 = Sp->inj_off[tile_id + 1];
    const float *srcrow = Sp->src + (long long)it * Sp->nsrc;
    const bool store = (flags & F_STORE) && (it % C.sub == 0);
    float amax = 0.f;

    if (lean) {
        const int gx = wx0 + warp;
        const int gz0 = wz0 + 2 * lane;
        const int ui = (warp + 4) * UZ + 2 * lane + 4;
        const int wi = (warp + 2) * WZ + 2 * lane + 2;
        const int cell0 = gx * ldz + gz0;
        // x-direction samples
        const float2 am2 = ld2(U0, ui - 2 * UZ), am1 = ld2(U0, ui - UZ), a00 = ld2(U0, ui), ap1 = ld2(U0, ui + UZ), ap2 = ld2(U0, ui + 2 * UZ);
        const float2 bm2 = ld2(U1, ui - 2 * UZ), bm1 = ld2(U1, ui - UZ), b00 = ld2(U1, ui), bp1 = ld2(U1, ui + UZ), bp2 = ld2(U1, ui + 2 * UZ);
        const float2 alo = ld2(U0, ui - 2), ahi = ld2(U0, ui + 2), blo = ld2(U1, ui - 2), bhi = ld2(U1, ui + 2);
        const float2 mm2 = ld2(MU, wi - 2 * WZ), mm1 = ld2(MU, wi - WZ), m00 = ld2(MU, wi), mp1v = ld2(MU, wi + WZ), mp2v = ld2(MU, wi + 2 * WZ);
        const float2 mlo = ld2(MU, wi - 2), mhi = ld2(MU, wi + 2);
        const float2 qm2 = ld2(Q, wi - 2 * WZ), qm1 = ld2(Q, wi - WZ), qp1 = ld2(Q, wi + WZ), qp2 = ld2(Q, wi + 2 * WZ);
        const float2 tm2 = ld2(T0, wi - 2 * WZ), tm1 = ld2(T0, wi - WZ), tp1 = ld2(T0, wi + WZ), tp2 = ld2(T0, wi + 2 * WZ);
        const float *TZS = VTI ? T1 : T0;
        const float2 tlo = ld2(TZS, wi - 2), tmid = ld2(TZS, wi), thi = ld2(TZS, wi + 2);
        const float2 cm2 = ld2(CZ, wi - 2 * WZ), cm1 = ld2(CZ, wi - WZ), cp1 = ld2(CZ, wi + WZ), cp2 = ld2(CZ, wi + 2 * WZ);
        const float2 xlo = ld2(BX, wi - 2), xmid = ld2(BX, wi), xhi = ld2(BX, wi + 2);
        const float2 tzv2 = *reinterpret_cast<const float2 *>(Sp->tz + gz0);
        const float txv = Sp->tx[gx];
        float2 pv0 = *reinterpret_cast<const float2 *>(pn + cell0);
        float2 pv1 = *reinterpret_cast<const float2 *>(pn + nxz + cell0);
        const float2 rho2 = *reinterpret_cast<const float2 *>(mp2 + gx * mld + gz0);
        // cells of the pair this tile owns (windows next to a flush window own part of theirs)
        const bool ownx = gx >= tr.ox0 && gx < tr.ox1;
        const bool own0 = ownx && gz0 >= tr.oz0 && gz0 < tr.oz1;
        const bool own1 = ownx && gz0 + 1 >= tr.oz0 && gz0 + 1 < tr.oz1;
        if (store) {
            const int slot = it / C.sub;
            const float sc = prec == SNAP_FP32 ? 1.f : snap_scale(Sp->snap_amax, slot);
            const long long o = (long long)slot * slot_elems + cell0;
            if (own0) {
                snap_store(Sp->snap, o, prec, a00.x, sc);
                snap_store(Sp->snap, o + nxz, prec, b00.x, sc);
            }
            if (own1) {
                snap_store(Sp->snap, o + 1, prec, a00.y, sc);
                snap_store(Sp->snap, o + nxz + 1, prec, b00.y, sc);
            }
        }
        // the pair's z-neighbours of a field with pairs (lo, 00, hi): (lo, lo|00, 00|hi, hi)
        const float2 mz1 = zsh(mlo, m00), mzp = zsh(m00, mhi);
        const Brk2 bkx = brk52(mm2, mm1, m00, mp1v, mp2v);
        const Brk2 bkz = brk52(mlo, mz1, m00, mzp, mhi);
        const float2 zero2 = make_float2(0.f, 0.f);
        float2 n0, n1;
        if (!VTI) n0 = d2s2(zero2, twice2(bkx), am2, am1, a00, ap1, ap2, C.inv_d2x);
        else n0 = d2s2(zero2, brk52(qm2, qm1, ld2(Q, wi), qp1, qp2), am2, am1, a00, ap1, ap2, C.inv_d2x);
        n1 = d2s2(zero2, twice2(bkz), blo, zsh(blo, b00), b00, zsh(b00, bhi), bhi, C.inv_d2z);
        n1 = d2s2(n1, bkx, bm2, bm1, b00, bp1, bp2, C.inv_d2x);
        n0 = d2s2(n0, bkz, alo, zsh(alo, a00), a00, zsh(a00, ahi), ahi, C.inv_d2z);
        if (!VTI) {
            const float2 qlo = ld2(Q, wi - 2), qmid = ld2(Q, wi), qhi = ld2(Q, wi + 2);
            n0 = add2(n0, md1s2(tm2, qm2, tm1, qm1, tp1, qp1, tp2, qp2, C.adx));
            n1 = add2(n1, md1s2(tlo, qlo, zsh(tlo, tmid), zsh(qlo, qmid), zsh(tmid, thi), zsh(qmid, qhi), thi, qhi,
                                C.adz));
        } else {
            n0 = add2(n0, d1s2(tm2, tm1, tp1, tp2, C.sdx));
            n1 = add2(n1, d1s2(tlo, zsh(tlo, tmid), zsh(tmid, thi), thi, C.sdz));
        }
        n1 = add2(n1, md1s2(cm2, mm2, cm1, mm1, cp1, mp1v, cp2, mp2v, C.adx));
        n0 = add2(n0, md1s2(xlo, mlo, zsh(xlo, xmid), mz1, zsh(xmid, xhi), mzp, xhi, mhi, C.adz));
        // sources, cell by cell in the reference's order
        for (int e = e0; e < e1; e++) {
            const InjEntry &E = Sp->inj[e];
            if (E.gx == gx && (E.gz == gz0 || E.gz == gz0 + 1)) {
                const float v = E.mt ? (E.wa * srcrow[E.ia] - E.wb * srcrow[E.ib]) : E.wa * srcrow[E.ia];
                if (E.comp == 0) {
                    if (E.gz == gz0) n0.x += v;
                    else n0.y += v;
                } else {
                    if (E.gz == gz0) n1.x += v;
                    else n1.y += v;
                }
            }
        }
        const float2 tzx = bc2(txv);
        if (it > 0) {
            pv0 = mul2(mul2(pv0, tzv2), tzx);
            pv1 = mul2(mul2(pv1, tzv2), tzx);
        }
        // leapfrog: dt^2 n / rho + 2 curr - prev (one IEEE division per cell)
        float2 q0 = mul2(bc2(C.dt2), n0), q1 = mul2(bc2(C.dt2), n1);
        q0 = make_float2(q0.x / rho2.x, q0.y / rho2.y);
        q1 = make_float2(q1.x / rho2.x, q1.y / rho2.y);
        n0 = sub2(add2(q0, mul2(bc2(2.f), a00)), pv0);
        n1 = sub2(add2(q1, mul2(bc2(2.f), b00)), pv1);
        const float2 out0 = mul2(mul2(n0, tzv2), tzx);
        const float2 out1 = mul2(mul2(n1, tzv2), tzx);
        if (own0 && own1) {
            *reinterpret_cast<float2 *>(pn + cell0) = out0;
            *reinterpret_cast<float2 *>(pn + nxz + cell0) = out1;
        } else {
            if (own0) {
                pn[cell0] = out0.x;
                pn[nxz + cell0] = out1.x;
            }
            if (own1) {
                pn[cell0 + 1] = out0.y;
                pn[nxz + cell0 + 1] = out1.y;
            }
        }
        if (own0) amax = fmaxf(amax, fmaxf(fabsf(out0.x), fabsf(out1.x)));
        if (own1) amax = fmaxf(amax, fmaxf(fabsf(out0.y), fabsf(out1.y)));

        if (GRAD && do_grad && (own0 || own1)) {
            const float2 ax0 = d1s2(am2, am1, ap1, ap2, C.sdx);
            const float2 az1 = d1s2(blo, zsh(blo, b00), zsh(b00, bhi), bhi, C.sdz);
            const float2 f0m2 = ld2(F0, wi - 2 * WZ), f0m1 = ld2(F0, wi - WZ), f0p1 = ld2(F0, wi + WZ), f0p2 = ld2(F0, wi + 2 * WZ);
            const float2 f1m2 = ld2(F1, wi - 2 * WZ), f1m1 = ld2(F1, wi - WZ), f1p1 = ld2(F1, wi + WZ), f1p2 = ld2(F1, wi + 2 * WZ);
            const float2 f0lo = ld2(F0, wi - 2), f0c = ld2(F0, wi), f0hi = ld2(F0, wi + 2);
            const float2 f1lo = ld2(F1, wi - 2), f1c = ld2(F1, wi), f1hi = ld2(F1, wi + 2);
            const int last = nt / C.sub;
            float2 fp0 = make_float2(0.f, 0.f), fp1 = fp0, fm0 = fp0, fm1 = fp0;
            if (itf + 1 <= last) {
                const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf + 1);
                const long long o = (long long)(itf + 1) * slot_elems + cell0;
                fp0 = snap_load2(snap, o, prec, inv);
                fp1 = snap_load2(snap, o + nxz, prec, inv);
            }
            if (itf > 0) {
                const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf - 1);
                const long long o = (long long)(itf - 1) * slot_elems + cell0;
                fm0 = snap_load2(snap, o, prec, inv);
                fm1 = snap_load2(snap, o + nxz, prec, inv);
            }
            const float2 t0 = d1s2(f0m2, f0m1, f0p1, f0p2, C.sdx);
            const float2 t1 = d1s2(f1lo, zsh(f1lo, f1c), zsh(f1c, f1hi), f1hi, C.sdz);
            const float2 t2 = d1s2(f1m2, f1m1, f1p1, f1p2, C.sdx);
            const float2 t3 = d1s2(f0lo, zsh(f0lo, f0c), zsh(f0c, f0hi), f0hi, C.sdz);
            const float2 az0 = ld2(CZ, wi), ax1 = xmid;
            const float2 two = bc2(2.f);
            float2 dl = make_float2(0.f, 0.f), dm;
            if (!VTI) {
                dm = add2(add2(mul2(add2(az0, ax1), add2(t2, t3)), mul2(mul2(two, ax0), t0)), mul2(mul2(two, az1), t1));
            } else {
                const long long mo = mofs + (long long)gx * mld + gz0;
                const float2 v2v = *reinterpret_cast<const float2 *>(M.gv2 + mo);
                const float2 v3v = *reinterpret_cast<const float2 *>(M.gv3 + mo);
                const float2 epsv = *reinterpret_cast<const float2 *>(M.eps + mo);
                const float2 e2 = add2(bc2(1.f), mul2(two, epsv));
                const float2 cross = add2(mul2(ax0, t1), mul2(az1, t0));
                dl = add2(add2(mul2(mul2(e2, ax0), t0), mul2(az1, t1)), mul2(v2v, cross));
                dm = add2(add2(add2(mul2(add2(az0, ax1), add2(t2, t3)), mul2(mul2(mul2(two, e2), ax0), t0)),
                               mul2(mul2(two, az1), t1)),
                          mul2(v3v, cross));
            }
            float *g0 = Sp->grad + cell0, *g1 = g0 + nxz, *g2 = g1 + nxz;
            float2 G0 = *reinterpret_cast<float2 *>(g0), G1 = *reinterpret_cast<float2 *>(g1), G2 = *reinterpret_cast<float2 *>(g2);
            const float gw = Sp->gwt[itf];
            const double wdt = (double)gw * 1.0 / (double)dtg;
            const float2 gd = bc2(gw * dtg);
            if (itf > 0) {
                // interior and last imaging times: FP32 terms (the density term below, in double)
                if (!VTI) G0 = add2(G0, mul2(mul2(gd, add2(ax0, az1)), add2(t0, t1)));
                else G0 = add2(G0, mul2(gd, dl));
                G1 = add2(G1, mul2(gd, dm));
            }
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const float f0 = pick(f0c, c), f1 = pick(f1c, c);
                const float a0 = pick(out0, c), a1 = pick(out1, c);
                float g0v = pick(G0, c), g1v = pick(G1, c), g2v = pick(G2, c);
                const float fp0c = pick(fp0, c), fp1c = pick(fp1, c), fm0c = pick(fm0, c), fm1c = pick(fm1, c);
                if (itf > 0 && itf < last) {
                    g2v = (float)((double)g2v + wdt * (double)(a0 * (fp0c - 2 * f0 + fm0c) + a1 * (fp1c - 2 * f1 + fm1c)));
                } else if (itf == 0) {
                    const double wh = (double)gw * 0.5 * (double)dtg;
                    const float ax0c = pick(ax0, c), az1c = pick(az1, c);
                    if (!VTI) g0v = (float)((double)g0v + wh * (double)(ax0c + az1c) * (double)(pick(t0, c) + pick(t1, c)));
                    else g0v = (float)((double)g0v + wh * (double)pick(dl, c));
                    g1v = (float)((double)g1v + wh * (double)pick(dm, c));
                    g2v = (float)((double)g2v + wdt * (double)(a0 * (fp0c - f0) + a1 * (fp1c - f1)));
                } else {
                    g2v = (float)((double)g2v + wdt * (double)(a0 * (-f0 + fm0c) + a1 * (-f1 + fm1c)));
                }
                if (c == 0) { G0.x = g0v; G1.x = g1v; G2.x = g2v; } else { G0.y = g0v; G1.y = g1v; G2.y = g2v; }
            }
            if (own0 && own1) {
                *reinterpret_cast<float2 *>(g0) = G0;
                *reinterpret_cast<float2 *>(g1) = G1;
                *reinterpret_cast<float2 *>(g2) = G2;
            } else if (own0) {
                g0[0] = G0.x;
                g1[0] = G1.x;
                g2[0] = G2.x;
            } else {
                g0[1] = G0.y;
                g1[1] = G1.y;
                g2[1] = G2.y;
            }
        }
    } else if (lean1) {
        // the general path's arithmetic in its interior forms (sbp.cuh d1i,
        // md1i, d2i): no SAT and no boundary divisor can reach these cells
        const int gx = wx0 + warp, gz = wz0 + lane;
        if (gx >= tr.ox0 && gx < tr.ox1 && gz >= tr.oz0 && gz < tr.oz1) {
        const int ui = (warp + 4) * UZ + (lane + 4);
        const int wi = (warp + 2) * WZ + (lane + 2);
        const int cell = gx * ldz + gz;
        if (store) {
            const int slot = it / C.sub;
            const float sc = prec == SNAP_FP32 ? 1.f : snap_scale(Sp->snap_amax, slot);
            const long long o = (long long)slot * slot_elems + cell;
            snap_store(Sp->snap, o, prec, U0[ui], sc);
            snap_store(Sp->snap, o + nxz, prec, U1[ui], sc);
        }
        float n0 = 0.f, n1 = 0.f;
        if (!VTI) {
            n0 = d2i(n0, twice(brackets(MU + wi, WZ)), U0 + ui, UZ, C.inv_d2x);
            n1 = d2i(n1, twice(brackets(MU + wi, 1)), U1 + ui, 1, C.inv_d2z);
        } else {
            n0 = d2i(n0, brackets(Q + wi, WZ), U0 + ui, UZ, C.inv_d2x);
            n1 = d2i(n1, twice(brackets(MU + wi, 1)), U1 + ui, 1, C.inv_d2z);
        }
        n1 = d2i(n1, brackets(MU + wi, WZ), U1 + ui, UZ, C.inv_d2x);
        n0 = d2i(n0, brackets(MU + wi, 1), U0 + ui, 1, C.inv_d2z);
        if (AE) {
            // the acoustic-elastic propagator's version-1 split, in the general path's order
            n0 += md1i(T0 + wi, Q + wi, WZ, C.adx);
            n1 += md1i(T1 + wi, Q + wi, 1, C.adz);
            n0 += md1i(T1 + wi, Q + wi, WZ, C.adx);
            n1 += md1i(T0 + wi, Q + wi, 1, C.adz);
        } else if (!VTI) {
            n0 += md1i(T0 + wi, Q + wi, WZ, C.adx);
            n1 += md1i(T0 + wi, Q + wi, 1, C.adz);
        } else {
            n0 += d1i(T0 + wi, WZ, C.sdx);
            n1 += d1i(T1 + wi, 1, C.sdz);
        }
        n1 += md1i(CZ + wi, MU + wi, WZ, C.adx);
        n0 += md1i(BX + wi, MU + wi, 1, C.adz);
        for (int e = e0; e < e1; e++) {
            const InjEntry &E = Sp->inj[e];
            if (E.gx == gx && E.gz == gz) {
                const float v = E.mt ? (E.wa * srcrow[E.ia] - E.wb * srcrow[E.ib]) : E.wa * srcrow[E.ia];
                if (E.comp == 0) n0 += v;
                else n1 += v;
            }
        }
        const float tzv = Sp->tz[gz], txv = Sp->tx[gx];
        cp_async_wait_all();
        const float *own = OWN + threadIdx.x;
        float p0 = own[OS_P0 * NT], p1 = own[OS_P1 * NT];
        if (it > 0) {
            p0 = p0 * tzv * txv;
            p1 = p1 * tzv * txv;
        }
        const float rho = own[OS_RHO * NT];
        n0 = C.dt2 * n0 / rho + 2 * U0[ui] - p0;
        n1 = C.dt2 * n1 / rho + 2 * U1[ui] - p1;
        n0 = n0 * tzv * txv;
        n1 = n1 * tzv * txv;
        pn[cell] = n0;
        pn[nxz + cell] = n1;
        amax = fmaxf(amax, fmaxf(fabsf(n0), fabsf(n1)));
        if (GRAD && do_grad) {
            const float ax0 = d1i(U0 + ui, UZ, C.sdx);
            const float az1 = d1i(U1 + ui, 1, C.sdz);
            const float t0 = d1i(F0 + wi, WZ, C.sdx);
            const float t1 = d1i(F1 + wi, 1, C.sdz);
            const float t2 = d1i(F1 + wi, WZ, C.sdx);
            const float t3 = d1i(F0 + wi, 1, C.sdz);
            const float az0 = CZ[wi], ax1 = BX[wi];
            const int last = nt / C.sub;
            const float f0 = F0[wi], f1 = F1[wi];
            float fp0 = 0.f, fp1 = 0.f, fm0 = 0.f, fm1 = 0.f;
            if (itf + 1 <= last) {
                const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf + 1);
                const long long o = (long long)(itf + 1) * slot_elems + cell;
                fp0 = snap_from_word(own[OS_FP0 * NT], o, prec, inv);
                fp1 = snap_from_word(own[OS_FP1 * NT], o + nxz, prec, inv);
            }
            if (itf > 0) {
                const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf - 1);
                const long long o = (long long)(itf - 1) * slot_elems + cell;
                fm0 = snap_from_word(own[OS_FM0 * NT], o, prec, inv);
                fm1 = snap_from_word(own[OS_FM1 * NT], o + nxz, prec, inv);
            }
            float dl, dm;
            if (!VTI) {
                dl = 0.f;
                dm = (az0 + ax1) * (t2 + t3) + 2 * ax0 * t0 + 2 * az1 * t1;
            } else {
                const float e2 = 1 + 2 * own[OS_EPS * NT];
                const float v2 = own[OS_V2 * NT], v3 = own[OS_V3 * NT];
                dl = e2 * ax0 * t0 + az1 * t1 + v2 * (ax0 * t1 + az1 * t0);
                dm = (az0 + ax1) * (t2 + t3) + 2 * e2 * ax0 * t0 + 2 * az1 * t1 + v3 * (ax0 * t1 + az1 * t0);
            }
            float *g0 = Sp->grad + cell, *g1 = g0 + nxz, *g2 = g1 + nxz;
            const float G0 = own[OS_G0 * NT], G1 = own[OS_G1 * NT], G2 = own[OS_G2 * NT];
            const float gw = Sp->gwt[itf];
            const double wdt = (double)gw * 1.0 / (double)dtg;
            if (itf > 0 && itf < last) {
                if (!VTI) *g0 = G0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                else *g0 = G0 + gw * dtg * dl;
                *g1 = G1 + gw * dtg * dm;
                *g2 = (float)((double)G2 + wdt * (double)(n0 * (fp0 - 2 * f0 + fm0) + n1 * (fp1 - 2 * f1 + fm1)));
            } else if (itf == 0) {
                const double wh = (double)gw * 0.5 * (double)dtg;
                if (!VTI) *g0 = (float)((double)G0 + wh * (double)(ax0 + az1) * (double)(t0 + t1));
                else *g0 = (float)((double)G0 + wh * (double)dl);
                *g1 = (float)((double)G1 + wh * (double)dm);
                *g2 = (float)((double)G2 + wdt * (double)(n0 * (fp0 - f0) + n1 * (fp1 - f1)));
            } else {
                if (!VTI) *g0 = G0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                else *g0 = G0 + gw * dtg * dl;
                *g1 = G1 + gw * dtg * dm;
                *g2 = (float)((double)G2 + wdt * (double)(n0 * (-f0 + fm0) + n1 * (-f1 + fm1)));
            }
        }
        }
    } else {
#pragma unroll
        for (int h = 0; h < RZ; h++) {
            const int tz = lane + 32 * h, tx = warp;
            const int gx = wx0 + tx, gz = wz0 + tz;
            const bool owned = gx >= tr.ox0 && gx < tr.ox1 && gz >= tr.oz0 && gz < tr.oz1;
            if (!owned) continue;
            const int ui = (tx + 4) * UZ + (tz + 4);
            const int wi = (tx + 2) * WZ + (tz + 2);
            const int cell = gx * ldz + gz;
            const int mcell = gx * mld + gz;
            // BAND: the imaging condition's global operands, loaded ahead
            float hfp0 = 0.f, hfp1 = 0.f, hfm0 = 0.f, hfm1 = 0.f, hg0 = 0.f, hg1 = 0.f, hg2 = 0.f;
            if (BAND && GRAD && do_grad) {
                const int last = nt / C.sub;
                if (itf + 1 <= last) {
                    const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf + 1);
                    const long long o = (long long)(itf + 1) * slot_elems + cell;
                    hfp0 = snap_load(snap, o, prec, inv);
                    hfp1 = snap_load(snap, o + nxz, prec, inv);
                }
                if (itf > 0) {
                    const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf - 1);
                    const long long o = (long long)(itf - 1) * slot_elems + cell;
                    hfm0 = snap_load(snap, o, prec, inv);
                    hfm1 = snap_load(snap, o + nxz, prec, inv);
                }
                const float *g = Sp->grad + cell;
                hg0 = g[0];
                hg1 = g[nxz];
                hg2 = g[2 * nxz];
            }
            if (store) {
                const int slot = it / C.sub;
                const float sc = prec == SNAP_FP32 ? 1.f : snap_scale(Sp->snap_amax, slot);
                const long long o = (long long)slot * slot_elems + cell;
                snap_store(Sp->snap, o, prec, U0[ui], sc);
                snap_store(Sp->snap, o + nxz, prec, U1[ui], sc);
            }
            const float mu = MU[wi];
            float n0 = 0.f, n1 = 0.f;
            if (!VTI) {
                d2acc(n0, U0 + ui, UZ, MU + wi, WZ, 2.f, gx, nx, C.inv_d2x, C.d2x);
                d2acc(n1, U1 + ui, 1, MU + wi, 1, 2.f, gz, nz, C.inv_d2z, C.d2z);
            } else {
                d2acc(n0, U0 + ui, UZ, Q + wi, WZ, 1.f, gx, nx, C.inv_d2x, C.d2x);
                d2acc(n1, U1 + ui, 1, MU + wi, 1, 2.f, gz, nz, C.inv_d2z, C.d2z);
            }
            d2acc(n1, U1 + ui, UZ, MU + wi, WZ, 1.f, gx, nx, C.inv_d2x, C.d2x);
            d2acc(n0, U0 + ui, 1, MU + wi, 1, 1.f, gz, nz, C.inv_d2z, C.d2z);
            if (AE) {
                n0 += md1(T0 + wi, Q + wi, WZ, gx, nx, C.adx);
                n1 += md1(T1 + wi, Q + wi, 1, gz, nz, C.adz);
                n0 += md1(T1 + wi, Q + wi, WZ, gx, nx, C.adx);
                n1 += md1(T0 + wi, Q + wi, 1, gz, nz, C.adz);
            } else if (!VTI) {
                n0 += md1(T0 + wi, Q + wi, WZ, gx, nx, C.adx);
                n1 += md1(T0 + wi, Q + wi, 1, gz, nz, C.adz);
            } else {
                n0 += d1(T0 + wi, WZ, gx, nx, C.dx, C.sdx);
                n1 += d1(T1 + wi, 1, gz, nz, C.dz, C.sdz);
            }
            n1 += md1(CZ + wi, MU + wi, WZ, gx, nx, C.adx);
            n0 += md1(BX + wi, MU + wi, 1, gz, nz, C.adz);

            for (int e = e0; e < e1; e++) {
                const InjEntry &E = Sp->inj[e];
                if (E.gx == gx && E.gz == gz) {
                    const float v = E.mt ? (E.wa * srcrow[E.ia] - E.wb * srcrow[E.ib]) : E.wa * srcrow[E.ia];
                    if (E.comp == 0) n0 += v;
                    else n1 += v;
                }
            }

            const float tzv = Sp->tz[gz], txv = Sp->tx[gx];
            float p0 = pn[cell], p1 = pn[nxz + cell];
            if (it > 0) {
                p0 = p0 * tzv * txv;
                p1 = p1 * tzv * txv;
            }
            const float rho = mp2[mcell];

            // SAT closures (spatial_operators.hpp:160-822), in the reference's side order
            const bool edge = gz == 0 || gz == nz - 1 || gx == 0 || gx == nx - 1;
            if (edge) {
                const float lam = VTI ? mp0[mcell] : Q[wi];
                const float c13 = VTI ? M.c13[mofs + mcell] : lam;
                const float fxx = VTI ? Q[wi] : 2 * mu;
                const float lamx = VTI ? M.lbis[mofs + mcell] : lam;
                const float eps = VTI ? M.eps[mofs + mcell] : 0.f;
                const float imp_s = 0.5f * sqrtf(mu * rho);
                const float imp_p = 0.5f * sqrtf((lam + 2 * mu) * rho);
                const float imp_px = VTI ? 0.5f * sqrtf((1 + 2 * eps) * (lam + 2 * mu) * rho) : imp_p;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    // the fluid interface (top) of the acoustic-elastic propagator comes last
                    const int side = AE ? (k + 1) & 3 : k;
                    const int bc = C.bc[side];
                    if (bc != 1 && bc != 2) continue;
                    const bool ab = bc == 2;
                    if (side < 2) {
                        if (gz != (side == 0 ? 0 : nz - 1)) continue;
                        const int in = side == 0 ? 1 : -1;
                        const float sg = side == 0 ? -1.f : 1.f;
                        {
                            float t = (sg * mu) * tsum(U1 + ui, UZ, gx, nx) / C.dx + mu * nsum(U0 + ui, in) / C.dz;
                            if (ab) t = t - imp_s * p0 / C.dt;
                            n0 = n0 - C.sat_z * t;
                        }
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
                        {
                            float t = (sg * c13) * tsum(U1 + ui, 1, gz, nz) / C.dz + fxx * nsum(U0 + ui, in) / C.dx;
                            if (ab) t = t - imp_px * p0 / C.dt;
                            n0 = n0 - C.sat_x * t;
                            n0 = n0 - C.nsat_x * lamx * ndsum(U0 + ui, in);
                        }
                        {
                            float t = (sg * mu) * tsum(U0 + ui, 1, gz, nz) / C.dz + mu * nsum(U1 + ui, in) / C.dx;
                            if (ab) t = t - imp_s * p1 / C.dt;
                            n1 = n1 - C.sat_x * t;
                        }
                    }
                }
            }

            n0 = C.dt2 * n0 / rho + 2 * U0[ui] - p0;
            n1 = C.dt2 * n1 / rho + 2 * U1[ui] - p1;

            if (edge) {
                const int per = 2 * nx + 2 * nz;
                int k;
                if (gz == 0) k = gx;
                else if (gz == nz - 1) k = nx + gx;
                else if (gx == 0) k = 2 * nx + gz;
                else k = 2 * nx + nz + gz;
                n0 = n0 / Sp->den[k];
                n1 = n1 / Sp->den[per + k];
            }

            n0 = n0 * tzv * txv;
            if (AE && gz == 0) Sp->halo_save[gx] = p1;   // interface row: coupled and tapered by ae_couple
            else n1 = n1 * tzv * txv;
            pn[cell] = n0;
            pn[nxz + cell] = n1;
            amax = fmaxf(amax, fmaxf(fabsf(n0), fabsf(n1)));

            if (GRAD && do_grad) {
                const float ax0 = d1(U0 + ui, UZ, gx, nx, C.dx, C.sdx);
                const float az1 = d1(U1 + ui, 1, gz, nz, C.dz, C.sdz);
                const float t0 = d1(F0 + wi, WZ, gx, nx, C.dx, C.sdx);
                const float t1 = d1(F1 + wi, 1, gz, nz, C.dz, C.sdz);
                const float t2 = d1(F1 + wi, WZ, gx, nx, C.dx, C.sdx);
                const float t3 = d1(F0 + wi, 1, gz, nz, C.dz, C.sdz);
                const float az0 = CZ[wi], ax1 = BX[wi];
                const int last = nt / C.sub;
                const float f0 = F0[wi], f1 = F1[wi];
                float fp0 = hfp0, fp1 = hfp1, fm0 = hfm0, fm1 = hfm1;
                if (!BAND && itf + 1 <= last) {
                    const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf + 1);
                    const long long o = (long long)(itf + 1) * slot_elems + cell;
                    fp0 = snap_load(snap, o, prec, inv);
                    fp1 = snap_load(snap, o + nxz, prec, inv);
                }
                if (!BAND && itf > 0) {
                    const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf - 1);
                    const long long o = (long long)(itf - 1) * slot_elems + cell;
                    fm0 = snap_load(snap, o, prec, inv);
                    fm1 = snap_load(snap, o + nxz, prec, inv);
                }
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
                float *g0 = Sp->grad + cell, *g1 = g0 + nxz, *g2 = g1 + nxz;
                const float gw = Sp->gwt[itf];
                const double wdt = (double)gw * 1.0 / (double)dtg;
                // acoustic-elastic interface row: the density term needs the coupled uz (ae_couple)
                const bool rho_here = !AE || gz != 0;
                const float G0 = BAND ? hg0 : *g0, G1 = BAND ? hg1 : *g1;
                if (itf > 0 && itf < last) {
                    if (!VTI) *g0 = G0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                    else *g0 = G0 + gw * dtg * dl;
                    *g1 = G1 + gw * dtg * dm;
                    if (rho_here)
                        *g2 = (float)((double)(BAND ? hg2 : *g2) +
                                      wdt * (double)(n0 * (fp0 - 2 * f0 + fm0) + n1 * (fp1 - 2 * f1 + fm1)));
                } else if (itf == 0) {
                    const double wh = (double)gw * 0.5 * (double)dtg;
                    if (!VTI) *g0 = (float)((double)G0 + wh * (double)(ax0 + az1) * (double)(t0 + t1));
                    else *g0 = (float)((double)G0 + wh * (double)dl);
                    *g1 = (float)((double)G1 + wh * (double)dm);
                    *g2 = (float)((double)(BAND ? hg2 : *g2) + wdt * (double)(n0 * (fp0 - f0) + n1 * (fp1 - f1)));
                } else {
                    if (!VTI) *g0 = G0 + gw * dtg * (ax0 + az1) * (t0 + t1);
                    else *g0 = G0 + gw * dtg * dl;
                    *g1 = G1 + gw * dtg * dm;
                    if (rho_here)
                        *g2 = (float)((double)(BAND ? hg2 : *g2) + wdt * (double)(n0 * (-f0 + fm0) + n1 * (-f1 + fm1)));
                }
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
        if (threadIdx.x < 32) {
            m = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (threadIdx.x == 0 && m > 0.f) atomicMax(Sp->snap_amax + (it + 1) / C.sub, __float_as_uint(m));
        }
    }
}

}  // namespace fwi2d
#include "march.cuh"
#include "zband.cuh"
#include "xband.cuh"
#include "acoustic.cuh"
namespace fwi2d {

// ---------------------------------------------------------------------------
// Initial state (we_op.cpp:657-663): inject sample 0 into a zeroed field and
// scale by dt^2/(2 rho) in double.  One thread per touched cell, entries in
// the reference's order.
// ---------------------------------------------------------------------------
__global__ void init_state(const ShotDev *__restrict__ shots, int nshots, const InitCell *__restrict__ cells,
                           const int *__restrict__ off, const int *__restrict__ idx)
{
    const int s = blockIdx.x;
    if (s >= nshots) return;
    const ShotDev &S = shots[s];
    const long long nxz = (long long)S.nx * S.ldz;
    const float *src0 = S.src;   // time sample 0 of the time-major traces
    for (int c = off[s] + threadIdx.x; c < off[s + 1]; c += blockDim.x) {
        const InitCell q = cells[c];
        float acc = 0.f;
        for (int k = q.i0; k < q.i1; k++) {
            const InjEntry &E = S.inj[idx[k]];
            acc += E.mt ? (E.wa * src0[E.ia] - E.wb * src0[E.ib]) : E.wa * src0[E.ia];
        }
        S.u[0][q.comp * nxz + (long long)q.gx * S.ldz + q.gz] = (float)((double)acc * q.factor);
    }
}

// ---------------------------------------------------------------------------
// Last sample: receivers and the final snapshot (we_op.cpp:874-881).
// One CTA per shot.
// ---------------------------------------------------------------------------
__global__ void finalize_shots(const ShotDev *__restrict__ shots, int nshots, StepConst C, int ncomp, int flags,
                               int t_store)
{
    const int s = blockIdx.y;
    if (s >= nshots) return;
    const ShotDev &S = shots[s];
    // t_store >= 0: the field of that time sample (curr after launch t_store-1)
    const int it = t_store >= 0 ? t_store : S.nt - 1;
    if (it > S.nt - 1) return;
    const float *curr = S.u[(it + 1) & 1];
    const long long nxz = (long long)S.nx * S.ldz;
    if (flags & F_EXTRACT) {
        const int e1 = S.n_ext;
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
// Checkpoints of the time loop: both field buffers of every shot (the state
// before a given launch: prev and curr) copied to (restore = 0) or from
// (restore = 1) checkpoint k of the shot's store [k][2][ncomp][nx][ldz].
// ---------------------------------------------------------------------------
__global__ void checkpoint_fields(const ShotDev *__restrict__ shots, int nshots, int ncomp, int k, int restore)
{
    const int s = blockIdx.y;
    if (s >= nshots) return;
    const ShotDev &S = shots[s];
    const long long n4 = (long long)ncomp * S.nx * S.ldz / 4;   // ldz is a multiple of 32
    float4 *ck = reinterpret_cast<float4 *>(S.ckpt) + (long long)k * 2 * n4;
    for (int b = 0; b < 2; b++) {
        float4 *u = reinterpret_cast<float4 *>(S.u[b]);
        float4 *c = ck + b * n4;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
             i += (long long)gridDim.x * blockDim.x) {
            if (restore) u[i] = c[i];
            else c[i] = u[i];
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
    const float2 one = make_float2(1.f, 1.f);
    cudaMemcpyToSymbol(kOne2, &one, sizeof(one));
}

template <bool VTI, int RZ, int TX, bool GRAD, bool AE = false>
static constexpr size_t elastic_smem_bytes()
{
    constexpr int TZ = 32 * RZ, UZ = TZ + 8, UX = TX + 8, WZ = TZ + 4, WX = TX + 4;
    constexpr int own = RZ == 1 ? own_slots<VTI, GRAD>() * 32 * TX : 0;   // scalar interior path
    return sizeof(float) * (2 * UX * UZ + (5 + ((VTI || AE) ? 1 : 0) + (GRAD ? 2 : 0)) * WX * WZ + TX + own);
}

template <bool VTI, int RZ, int TX, bool GRAD, bool AE = false, bool CORE = false, bool BAND = false>
static void launch_elastic_g(const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                             const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    constexpr size_t bytes = elastic_smem_bytes<VTI, RZ, TX, GRAD, AE>();
    static bool configured = false;   // per process; a kernel attribute applies to every device
    if (!configured) {
        cudaFuncSetAttribute(elastic_step<VTI, RZ, TX, GRAD, AE, CORE, BAND>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        configured = true;
    }
    elastic_step<VTI, RZ, TX, GRAD, AE, CORE, BAND><<<ntiles, 32 * TX, bytes, st>>>(shots, tiles, M, C, it, flags,
                                                                                    dtg);
}

template <bool VTI, int RZ, int TX>
static void launch_elastic_t(const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M, const StepConst &C,
                             int it, int flags, float dtg, cudaStream_t st, bool core)
{
    if (core) {
        if (flags & F_GRAD) launch_elastic_g<VTI, RZ, TX, true, false, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
        else launch_elastic_g<VTI, RZ, TX, false, false, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
        return;
    }
    if (flags & F_GRAD) launch_elastic_g<VTI, RZ, TX, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
    else launch_elastic_g<VTI, RZ, TX, false>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
}

// tile shapes offered to the autotuner: (TZ, TX); TZ = 64 tiles take the lean interior path
int elastic_tile_count() { return 4; }
void elastic_tile_shape(int i, int *tz, int *tx)
{
    static const int s[4][2] = {{64, 16}, {64, 8}, {32, 16}, {32, 8}};
    *tz = s[i][0];
    *tx = s[i][1];
}

void launch_elastic_xband(bool vti, bool split, const ShotDev *shots, const TileRef *tiles, int ntiles,
                          const ModelDev &M, const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    if (ntiles <= 0) return;
    const bool grad = (flags & F_GRAD) != 0;
    if (split) {
        constexpr int nf = xband_threads<false>(), ng = xband_threads<true>();
        if (vti) {
            if (grad) elastic_xband<true, true><<<ntiles, ng, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
            else elastic_xband<true, false><<<ntiles, nf, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
        } else {
            if (grad) elastic_xband<false, true><<<ntiles, ng, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
            else elastic_xband<false, false><<<ntiles, nf, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
        }
        return;
    }
    if (vti) {
        if (grad) launch_elastic_g<true, 1, 8, true, false, false, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
        else launch_elastic_g<true, 1, 8, false, false, false, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
    } else {
        if (grad) launch_elastic_g<false, 1, 8, true, false, false, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
        else launch_elastic_g<false, 1, 8, false, false, false, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
    }
}

void launch_elastic_step(int shape, bool vti, const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                         const StepConst &C, int it, int flags, float dtg, cudaStream_t st, bool core)
{
    if (ntiles <= 0) return;
    switch (shape) {
    case 0: vti ? launch_elastic_t<true, 2, 16>(shots, tiles, ntiles, M, C, it, flags, dtg, st, core)
                : launch_elastic_t<false, 2, 16>(shots, tiles, ntiles, M, C, it, flags, dtg, st, core); break;
    case 1: vti ? launch_elastic_t<true, 2, 8>(shots, tiles, ntiles, M, C, it, flags, dtg, st, core)
                : launch_elastic_t<false, 2, 8>(shots, tiles, ntiles, M, C, it, flags, dtg, st, core); break;
    case 2: vti ? launch_elastic_t<true, 1, 16>(shots, tiles, ntiles, M, C, it, flags, dtg, st, core)
                : launch_elastic_t<false, 1, 16>(shots, tiles, ntiles, M, C, it, flags, dtg, st, core); break;
    default: vti ? launch_elastic_t<true, 1, 8>(shots, tiles, ntiles, M, C, it, flags, dtg, st, core)
                 : launch_elastic_t<false, 1, 8>(shots, tiles, ntiles, M, C, it, flags, dtg, st, core); break;
    }
}

template <bool VTI, bool GRAD, int NTH>
static void launch_march_n(const ShotDev *shots, const MarchRef *units, int nunits, const ModelDev &M,
                           const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    constexpr size_t bytes = sizeof(float) * MarchLayout<VTI, GRAD, NTH>::FLOATS;
    static bool configured = false;   // per process; a kernel attribute applies to every device
    if (!configured) {
        cudaFuncSetAttribute(elastic_march<VTI, GRAD, NTH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        configured = true;
    }
    elastic_march<VTI, GRAD, NTH><<<nunits, NTH, bytes, st>>>(shots, units, M, C, it, flags, dtg);
}

template <bool VTI, bool GRAD>
static void launch_march_g(const ShotDev *shots, const MarchRef *units, int nunits, int nth, const ModelDev &M,
                           const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    switch (nth) {
    case 128: launch_march_n<VTI, GRAD, 128>(shots, units, nunits, M, C, it, flags, dtg, st); break;
    case 192: launch_march_n<VTI, GRAD, 192>(shots, units, nunits, M, C, it, flags, dtg, st); break;
    case 224: launch_march_n<VTI, GRAD, 224>(shots, units, nunits, M, C, it, flags, dtg, st); break;
    default: launch_march_n<VTI, GRAD, 256>(shots, units, nunits, M, C, it, flags, dtg, st); break;
    }
}

bool march_threads_ok(int nth) { return nth == 128 || nth == 192 || nth == 224 || nth == 256; }

void launch_elastic_march(bool vti, const ShotDev *shots, const MarchRef *units, int nunits, int nth,
                          const ModelDev &M, const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    if (nunits <= 0) return;
    const bool grad = (flags & F_GRAD) != 0;
    if (vti) {
        if (grad) launch_march_g<true, true>(shots, units, nunits, nth, M, C, it, flags, dtg, st);
        else launch_march_g<true, false>(shots, units, nunits, nth, M, C, it, flags, dtg, st);
    } else {
        if (grad) launch_march_g<false, true>(shots, units, nunits, nth, M, C, it, flags, dtg, st);
        else launch_march_g<false, false>(shots, units, nunits, nth, M, C, it, flags, dtg, st);
    }
}

template <bool SPLIT>
static void launch_zband_s(bool vti, const BandRef *units, int nunits, const ShotDev *shots, const ModelDev &M,
                           const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    const bool grad = (flags & F_GRAD) != 0;
    if (vti) {
        if (grad) elastic_zband<true, true, SPLIT><<<nunits, kZbThreads, 0, st>>>(shots, units, M, C, it, flags, dtg);
        else elastic_zband<true, false, SPLIT><<<nunits, kZbThreads, 0, st>>>(shots, units, M, C, it, flags, dtg);
    } else {
        if (grad) elastic_zband<false, true, SPLIT><<<nunits, kZbThreads, 0, st>>>(shots, units, M, C, it, flags, dtg);
        else elastic_zband<false, false, SPLIT><<<nunits, kZbThreads, 0, st>>>(shots, units, M, C, it, flags, dtg);
    }
}

void launch_elastic_zband(bool vti, bool split, const BandRef *units, int nunits, const ShotDev *shots,
                          const ModelDev &M, const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    if (nunits <= 0) return;
    if (split) launch_zband_s<true>(vti, units, nunits, shots, M, C, it, flags, dtg, st);
    else launch_zband_s<false>(vti, units, nunits, shots, M, C, it, flags, dtg, st);
}

int zband_rows(bool split) { return split ? kZbSplitRows : kZbRows; }

// tile shapes of the acoustic kernel: (32, 16) and (32, 8), the elastic shapes 2 and 3
bool acoustic_shape_ok(int shape) { return shape == 2 || shape == 3; }

void launch_acoustic_step(int shape, const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                          const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    const bool grad = (flags & F_GRAD) != 0;
    if (shape == 2) {
        if (grad) acoustic_step<16, true, false><<<ntiles, 512, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
        else acoustic_step<16, false, false><<<ntiles, 512, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
    } else {
        if (grad) acoustic_step<8, true, false><<<ntiles, 256, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
        else acoustic_step<8, false, false><<<ntiles, 256, 0, st>>>(shots, tiles, M, C, it, flags, dtg);
    }
}

// Acoustic-elastic propagator: one step of the fluid layer (tile shape 2 or
// 3), of the elastic grid (tile shape 2 or 3, general path) and the interface
// coupling.
void launch_ae_fluid_step(int shape, const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                          const StepConst &C, int it, int flags, cudaStream_t st)
{
    if (shape == 2) acoustic_step<16, false, true><<<ntiles, 512, 0, st>>>(shots, tiles, M, C, it, flags, 1.f);
    else acoustic_step<8, false, true><<<ntiles, 256, 0, st>>>(shots, tiles, M, C, it, flags, 1.f);
}

void launch_ae_elastic_step(int shape, const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                            const StepConst &C, int it, int flags, float dtg, cudaStream_t st)
{
    const bool grad = (flags & F_GRAD) != 0;
    if (shape == 2) {
        if (grad) launch_elastic_g<false, 1, 16, true, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
        else launch_elastic_g<false, 1, 16, false, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
    } else {
        if (grad) launch_elastic_g<false, 1, 8, true, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
        else launch_elastic_g<false, 1, 8, false, true>(shots, tiles, ntiles, M, C, it, flags, dtg, st);
    }
}

void launch_ae_couple(const ShotDev *elastic, const ShotDev *fluid, int nshots, int nx_max, const ModelDev &M,
                      const StepConst &C, int it, int flags, float dtg, float Kw, float val0, int sign, cudaStream_t st)
{
    dim3 grid((nx_max + 127) / 128, nshots);
    ae_couple<<<grid, 128, 0, st>>>(elastic, fluid, nshots, M, C, it, flags, dtg, Kw, val0, sign);
}

void launch_acoustic_final_grad(const ShotDev *shots, int nshots, const ModelDev &M, const StepConst &C, float dtg,
                                cudaStream_t st)
{
    dim3 grid(148, nshots);
    acoustic_final_grad<<<grid, 256, 0, st>>>(shots, nshots, M, C, dtg);
}

void launch_init_state(const ShotDev *shots, int nshots, const InitCell *cells, const int *off, const int *idx,
                       cudaStream_t st)
{
    init_state<<<nshots, 128, 0, st>>>(shots, nshots, cells, off, idx);
}

void launch_finalize(const ShotDev *shots, int nshots, const StepConst &C, int ncomp, int flags, cudaStream_t st,
                     int t_store)
{
    dim3 grid(148, nshots);
    finalize_shots<<<grid, 256, 0, st>>>(shots, nshots, C, ncomp, flags, t_store);
}

void launch_checkpoint(const ShotDev *shots, int nshots, int ncomp, int k, bool restore, cudaStream_t st)
{
    dim3 grid(148, nshots);
    checkpoint_fields<<<grid, 256, 0, st>>>(shots, nshots, ncomp, k, restore ? 1 : 0);
}

void launch_vti_grad_coefs(int n, const float *lam, const float *mu, const float *c13, float *v2, float *v3, cudaStream_t st)
{
    vti_grad_coefs<<<296, 256, 0, st>>>(n, lam, mu, c13, v2, v3);
}

// Moves the marching kernel's timeout flag into *status (keeping the first
// row recorded) and clears the flag, in stream order.
__global__ void take_timeout(int *status)
{
    const int v = g_march_timeout;
    if (v != 0) {
        if (*status == 0) *status = v;
        g_march_timeout = 0;
    }
}

void launch_take_timeout(int *status, cudaStream_t st) { take_timeout<<<1, 1, 0, st>>>(status); }

}  // namespace fwi2d
