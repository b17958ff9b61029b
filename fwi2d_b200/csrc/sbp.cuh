// SBP operator building blocks on shared-memory tiles.
//
// Every routine restates one reference operator at a single sample, in the
// same single-precision operation order (this library is compiled with
// --fmad=false so that no multiply-add is contracted):
//   d1    Dx/Dz              src/cpp/spatial_operators.cpp:100-154 + .ispc:7-25
//   md1   mult_Dx/mult_Dz    src/cpp/spatial_operators.cpp:156-210 + .ispc:27-45
//   d2acc Dxx_var/Dzz_var    src/include/spatial_operators.hpp:31-156
//   tsum / nsum              the boundary sums of esat_* (spatial_operators.hpp:160-727)
// A pointer `p` addresses the sample being evaluated inside a tile, `st` is
// the tile stride along the derivative axis, `g` the global index of the
// sample on that axis and `n` the axis length.
#pragma once
#include <cuda_runtime.h>

namespace fwi2d {

// Coefficient tables, one copy in the single translation unit that holds the
// kernels (kernels.cu); upload_sbp_tables() fills them per device from the
// same rationals as the reference's initialisers.
static __constant__ float kB1[4][6];      // first-derivative boundary closure
static __constant__ float kB2[6][8][8];   // variable-coefficient second-derivative closure
static __constant__ float kC2[10];        // its interior weights
static __constant__ float kC1[2];         // 2/3, -1/12
static __constant__ float kSC[4];         // one-sided boundary derivative 11/6, -3, 3/2, -1/3
static __constant__ float kHC[4];         // H-norm boundary weights 17/48, 59/48, 43/48, 49/48
static __constant__ float2 kOne2;         // (1, 1), set at run time: the packed sums' multiplier (add2)

__device__ __forceinline__ float d1(const float *p, int st, int g, int n, float d, float scale)
{
    if (g < 4) {
        const float *b = p - g * st;
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 6; k++) s += kB1[g][k] * b[k * st];
        return s / d;
    }
    if (g >= n - 4) {
        const int r = n - 1 - g;
        const float *b = p + r * st;
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 6; k++) s -= kB1[r][k] * b[-k * st];
        return s / d;
    }
    return scale * (kC1[0] * (p[st] - p[-st]) + kC1[1] * (p[2 * st] - p[-2 * st]));
}

__device__ __forceinline__ float md1(const float *p, const float *q, int st, int g, int n, float ad)
{
    if (g < 4) {
        const float *b = p - g * st, *c = q - g * st;
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 6; k++) s += kB1[g][k] * b[k * st] * c[k * st];
        return ad * s;
    }
    if (g >= n - 4) {
        const int r = n - 1 - g;
        const float *b = p + r * st, *c = q + r * st;
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 6; k++) s -= kB1[r][k] * b[-k * st] * c[-k * st];
        return ad * s;
    }
    return ad * (kC1[0] * (p[st] * q[st] - p[-st] * q[-st]) + kC1[1] * (p[2 * st] * q[2 * st] - p[-2 * st] * q[-2 * st]));
}

// acc += D2(f, u) at one sample.  fs scales every coefficient sample
// (1 or exactly 2: the reference's expr4b = 2*mu is an exact doubling).
__device__ __forceinline__ void d2acc(float &acc, const float *pu, int su, const float *pf, int sf, float fs,
                                      int g, int n, float invd2, float d2)
{
    if (g < 6 || g >= n - 6) {
        const bool top = g < 6;
        const int r = top ? g : n - 1 - g;
        const int dir = top ? 1 : -1;
        const float *bu = top ? pu - g * su : pu + r * su;
        const float *bf = top ? pf - g * sf : pf + r * sf;
        float fk[8];
#pragma unroll
        for (int k = 0; k < 8; k++) fk[k] = fs * bf[dir * k * sf];
        // rolled over the eight samples (the unrolled closure overflows the
        // instruction cache of the latency-bound band kernels)
#pragma unroll 1
        for (int jj = 0; jj < 8; jj++) {
            float val = 0.f;
#pragma unroll
            for (int k = 0; k < 8; k++) val += kB2[r][jj][k] * fk[k];
            acc += val * bu[dir * jj * su] / d2;
        }
        return;
    }
    const float fm2 = fs * pf[-2 * sf], fm1 = fs * pf[-sf], f0 = fs * pf[0], fp1 = fs * pf[sf], fp2 = fs * pf[2 * sf];
    const float um2 = pu[-2 * su], um1 = pu[-su], u0 = pu[0], up1 = pu[su], up2 = pu[2 * su];
    acc = acc + invd2 * ((kC2[0] * f0 + kC2[1] * (fm1 + fp1) + kC2[2] * (fm2 + fp2)) * u0
                       + (kC2[3] * fm2 + kC2[4] * fm1 + kC2[5] * f0 + kC2[6] * fp1) * um1
                       + (kC2[3] * fp2 + kC2[4] * fp1 + kC2[5] * f0 + kC2[6] * fm1) * up1
                       + (kC2[7] * fm2 + kC2[8] * fm1 + kC2[9] * f0) * um2
                       + (kC2[7] * fp2 + kC2[8] * fp1 + kC2[9] * f0) * up2);
}

// Tangential first-derivative sum along a boundary line (no division by d).
__device__ __forceinline__ float tsum(const float *p, int st, int g, int n)
{
    float s = 0.f;
    if (g < 4) {
        const float *b = p - g * st;
#pragma unroll
        for (int j = 0; j < 6; j++) s += kB1[g][j] * b[j * st];
    } else if (g >= n - 4) {
        const int r = n - 1 - g;
        const float *b = p + r * st;
#pragma unroll
        for (int j = 0; j < 6; j++) s -= kB1[r][j] * b[-j * st];
    } else {
        s += kC1[0] * (p[st] - p[-st]);
        s += kC1[1] * (p[2 * st] - p[-2 * st]);
    }
    return s;
}

// One-sided outward derivative sum S.u at a boundary sample; `in` is the
// stride pointing into the domain.
__device__ __forceinline__ float nsum(const float *p, int in)
{
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) s += kSC[k] * p[k * in];
    return s;
}

// -(D u)_0 at a boundary sample: the sum of esat_Dz_top & co.
__device__ __forceinline__ float ndsum(const float *p, int in)
{
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 6; j++) s -= kB1[0][j] * p[j * in];
    return s;
}

}  // namespace fwi2d

namespace fwi2d {

// ---------------------------------------------------------------------------
// Interior forms (no boundary band within reach), same arithmetic as above.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float d1i(const float *p, int st, float scale)
{
    return scale * (kC1[0] * (p[st] - p[-st]) + kC1[1] * (p[2 * st] - p[-2 * st]));
}

__device__ __forceinline__ float md1i(const float *p, const float *q, int st, float ad)
{
    return ad * (kC1[0] * (p[st] * q[st] - p[-st] * q[-st]) + kC1[1] * (p[2 * st] * q[2 * st] - p[-2 * st] * q[-2 * st]));
}

// The five coefficient brackets of the interior Dxx_var/Dzz_var stencil for
// the samples u0, u-1, u+1, u-2, u+2.  They depend on the coefficient only,
// so one set serves every field differentiated with the same coefficient;
// scaling the coefficient by 2 (expr4b = 2 mu) scales each bracket by exactly 2.
struct Brk {
    float b0, bm1, bp1, bm2, bp2;
};

__device__ __forceinline__ Brk brackets(const float *pf, int sf)
{
    const float fm2 = pf[-2 * sf], fm1 = pf[-sf], f0 = pf[0], fp1 = pf[sf], fp2 = pf[2 * sf];
    Brk b;
    b.b0 = kC2[0] * f0 + kC2[1] * (fm1 + fp1) + kC2[2] * (fm2 + fp2);
    b.bm1 = kC2[3] * fm2 + kC2[4] * fm1 + kC2[5] * f0 + kC2[6] * fp1;
    b.bp1 = kC2[3] * fp2 + kC2[4] * fp1 + kC2[5] * f0 + kC2[6] * fm1;
    b.bm2 = kC2[7] * fm2 + kC2[8] * fm1 + kC2[9] * f0;
    b.bp2 = kC2[7] * fp2 + kC2[8] * fp1 + kC2[9] * f0;
    return b;
}

__device__ __forceinline__ Brk twice(const Brk &a)
{
    Brk b;
    b.b0 = 2.f * a.b0;
    b.bm1 = 2.f * a.bm1;
    b.bp1 = 2.f * a.bp1;
    b.bm2 = 2.f * a.bm2;
    b.bp2 = 2.f * a.bp2;
    return b;
}

// acc + (1/d^2) * (b0 u0 + b-1 u-1 + b+1 u+1 + b-2 u-2 + b+2 u+2)
__device__ __forceinline__ float d2i(float acc, const Brk &b, const float *pu, int su, float invd2)
{
    return acc + invd2 * (b.b0 * pu[0] + b.bm1 * pu[-su] + b.bp1 * pu[su] + b.bm2 * pu[-2 * su] + b.bp2 * pu[2 * su]);
}

}  // namespace fwi2d

namespace fwi2d {

// Scalar-argument interior forms for register-resident samples (the lean
// path of the step kernels); arithmetic identical to d1i / md1i / d2i.
__device__ __forceinline__ float d1s(float vm2, float vm1, float vp1, float vp2, float scale)
{
    return scale * (kC1[0] * (vp1 - vm1) + kC1[1] * (vp2 - vm2));
}

__device__ __forceinline__ float md1s(float pm2, float qm2, float pm1, float qm1, float pp1, float qp1, float pp2,
                                      float qp2, float ad)
{
    return ad * (kC1[0] * (pp1 * qp1 - pm1 * qm1) + kC1[1] * (pp2 * qp2 - pm2 * qm2));
}

__device__ __forceinline__ Brk brk5(float fm2, float fm1, float f0, float fp1, float fp2)
{
    Brk b;
    b.b0 = kC2[0] * f0 + kC2[1] * (fm1 + fp1) + kC2[2] * (fm2 + fp2);
    b.bm1 = kC2[3] * fm2 + kC2[4] * fm1 + kC2[5] * f0 + kC2[6] * fp1;
    b.bp1 = kC2[3] * fp2 + kC2[4] * fp1 + kC2[5] * f0 + kC2[6] * fm1;
    b.bm2 = kC2[7] * fm2 + kC2[8] * fm1 + kC2[9] * f0;
    b.bp2 = kC2[7] * fp2 + kC2[8] * fp1 + kC2[9] * f0;
    return b;
}

__device__ __forceinline__ float d2s(float acc, const Brk &b, float um2, float um1, float u0, float up1, float up2,
                                     float invd2)
{
    return acc + invd2 * (b.b0 * u0 + b.bm1 * um1 + b.bp1 * up1 + b.bm2 * um2 + b.bp2 * up2);
}

}  // namespace fwi2d

namespace fwi2d {

// ---------------------------------------------------------------------------
// Packed pairs of samples (sm_100 f32x2 arithmetic): each lane is rounded to
// nearest on its own, exactly as the scalar operation on that lane, so a pair
// of neighbouring cells evaluated with these forms gives the scalar forms'
// results bit for bit with half the floating-point instructions.  The
// operation order of every form is that of its scalar counterpart above.
//
// The assembler fuses a packed multiply into a packed add that consumes it
// (one rounding instead of two) even with an explicit .rn and --fmad=false,
// which would break the bitwise match with the reference.  A packed sum is
// therefore an fma.rn.f32x2 with the multiplier kOne2, which is (1, 1) at run
// time but unknown to the assembler: 1 * x + y rounds once, to x + y, and
// there is no product left to fuse.  It costs one instruction, as the add.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    float2 r;
    const float2 one = kOne2;
    asm("{\n .reg .b64 po, pa, pb, pd;\n mov.b64 po, {%2, %3};\n mov.b64 pa, {%4, %5};\n"
        " mov.b64 pb, {%6, %7};\n fma.rn.f32x2 pd, po, pa, pb;\n mov.b64 {%0, %1}, pd;\n}\n"
        : "=f"(r.x), "=f"(r.y)
        : "f"(one.x), "f"(one.y), "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b)
{
    float2 r;
    asm("{\n .reg .b64 pa, pb, pd;\n mov.b64 pa, {%2, %3};\n mov.b64 pb, {%4, %5};\n"
        " mul.rn.f32x2 pd, pa, pb;\n mov.b64 {%0, %1}, pd;\n}\n"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
// a - b == a + (-b) exactly in IEEE arithmetic
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return add2(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
// the pair shifted by one cell: (a.y, b.x) from the pairs (a) and (b) that follow each other
__device__ __forceinline__ float2 zsh(float2 a, float2 b) { return make_float2(a.y, b.x); }

__device__ __forceinline__ float2 d1s2(float2 vm2, float2 vm1, float2 vp1, float2 vp2, float scale)
{
    return mul2(bc2(scale), add2(mul2(bc2(kC1[0]), sub2(vp1, vm1)), mul2(bc2(kC1[1]), sub2(vp2, vm2))));
}

__device__ __forceinline__ float2 md1s2(float2 pm2, float2 qm2, float2 pm1, float2 qm1, float2 pp1, float2 qp1,
                                        float2 pp2, float2 qp2, float ad)
{
    return mul2(bc2(ad), add2(mul2(bc2(kC1[0]), sub2(mul2(pp1, qp1), mul2(pm1, qm1))),
                              mul2(bc2(kC1[1]), sub2(mul2(pp2, qp2), mul2(pm2, qm2)))));
}

struct Brk2 {
    float2 b0, bm1, bp1, bm2, bp2;
};

__device__ __forceinline__ Brk2 brk52(float2 fm2, float2 fm1, float2 f0, float2 fp1, float2 fp2)
{
    Brk2 b;
    b.b0 = add2(add2(mul2(bc2(kC2[0]), f0), mul2(bc2(kC2[1]), add2(fm1, fp1))), mul2(bc2(kC2[2]), add2(fm2, fp2)));
    b.bm1 = add2(add2(add2(mul2(bc2(kC2[3]), fm2), mul2(bc2(kC2[4]), fm1)), mul2(bc2(kC2[5]), f0)),
                 mul2(bc2(kC2[6]), fp1));
    b.bp1 = add2(add2(add2(mul2(bc2(kC2[3]), fp2), mul2(bc2(kC2[4]), fp1)), mul2(bc2(kC2[5]), f0)),
                 mul2(bc2(kC2[6]), fm1));
    b.bm2 = add2(add2(mul2(bc2(kC2[7]), fm2), mul2(bc2(kC2[8]), fm1)), mul2(bc2(kC2[9]), f0));
    b.bp2 = add2(add2(mul2(bc2(kC2[7]), fp2), mul2(bc2(kC2[8]), fp1)), mul2(bc2(kC2[9]), f0));
    return b;
}

__device__ __forceinline__ Brk2 twice2(const Brk2 &a)
{
    Brk2 b;
    b.b0 = mul2(bc2(2.f), a.b0);
    b.bm1 = mul2(bc2(2.f), a.bm1);
    b.bp1 = mul2(bc2(2.f), a.bp1);
    b.bm2 = mul2(bc2(2.f), a.bm2);
    b.bp2 = mul2(bc2(2.f), a.bp2);
    return b;
}

__device__ __forceinline__ float2 d2s2(float2 acc, const Brk2 &b, float2 um2, float2 um1, float2 u0, float2 up1,
                                       float2 up2, float invd2)
{
    const float2 s = add2(add2(add2(add2(mul2(b.b0, u0), mul2(b.bm1, um1)), mul2(b.bp1, up1)), mul2(b.bm2, um2)),
                          mul2(b.bp2, up2));
    return add2(acc, mul2(bc2(invd2), s));
}

}  // namespace fwi2d
