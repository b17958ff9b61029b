// Time-axis kernels of the FWI data path when the data are sampled on their
// own time axis (nd samples at dd) and the propagation runs at dt <= dd:
//   * the reference's windowed-sinc and linear resamplers, sinc_resampler and
//     linear_resampler (src/cpp/operator.cpp:755-856), forward (interpolation,
//     data axis -> propagation axis) and adjoint (propagation -> data);
//   * the receiver side of nl_we_op_e::apply_forward (we_op.cpp:1030-1054):
//     Dt of the extracted traces, the fluid sign of the acoustic-elastic
//     propagator, the rate ratio alpha = dt / dd;
//   * the residual, misfit and applyHt weighting of
//     nlls_fwi_eco::compute_res_and_grad on the data axis (optimization.hpp:
//     760-780, 937-951);
//   * the adjoint-source side of apply_jacobianT (we_op.cpp:1108-1124):
//     applyHt^-1, time reversal, -alpha, Dt^T and the fluid sign.
// Row-major trace blocks [rows][n] unless a name says time-major ([n][rows],
// the layout the step kernels read).  Each step keeps the reference's
// single-precision operation order and its double promotions.
#pragma once

#include <cuda_runtime.h>

namespace fwi2d {

// sinc(x) = sin(x)/x of a single-precision x, evaluated in double as the
// reference's unqualified sin of a float is (::sin(double), operator.cpp:755-758).
__device__ __forceinline__ float rs_sinc(float x)
{
    if (x == 0.0f) return 1.0f;
    return (float)(sin((double)x) / (double)x);
}

// sinc weight of domain sample itm for range time t (operator.cpp:822-823):
// the argument pi (t - itm dm) / dm and the cosine window a + (1-a) cos(pi
// (itm - t/dm) / hl) are formed in double from single-precision terms (M_PI is
// a double); a = 1/2.
__device__ __forceinline__ void rs_sinc_weight(float t, int itm, float dm, int hl, float &s, double &w)
{
    const double pi = 3.14159265358979323846;
    s = rs_sinc((float)(pi * (double)(t - itm * dm) / (double)dm));
    w = 0.5 + 0.5 * cos(pi * (double)(itm - t / dm) / hl);
}

// Forward resampling: in [rows][nm] on the domain axis (dm) -> out [rows][np]
// on the range axis (dp).  One thread per output sample; grid.y = rows.
__global__ void k_resample_fwd(const float *__restrict__ in, float *__restrict__ out, int nm, float dm, int np,
                               float dp, int hl, int linear)
{
    const int itd = blockIdx.x * blockDim.x + threadIdx.x;
    if (itd >= np) return;
    const float *pm = in + (size_t)blockIdx.y * nm;
    float v;
    if (linear) {
        // operator.cpp:772-777
        const float x = itd * dp / dm;
        const int i = min(nm - 1, (int)floorf(x)), j = min(nm - 1, (int)ceilf(x));
        const float wj = (itd * dp - i * dm) / dm, wi = 1 - wj;
        v = wi * pm[i] + wj * pm[j];
    } else {
        // operator.cpp:816-825
        const float t = itd * dp;
        const int itm0 = (int)floorf(t / dm);
        const int lo = max(0, itm0 - hl + 1), hi = min(nm - 1, itm0 + hl);
        v = 0.f;
        for (int itm = lo; itm <= hi; itm++) {
            float s;
            double w;
            rs_sinc_weight(t, itm, dm, hl, s, w);
            v = (float)((double)v + (double)(pm[itm] * s) * w);
        }
    }
    out[(size_t)blockIdx.y * np + itd] = v;
}

// Adjoint resampling: in [rows][np] on the range axis -> out [rows][nm] on the
// domain axis.  The reference scatters (pmod[itm] += ...) in ascending range
// sample order; here one thread per domain sample gathers the same terms in
// the same order, so no atomics and the same rounding.  grid.y = rows.
__global__ void k_resample_adj(const float *__restrict__ in, float *__restrict__ out, int nm, float dm, int np,
                               float dp, int hl, int linear)
{
    const int itm = blockIdx.x * blockDim.x + threadIdx.x;
    if (itm >= nm) return;
    const float *pd = in + (size_t)blockIdx.y * np;
    auto x_of = [&](int itd) { return itd * dp / dm; };
    float acc = 0.f;
    if (linear) {
        // operator.cpp:795-803: sample itd feeds i = min(nm-1, floor x) with wi
        // and j = min(nm-1, ceil x) with wj.  First itd that can reach itm:
        // j(itd) >= itm.
        auto jof = [&](int itd) { return min(nm - 1, (int)ceilf(x_of(itd))); };
        int itd = max(0, (int)floor((double)(itm - 1) * (double)dm / (double)dp) - 2);
        while (itd > 0 && jof(itd - 1) >= itm) itd--;
        for (; itd < np; itd++) {
            const float x = x_of(itd);
            const int i = min(nm - 1, (int)floorf(x)), j = min(nm - 1, (int)ceilf(x));
            if (i > itm) break;
            const float wj = (itd * dp - i * dm) / dm, wi = 1 - wj;
            if (i == itm) acc += wi * pd[itd];
            if (j == itm) acc += wj * pd[itd];
        }
    } else {
        // operator.cpp:845-852: sample itd feeds itm in [itm0 - hl + 1, itm0 + hl]
        // with itm0 = floor(itd dp / dm); itm0 never decreases with itd.
        auto m0 = [&](int itd) { return (int)floorf((itd * dp) / dm); };
        int itd = max(0, (int)floor((double)(itm - hl) * (double)dm / (double)dp) - 2);
        while (itd > 0 && m0(itd - 1) >= itm - hl) itd--;
        for (; itd < np; itd++) {
            const float t = itd * dp;
            const int i0 = (int)floorf(t / dm);
            if (i0 > itm + hl - 1) break;
            if (i0 < itm - hl) continue;
            float s;
            double w;
            rs_sinc_weight(t, itm, dm, hl, s, w);
            acc = (float)((double)acc + (double)(pd[itd] * s) * w);
        }
    }
    out[(size_t)blockIdx.y * nm + itm] = acc;
}

// Receiver side of apply_forward on the propagation axis: u time-major
// [nt][rows] (the extracted field) -> out [rows][nt] = alpha * Dt(u)
// (seismotype 1, misc.cpp:71-84; fluid rows [0, neg_rows) negated,
// we_op.cpp:1033-1040) or alpha * u (seismotype 0).  One thread per (row,
// sample).
__global__ void k_rcv_to_rate(const float *__restrict__ u, float *__restrict__ out, int rows, int nt, float dt,
                              float alpha, int seismotype, int neg_rows)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = blockIdx.y;
    if (r >= rows) return;
    auto U = [&](int k) { return u[(long long)k * rows + r]; };
    float v;
    if (!seismotype) v = U(t);
    else {
        if (t == 0) v = (U(1) - U(0)) / dt;
        else if (t == nt - 1) v = (U(nt - 1) - U(nt - 2)) / dt;
        else v = (U(t + 1) - U(t - 1)) / (2 * dt);
        if (r < neg_rows) v = v * -1.f;
    }
    out[(long long)r * nt + t] = v * alpha;
}

constexpr int kRsChunk = 64;

// Residual on the data axis (optimization.hpp:760-780): r = syn - obs on
// [rows][nd]; per (row, chunk of kRsChunk samples) the Neumaier-summed part
// of sum(r^2) - (r_0^2 + r_{nd-1}^2)/2 (getFunc, optimization.hpp:937-951);
// and w = applyHt(r) with the data step dd (misc.cpp:45-56: the end samples
// r * 0.5 * dd in double, the others r * dd).
__global__ void k_residual_axis(const float *__restrict__ syn, const float *__restrict__ obs,
                                float *__restrict__ w, float2 *__restrict__ part, int rows, int nd, float dd)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int t0 = blockIdx.y * kRsChunk, t1 = min(nd, t0 + kRsChunk);
    float sum = 0.f, comp = 0.f;
    for (int t = t0; t < t1; t++) {
        const long long i = (long long)r * nd + t;
        const float rv = syn[i] - obs[i];
        const bool end = t == 0 || t == nd - 1;
        float term = rv * rv;
        if (end) term = 0.5f * term;
        const float y = sum + term;
        if (fabsf(sum) >= fabsf(term)) comp += (sum - y) + term;
        else comp += (term - y) + sum;
        sum = y;
        w[i] = end ? (float)((double)rv * 0.5 * (double)dd) : rv * dd;
    }
    part[(long long)blockIdx.y * rows + r] = make_float2(sum, comp);
}

// Adjoint sources on the propagation axis (we_op.cpp:1108-1124): a [rows][nt]
// (the resampled, Ht-weighted residual) -> q time-major [nt][rows]:
//   b = applyHt^-1(a) with dt (misc.cpp:57-67: ends a / (0.5 dt) in double),
//   c[t] = -alpha * b[nt-1-t],
//   q = Dt^T(c) (misc.cpp:85-94) with the fluid rows negated (seismotype 1),
//   or q = c (seismotype 0).
__global__ void k_adjoint_source_axis(const float *__restrict__ a, float *__restrict__ q, int rows, int nt, float dt,
                                      float alpha, int seismotype, int neg_rows)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = blockIdx.y;
    if (r >= rows) return;
    const float *ar = a + (long long)r * nt;
    const float nalpha = -alpha;
    auto c = [&](int k) {
        const int s = nt - 1 - k;
        const float b = (s == 0 || s == nt - 1) ? (float)((double)ar[s] / (0.5 * (double)dt)) : ar[s] / dt;
        return b * nalpha;
    };
    float v;
    if (!seismotype) v = c(t);
    else {
        if (t == 0) v = (c(1) + c(0)) / dt;
        else if (t == nt - 1) v = (-c(nt - 1) - c(nt - 2)) / dt;
        else v = (c(t + 1) - c(t - 1)) / (2 * dt);
        if (r < neg_rows) v = v * -1.f;
    }
    q[(long long)t * rows + r] = v;
}

}  // namespace fwi2d
