// C++ restatement of the six SIMD loops of the reference's
// src/cpp/spatial_operators.ispc:7-68 (ISPC is not installed here).  Same
// signatures and single-precision arithmetic order as the ISPC source; no FMA
// contraction (x86-64 baseline target).
#include <cmath>
#ifdef DOUBLE_PRECISION
typedef double real_t;
#else
typedef float real_t;
#endif

static const real_t kC0 = (real_t)(2.0 / 3);
static const real_t kC1 = (real_t)(-1.0 / 12);

extern "C" {

void Dz_ispc(int add, const real_t *v, real_t *out, real_t scale, int col, int lo, int hi)
{
    for (int j = lo; j < hi; j++) {
        const real_t *c = v + col + j;
        out[col + j] = add * out[col + j] + scale * (kC0 * (c[1] - c[-1]) + kC1 * (c[2] - c[-2]));
    }
}

void Dx_ispc(int add, const real_t *v, real_t *out, real_t scale, int row, int n, int lo, int hi)
{
    for (int j = lo; j < hi; j++) {
        real_t dp1 = v[(row + 1) * n + j] - v[(row - 1) * n + j];
        real_t dp2 = v[(row + 2) * n + j] - v[(row - 2) * n + j];
        out[row * n + j] = add * out[row * n + j] + scale * (kC0 * dp1 + kC1 * dp2);
    }
}

void mult_Dz_ispc(int add, const real_t *v, real_t *out, real_t scale, int col, int lo, int hi, const real_t *p)
{
    for (int j = lo; j < hi; j++) {
        int i = col + j;
        out[i] = add * out[i] + scale * (kC0 * (v[i + 1] * p[i + 1] - v[i - 1] * p[i - 1])
                                       + kC1 * (v[i + 2] * p[i + 2] - v[i - 2] * p[i - 2]));
    }
}

void mult_Dx_ispc(int add, const real_t *v, real_t *out, real_t scale, int row, int n, int lo, int hi, const real_t *p)
{
    for (int j = lo; j < hi; j++) {
        int a = (row + 1) * n + j, b = (row - 1) * n + j, c = (row + 2) * n + j, d = (row - 2) * n + j;
        out[row * n + j] = add * out[row * n + j] + scale * (kC0 * (v[a] * p[a] - v[b] * p[b]) + kC1 * (v[c] * p[c] - v[d] * p[d]));
    }
}

void taperz_ispc(real_t *u, int col, int istart, int iend, real_t a)
{
    const real_t pi = (real_t)M_PI, half = (real_t)0.5;
    if (iend > istart) {
        for (int i = istart; i < iend; i++) {
            real_t c = std::cos(a * half * pi * (real_t)(i - istart) / (real_t)(iend - istart));
            u[col + i] *= c * c;
        }
    } else {
        for (int i = iend; i < istart; i++) {
            real_t c = std::cos(a * half * pi * (real_t)(i + 1 - istart) / (real_t)(iend - istart));
            u[col + i] *= c * c;
        }
    }
}

void taperx_ispc(real_t *u, int col, int n, int lo, int hi, real_t a)
{
    (void)n;
    for (int j = lo; j < hi; j++) u[col + j] = a * a * u[col + j];
}

}
