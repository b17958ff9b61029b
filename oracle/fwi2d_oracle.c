/*
 * fwi2d oracle -- CPU restatement of the reference's SBP time loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * fwi2d_b200: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference legs of bench.py may load it.  The product never links or calls
 * it, and has no CPU fallback through it.
 *
 * It restates, in plain C and in the same floating-point operation order, the
 * single-precision CPU path of nmbader/fwi2d for the propagators on the hot
 * path (version-2 operator split):
 *   - elastic isotropic   nl_we_op_e::propagate          src/cpp/we_op.cpp:564-902
 *   - elastic VTI         nl_we_op_vti::propagate        src/cpp/we_op.cpp:1559-1861
 *   - acoustic            nl_we_op_a::propagate          src/cpp/we_op.cpp:1937-2134
 *   - acoustic-elastic    nl_we_op_ae::propagate         src/cpp/we_op.cpp:2137-2577
 * with their imaging conditions (compute_gradients, we_op.cpp:505-562,
 * 1478-1557, 1883-1935), the SBP operators of src/include/spatial_operators.hpp
 * and src/cpp/spatial_operators.cpp, the ISPC interior loops of
 * src/cpp/spatial_operators.ispc, and the injectors of src/cpp/injector.cpp.
 *
 * Built twice: with -DORACLE_DOUBLE (the FP64 error oracle, as the reference's
 * ENABLE_DOUBLE_PRECISION build) and without (FP32 parity oracle).
 *
 * Pinned against the reference itself: tests/golden/ holds outputs of the
 * reference sources compiled here (oracle/build_ref.sh), and the
 * "not gpu" tests check this restatement against them.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_DOUBLE
typedef double real;
#define R_SQRT sqrt
#define R_COS cos
#define ORC(name) orc64_##name
#else
typedef float real;
#define R_SQRT sqrtf
#define R_COS cosf
#define ORC(name) orc32_##name
#endif

#ifdef _OPENMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

/* ---------------------------------------------------------------------------
 * ABI structs (shared by the float and the double build: reals are double).
 * ------------------------------------------------------------------------- */
typedef struct {
    int type;          /* 0: 3x3 discrete delta (delta_m3), 1: moment-tensor (ddelta_m3) */
    int ntr;
    const int *xind;   /* [ntr][3] */
    const int *zind;   /* [ntr][3] */
    const void *xw;    /* real [ntr][2][3] (type 0) or [ntr][2][6] (type 1) */
    const void *zw;
} orc_injector;

typedef struct {
    int nt, sub;
    double dt;
    int ns, nr;                       /* trace counts of the source / receiver blocks */
    int bc_top, bc_bottom, bc_left, bc_right;
    int taper_top, taper_bottom, taper_left, taper_right;
    double taper_strength, free_surface_stiffness;
    int mt;
    double gdamp_tmin, gdamp_tmax, gdamp_power;
    int nza;                          /* acoustic-elastic: water rows */
    double water_velocity, water_density;
    int acoustic_source;
} orc_param;

/* ---------------------------------------------------------------------------
 * SBP coefficient tables.  Values are the reference's (spatial_operators.hpp:
 * 34-41 and spatial_operators.cpp:102,129), each a rational evaluated in double
 * and rounded to `real`, exactly as the reference's constant initialisers.
 * ------------------------------------------------------------------------- */
typedef struct { int r, j, k; long long num, den; } q_entry;

/* 4x6 first-derivative boundary closure (rows 0..3). */
static const q_entry D1_Q[] = {
    {0,0,0,-24,17},{0,0,1,59,34},{0,0,2,-4,17},{0,0,3,-3,34},
    {0,1,0,-1,2},{0,1,2,1,2},
    {0,2,0,4,43},{0,2,1,-59,86},{0,2,3,59,86},{0,2,4,-4,43},
    {0,3,0,3,98},{0,3,2,-59,98},{0,3,4,32,49},{0,3,5,-4,49},
};
/* 6x8x8 variable-coefficient second-derivative boundary closure (nonzeros). */
static const q_entry D2_Q[] = {
    {0,0,0,920LL,289LL},
    {0,0,1,-59LL,68LL},
    {0,0,2,-7549318LL,34157643LL},
    {0,0,3,-17440994LL,184112825LL},
    {0,1,0,-1740LL,289LL},
    {0,1,2,295314153LL,366719282LL},
    {0,1,3,262545878LL,1218454145LL},
    {0,2,0,1128LL,289LL},
    {0,2,1,59LL,68LL},
    {0,2,2,-19250923LL,26254840LL},
    {0,2,3,-12192537LL,324892213LL},
    {0,3,0,-308LL,289LL},
    {0,3,2,42283069LL,254173229LL},
    {0,3,3,-43013531LL,427521546LL},
    {0,4,2,-18700293LL,1355757959LL},
    {0,4,3,18700293LL,1355757959LL},
    {0,5,2,-3LL,833LL},
    {0,5,3,3LL,833LL},
    {1,0,0,12LL,17LL},
    {1,0,2,89562243LL,385991318LL},
    {1,0,3,16914691LL,272440171LL},
    {1,1,0,-59LL,68LL},
    {1,1,2,-47979680LL,48852831LL},
    {1,1,3,-18034913LL,120051851LL},
    {1,2,0,2LL,17LL},
    {1,2,2,299262497LL,373256703LL},
    {1,2,3,16156647LL,200473586LL},
    {1,3,0,3LL,68LL},
    {1,3,2,-14723969LL,177744748LL},
    {1,3,3,22633571LL,584543661LL},
    {1,4,2,46802031LL,1628311862LL},
    {1,4,3,-46802031LL,1628311862LL},
    {1,5,2,441LL,181507LL},
    {1,5,3,-441LL,181507LL},
    {2,0,0,-96LL,731LL},
    {2,0,1,59LL,172LL},
    {2,0,2,-47632751LL,164317197LL},
    {2,0,3,-5570723LL,375470930LL},
    {2,1,0,118LL,731LL},
    {2,1,2,54282598LL,49343777LL},
    {2,1,3,23802793LL,215253532LL},
    {2,2,0,-16LL,731LL},
    {2,2,1,-59LL,172LL},
    {2,2,2,-39119273LL,25083370LL},
    {2,2,3,-35971870LL,61324629LL},
    {2,2,4,-26254LL,557679LL},
    {2,3,0,-6LL,731LL},
    {2,3,2,360454121LL,368940022LL},
    {2,3,3,17254963LL,80047776LL},
    {2,3,4,1500708LL,7993399LL},
    {2,4,2,-18024731LL,79673021LL},
    {2,4,3,24178273LL,88099647LL},
    {2,4,4,-26254LL,185893LL},
    {2,5,2,-870707LL,620833782LL},
    {2,5,3,960119LL,1147305747LL},
    {2,5,4,13564LL,23980197LL},
    {3,0,0,-36LL,833LL},
    {3,0,2,54741803LL,948483020LL},
    {3,0,3,-13602043LL,389676498LL},
    {3,1,0,177LL,3332LL},
    {3,1,2,-35820026LL,359121865LL},
    {3,1,3,24921773LL,534548210LL},
    {3,2,0,-6LL,833LL},
    {3,2,2,813284372LL,948584067LL},
    {3,2,3,30057666LL,158897885LL},
    {3,2,4,1500708LL,9108757LL},
    {3,3,0,-9LL,3332LL},
    {3,3,2,-95056924LL,90903639LL},
    {3,3,3,-23417695LL,47008088LL},
    {3,3,4,-7476412LL,9108757LL},
    {3,3,5,-2LL,49LL},
    {3,4,2,23159719LL,99948527LL},
    {3,4,3,110687545LL,265515812LL},
    {3,4,4,4502124LL,9108757LL},
    {3,4,5,8LL,49LL},
    {3,5,2,-3671038LL,2687426923LL},
    {3,5,3,-1063649LL,8893843LL},
    {3,5,4,1473580LL,9108757LL},
    {3,5,5,-6LL,49LL},
    {4,0,2,-9437957LL,1931986386LL},
    {4,0,3,9437957LL,1931986386LL},
    {4,1,2,17289851LL,489388053LL},
    {4,1,3,-17289851LL,489388053LL},
    {4,2,2,-66355919LL,327412264LL},
    {4,2,3,24178273LL,98343792LL},
    {4,2,4,-564461LL,4461432LL},
    {4,3,2,17638343LL,74566894LL},
    {4,3,3,103749401LL,243793650LL},
    {4,3,4,375177LL,743572LL},
    {4,3,5,1LL,6LL},
    {4,4,2,-19321801LL,295845927LL},
    {4,4,3,-50677283LL,62943042LL},
    {4,4,4,-280535LL,371786LL},
    {4,4,5,-5LL,6LL},
    {4,4,6,-1LL,24LL},
    {4,5,2,5130905LL,5183662662LL},
    {4,5,3,35039615LL,213452232LL},
    {4,5,4,1118749LL,2230716LL},
    {4,5,5,1LL,2LL},
    {4,5,6,1LL,6LL},
    {4,6,4,-1LL,8LL},
    {4,6,5,1LL,6LL},
    {4,6,6,-1LL,8LL},
    {5,0,2,-1LL,784LL},
    {5,0,3,1LL,784LL},
    {5,1,2,8673LL,2904112LL},
    {5,1,3,-8673LL,2904112LL},
    {5,2,2,-403062LL,320810033LL},
    {5,2,3,960119LL,1280713392LL},
    {5,2,4,3391LL,6692148LL},
    {5,3,2,-1920494LL,1377228165LL},
    {5,3,3,-1063649LL,8712336LL},
    {5,3,4,368395LL,2230716LL},
    {5,3,5,-1LL,8LL},
    {5,4,2,5130905LL,5183662662LL},
    {5,4,3,35039615LL,213452232LL},
    {5,4,4,1118749LL,2230716LL},
    {5,4,5,1LL,2LL},
    {5,4,6,1LL,6LL},
    {5,5,2,-117380LL,2351569839LL},
    {5,5,3,-3290636LL,80044587LL},
    {5,5,4,-5580181LL,6692148LL},
    {5,5,5,-3LL,4LL},
    {5,5,6,-5LL,6LL},
    {5,5,7,-1LL,24LL},
    {5,6,4,1LL,6LL},
    {5,6,5,1LL,2LL},
    {5,6,6,1LL,2LL},
    {5,6,7,1LL,6LL},
    {5,7,5,-1LL,8LL},
    {5,7,6,1LL,6LL},
    {5,7,7,-1LL,8LL}
};

static real B1[4][6];
static real B2[6][8][8];
static real C2[10];
static real C1[2];
static real SC[4];
static real HC[4];
static real H0;
static int tables_ready = 0;

static void init_tables(void)
{
    if (tables_ready) return;
    memset(B1, 0, sizeof(B1));
    memset(B2, 0, sizeof(B2));
    for (size_t i = 0; i < sizeof(D1_Q) / sizeof(D1_Q[0]); i++)
        B1[D1_Q[i].j][D1_Q[i].k] = (real)((double)D1_Q[i].num / (double)D1_Q[i].den);
    for (size_t i = 0; i < sizeof(D2_Q) / sizeof(D2_Q[0]); i++)
        B2[D2_Q[i].r][D2_Q[i].j][D2_Q[i].k] = (real)((double)D2_Q[i].num / (double)D2_Q[i].den);
    const double c2[10] = {-3.0/4, -5.0/6, -1.0/24, 1.0/6, 1.0/2, 1.0/2, 1.0/6, -1.0/8, 1.0/6, -1.0/8};
    for (int i = 0; i < 10; i++) C2[i] = (real)c2[i];
    C1[0] = (real)(2.0/3); C1[1] = (real)(-1.0/12);
    SC[0] = (real)(11.0/6); SC[1] = (real)-3; SC[2] = (real)1.5; SC[3] = (real)(-1.0/3);
    HC[0] = (real)(17.0/48); HC[1] = (real)(59.0/48); HC[2] = (real)(43.0/48); HC[3] = (real)(49.0/48);
    H0 = (real)(17.0/48);
    tables_ready = 1;
}

/* ---------------------------------------------------------------------------
 * 1-D SBP operators on a strided line of n samples (z: stride 1, x: stride nz).
 * ------------------------------------------------------------------------- */

/* first derivative: spatial_operators.cpp:100-154 + spatial_operators.ispc:7-25 */
static inline real d1_at(const real *v, long st, int n, int j, real d, real scale)
{
    if (j < 4) {
        real s = 0;
        for (int k = 0; k < 6; k++) s += B1[j][k] * v[k * st];
        return s / d;
    }
    if (j >= n - 4) {
        int r = n - 1 - j;
        real s = 0;
        for (int k = 0; k < 6; k++) s -= B1[r][k] * v[(long)(n - 1 - k) * st];
        return s / d;
    }
    return scale * (C1[0] * (v[(j + 1) * st] - v[(j - 1) * st]) + C1[1] * (v[(j + 2) * st] - v[(j - 2) * st]));
}

/* D(par * in): spatial_operators.cpp:156-210 + spatial_operators.ispc:27-45 */
static inline real md1_at(const real *v, const real *p, long st, int n, int j, real ad)
{
    if (j < 4) {
        real s = 0;
        for (int k = 0; k < 6; k++) s += B1[j][k] * v[k * st] * p[k * st];
        return ad * s;
    }
    if (j >= n - 4) {
        int r = n - 1 - j;
        real s = 0;
        for (int k = 0; k < 6; k++) {
            long q = (long)(n - 1 - k) * st;
            s -= B1[r][k] * v[q] * p[q];
        }
        return ad * s;
    }
    return ad * (C1[0] * (v[(j + 1) * st] * p[(j + 1) * st] - v[(j - 1) * st] * p[(j - 1) * st])
               + C1[1] * (v[(j + 2) * st] * p[(j + 2) * st] - v[(j - 2) * st] * p[(j - 2) * st]));
}

/* variable-coefficient second derivative accumulated into *o:
 * spatial_operators.hpp:31-156 */
static inline void d2v_at(real *o, int add, const real *v, const real *f, long st, int n, int j, real a, real d2)
{
    real acc = add ? *o : (real)0;
    if (j < 6 || j >= n - 6) {
        int top = j < 6;
        int r = top ? j : n - 1 - j;
        for (int jj = 0; jj < 8; jj++) {
            real val = 0;
            for (int k = 0; k < 8; k++) {
                long q = top ? (long)k * st : (long)(n - 1 - k) * st;
                val += B2[r][jj][k] * f[q];
            }
            long qi = top ? (long)jj * st : (long)(n - 1 - jj) * st;
            acc += a * val * v[qi] / d2;
        }
        *o = acc;
        return;
    }
    const real fm2 = f[(j - 2) * st], fm1 = f[(j - 1) * st], f0 = f[j * st], fp1 = f[(j + 1) * st], fp2 = f[(j + 2) * st];
    const real um2 = v[(j - 2) * st], um1 = v[(j - 1) * st], u0 = v[j * st], up1 = v[(j + 1) * st], up2 = v[(j + 2) * st];
    *o = acc + a / d2 * ((C2[0] * f0 + C2[1] * (fm1 + fp1) + C2[2] * (fm2 + fp2)) * u0
                       + (C2[3] * fm2 + C2[4] * fm1 + C2[5] * f0 + C2[6] * fp1) * um1
                       + (C2[3] * fp2 + C2[4] * fp1 + C2[5] * f0 + C2[6] * fm1) * up1
                       + (C2[7] * fm2 + C2[8] * fm1 + C2[9] * f0) * um2
                       + (C2[7] * fp2 + C2[8] * fp1 + C2[9] * f0) * up2);
}

/* Whole-grid wrappers.  Layout a[ix*nz+iz]. */
static void Dz_(int add, const real *in, real *out, int nx, int nz, real d)
{
    real scale = (real)(1.0 / (double)d);
    OMP_FOR
    for (int ix = 0; ix < nx; ix++) {
        const real *v = in + (long)ix * nz;
        for (int iz = 0; iz < nz; iz++) {
            real r = d1_at(v, 1, nz, iz, d, scale);
            long i = (long)ix * nz + iz;
            out[i] = add ? out[i] + r : r;
        }
    }
}
static void Dx_(int add, const real *in, real *out, int nx, int nz, real d)
{
    real scale = (real)(1.0 / (double)d);
    OMP_FOR
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            real r = d1_at(in + iz, nz, nx, ix, d, scale);
            long i = (long)ix * nz + iz;
            out[i] = add ? out[i] + r : r;
        }
}
static void mDz_(const real *in, real *out, int nx, int nz, real d, const real *p)
{
    real ad = (real)1 / d;
    OMP_FOR
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            long i = (long)ix * nz + iz;
            out[i] = out[i] + md1_at(in + (long)ix * nz, p + (long)ix * nz, 1, nz, iz, ad);
        }
}
static void mDx_(const real *in, real *out, int nx, int nz, real d, const real *p)
{
    real ad = (real)1 / d;
    OMP_FOR
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
            long i = (long)ix * nz + iz;
            out[i] = out[i] + md1_at(in + iz, p + iz, nz, nx, ix, ad);
        }
}
static void Dzzv_(int add, const real *in, real *out, int nx, int nz, real d, const real *f)
{
    real d2 = d * d;
    OMP_FOR
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++)
            d2v_at(out + (long)ix * nz + iz, add, in + (long)ix * nz, f + (long)ix * nz, 1, nz, iz, (real)1, d2);
}
static void Dxxv_(int add, const real *in, real *out, int nx, int nz, real d, const real *f)
{
    real d2 = d * d;
    OMP_FOR
    for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++)
            d2v_at(out + (long)ix * nz + iz, add, in + iz, f + iz, nz, nx, ix, (real)1, d2);
}

/* ---------------------------------------------------------------------------
 * Elastic SAT closures (spatial_operators.hpp:160-822).
 * side: 0 top, 1 bottom, 2 left, 3 right.
 * in1: field differentiated along the boundary, in2: field differentiated
 * outwards, in3: previous field for the absorbing term (NULL = traction free).
 * ------------------------------------------------------------------------- */
static inline real tangential_d1(const real *edge, long st, int n, int p)
{
    real s = 0;
    if (p < 4) {
        for (int j = 0; j < 6; j++) s += B1[p][j] * edge[j * st];
    } else if (p >= n - 4) {
        int r = n - 1 - p;
        for (int j = 0; j < 6; j++) s -= B1[r][j] * edge[(long)(n - 1 - j) * st];
    } else {
        for (int j = 1; j <= 2; j++) s += C1[j - 1] * (edge[(p + j) * st] - edge[(p - j) * st]);
    }
    return s;
}

static void esat_side(int side, const real *in1, const real *in2, const real *in3, real *out,
                      int nx, int nz, real dx, real dz, real dt,
                      const real *f1, const real *f2, const real *f3)
{
    const real a = 1;
    if (side == 0 || side == 1) {
        const int base = side == 0 ? 0 : nz - 1;
        const long inward = side == 0 ? 1 : -1;
        const real sgn = side == 0 ? (real)-1 : (real)1;
        OMP_FOR
        for (int ix = 0; ix < nx; ix++) {
            long c = (long)ix * nz + base;
            real sumx = tangential_d1(in1 + base, nz, nx, ix);
            real sumz = 0;
            for (int k = 0; k < 4; k++) sumz += SC[k] * in2[c + k * inward];
            real t = (sgn * f1[c]) * sumx / dx + f2[c] * sumz / dz;
            if (in3) t = t - f3[c] * in3[c] / dt;
            out[c] = out[c] - a / (dz * H0) * t;
        }
    } else {
        const long base = side == 2 ? 0 : (long)(nx - 1) * nz;
        const long inward = side == 2 ? nz : -(long)nz;
        const real sgn = side == 2 ? (real)-1 : (real)1;
        OMP_FOR
        for (int iz = 0; iz < nz; iz++) {
            long c = base + iz;
            real sumz = tangential_d1(in1 + base, 1, nz, iz);
            real sumx = 0;
            for (int k = 0; k < 4; k++) sumx += SC[k] * in2[c + k * inward];
            real t = (sgn * f1[c]) * sumz / dz + f2[c] * sumx / dx;
            if (in3) t = t - f3[c] * in3[c] / dt;
            out[c] = out[c] - a / (dx * H0) * t;
        }
    }
}

/* extra version-2 SAT -H^-1 (f . D_normal in)_0: spatial_operators.hpp:732-822 */
static void esat_normal_d1(int side, const real *in, real *out, int nx, int nz, real d, const real *f)
{
    const real sc = (real)1 / (d * d * H0);
    if (side == 0 || side == 1) {
        OMP_FOR
        for (int ix = 0; ix < nx; ix++) {
            long c = (long)ix * nz + (side == 0 ? 0 : nz - 1);
            long st = side == 0 ? 1 : -1;
            real s = 0;
            for (int j = 0; j < 6; j++) s -= B1[0][j] * in[c + j * st];
            out[c] = out[c] - sc * f[c] * s;
        }
    } else {
        OMP_FOR
        for (int iz = 0; iz < nz; iz++) {
            long c = (side == 2 ? 0 : (long)(nx - 1) * nz) + iz;
            long st = side == 2 ? nz : -(long)nz;
            real s = 0;
            for (int j = 0; j < 6; j++) s -= B1[0][j] * in[c + j * st];
            out[c] = out[c] - sc * f[c] * s;
        }
    }
}

/* implicit part of the absorbing SAT: spatial_operators.cpp:307-521.
 * The reference calls the double sqrt on single-precision arguments, so each
 * scaler is evaluated in double and rounded once to `real`; DS() restates
 * that.  CXX(i) is the x-wave modulus: lambda+2mu (iso) or (1+2eps)(lambda+2mu) (VTI). */
#define DS(x) sqrt((double)(x))
static void esat_scale(real *u0, real *u1, int nx, int nz, real dx, real dz, real dt,
                       const real *lam, const real *mu, const real *rho, const real *eps,
                       int top, int bottom, int left, int right)
{
    const real h0 = H0;
    const double ddt = (double)dt;
    const double vz = (double)(2 * dz * h0), vx = (double)(2 * dx * h0);
#define CXX(i) (eps ? ((1 + 2 * eps[i]) * (lam[i] + 2 * mu[i])) : (lam[i] + 2 * mu[i]))
    real sc1x = 0, sc1z = 0, sc2x = 0, sc2z = 0;
    if (top) {
        sc1x = (real)(DS(mu[0] / rho[0]) * ddt / vz);
        sc1z = (real)(sc1x * DS((lam[0] + 2 * mu[0]) / mu[0]));
        long c = (long)(nx - 1) * nz;
        sc2x = (real)(DS(mu[c] / rho[c]) * ddt / vz);
        sc2z = (real)(sc1x * DS((lam[c] + 2 * mu[c]) / mu[c]));   /* the reference pairs sc1x here */
        for (int ix = 1; ix < nx - 1; ix++) {
            long i = (long)ix * nz;
            real sx = (real)(DS(mu[i] / rho[i]) * ddt / vz);
            real sz = (real)(sx * DS((lam[i] + 2 * mu[i]) / mu[i]));
            u0[i] = u0[i] / (1 + sx);
            u1[i] = u1[i] / (1 + sz);
        }
    }
    if (left) {
        sc1x = (real)(sc1x + DS(CXX(0) / rho[0]) * ddt / vx);
        sc1z = (real)(sc1z + DS(mu[0] / rho[0]) * ddt / vx);
        u0[0] = u0[0] / (1 + sc1x);
        u1[0] = u1[0] / (1 + sc1z);
        long b = nz - 1;
        sc1x = (real)(DS(CXX(b) / rho[b]) * ddt / vx);
        sc1z = (real)(sc1x * DS(mu[b] / CXX(b)));
        for (int iz = 1; iz < nz - 1; iz++) {
            real sx = (real)(DS(CXX(iz) / rho[iz]) * ddt / vx);
            real sz = (real)(sx * DS(mu[iz] / CXX(iz)));
            u0[iz] = u0[iz] / (1 + sx);
            u1[iz] = u1[iz] / (1 + sz);
        }
    } else {
        u0[0] = u0[0] / (1 + sc1x);
        u1[0] = u1[0] / (1 + sc1z);
        sc1x = 0; sc1z = 0;
    }
    if (bottom) {
        long b = nz - 1;
        sc1x = (real)(sc1x + DS(mu[b] / rho[b]) * ddt / vz);
        sc1z = (real)(sc1z + DS((lam[b] + 2 * mu[b]) / rho[b]) * ddt / vz);
        u0[b] = u0[b] / (1 + sc1x);
        u1[b] = u1[b] / (1 + sc1z);
        long c = (long)(nx - 1) * nz + nz - 1;
        sc1x = (real)(DS(mu[c] / rho[c]) * ddt / vz);
        sc1z = (real)(sc1x * DS((lam[c] + 2 * mu[c]) / mu[c]));
        for (int ix = 1; ix < nx - 1; ix++) {
            long i = (long)ix * nz + nz - 1;
            real sx = (real)(DS(mu[i] / rho[i]) * ddt / vz);
            real sz = (real)(sx * DS((lam[i] + 2 * mu[i]) / mu[i]));
            u0[i] = u0[i] / (1 + sx);
            u1[i] = u1[i] / (1 + sz);
        }
    } else {
        long b = nz - 1;
        u0[b] = u0[b] / (1 + sc1x);
        u1[b] = u1[b] / (1 + sc1z);
        sc1x = 0; sc1z = 0;
    }
    if (right) {
        long c = (long)(nx - 1) * nz + nz - 1;
        sc1x = (real)(sc1x + DS(CXX(c) / rho[c]) * ddt / vx);
        sc1z = (real)(sc1z + DS(mu[c] / rho[c]) * ddt / vx);
        u0[c] = u0[c] / (1 + sc1x);
        u1[c] = u1[c] / (1 + sc1z);
        for (int iz = 1; iz < nz - 1; iz++) {
            long i = (long)(nx - 1) * nz + iz;
            real sx = (real)(DS(CXX(i) / rho[i]) * ddt / vx);
            real sz = (real)(sx * DS(mu[i] / CXX(i)));
            u0[i] = u0[i] / (1 + sx);
            u1[i] = u1[i] / (1 + sz);
        }
        long t = (long)(nx - 1) * nz;
        sc2x = (real)(sc2x + DS(CXX(t) / rho[t]) * ddt / vx);
        sc2z = (real)(sc2z + DS(mu[t] / rho[t]) * ddt / vx);
        u0[t] = u0[t] / (1 + sc2x);
        u1[t] = u1[t] / (1 + sc2z);
    } else {
        long c = (long)(nx - 1) * nz + nz - 1;
        u0[c] = u0[c] / (1 + sc1x);
        u1[c] = u1[c] / (1 + sc1z);
        long t = (long)(nx - 1) * nz;
        u0[t] = u0[t] / (1 + sc2x);
        u1[t] = u1[t] / (1 + sc2z);
    }
#undef CXX
}

/* ---------------------------------------------------------------------------
 * Acoustic SAT closures (spatial_operators.cpp:551-860).  Model (K, 1/rho).
 * ------------------------------------------------------------------------- */
static void asat_dirichlet(int side, const real *in, real *out, int nx, int nz, real dx, real dz, const real *irho, real alpha)
{
    if (side == 0 || side == 1) {
        real dz2 = dz * dz;
        OMP_FOR
        for (int ix = 0; ix < nx; ix++) {
            long b = (long)ix * nz + (side == 0 ? 0 : nz - 1);
            long st = side == 0 ? 1 : -1;
            for (int k = 0; k < 4; k++)
                out[b + k * st] = out[b + k * st] + 1.0 / (HC[k] * dz2) * SC[k] * irho[b] * in[b];
            out[b] -= irho[b] * in[b] / (alpha * HC[0] * dz2);
        }
    } else {
        real dx2 = dx * dx;
        long base = side == 2 ? 0 : (long)(nx - 1) * nz;
        long st = side == 2 ? nz : -(long)nz;
        OMP_FOR
        for (int iz = 0; iz < nz; iz++)
            for (int k = 0; k < 4; k++)
                out[base + iz + k * st] = out[base + iz + k * st] + 1.0 / (HC[k] * dx2) * SC[k] * irho[base + iz] * in[base + iz];
        OMP_FOR
        for (int iz = 0; iz < nz; iz++) out[base + iz] -= irho[base + iz] * in[base + iz] / (alpha * HC[0] * dx2);
    }
}

/* Neumann (in3 == NULL) or absorbing acoustic SAT. */
static void asat_nabs(int side, const real *in, const real *in3, real *out, int nx, int nz, real dx, real dz, real dt,
                      const real *K, const real *irho)
{
    int horiz = (side == 0 || side == 1);
    real d = horiz ? dz : dx;
    long st = side == 0 ? 1 : side == 1 ? -1 : side == 2 ? nz : -(long)nz;
    int n = horiz ? nx : nz;
    OMP_FOR
    for (int p = 0; p < n; p++) {
        long c = horiz ? (long)p * nz + (side == 0 ? 0 : nz - 1) : (side == 2 ? 0 : (long)(nx - 1) * nz) + p;
        real s = 0;
        for (int k = 0; k < 4; k++) s += SC[k] * in[c + k * st];
        if (in3)
            out[c] = out[c] - 1.0 / (H0 * d) * ((double)(irho[c] * s / d) - in3[c] / ((double)(2 * dt) * DS(K[c] / irho[c])));
        else
            out[c] = out[c] - 1.0 / (H0 * d) * irho[c] * s / d;
    }
}

static void asat_scale(real *u, int nx, int nz, real dx, real dz, real dt, const real *K, const real *irho,
                       int top, int bottom, int left, int right)
{
    const real h0 = H0;
    const double ddt = (double)dt;
    const double vz = (double)(2 * dz * h0), vx = (double)(2 * dx * h0);
    real sc1 = 0, sc2 = 0;
    if (top) {
        sc1 = (real)(DS(K[0] * irho[0]) * ddt / vz);
        long t = (long)(nx - 1) * nz;
        sc2 = (real)(DS(K[t] * irho[t]) * ddt / vz);
        for (int ix = 1; ix < nx - 1; ix++) {
            long i = (long)ix * nz;
            real s = (real)(DS(K[i] * irho[i]) * ddt / vz);
            u[i] = u[i] / (1 + s);
        }
    }
    if (left) {
        sc1 = (real)(sc1 + DS(K[0] * irho[0]) * ddt / vx);
        u[0] = u[0] / (1 + sc1);
        long b = nz - 1;
        sc1 = (real)(DS(K[b] * irho[b]) * ddt / vx);
        for (int iz = 1; iz < nz - 1; iz++) {
            real s = (real)(DS(K[iz] * irho[iz]) * ddt / vx);
            u[iz] = u[iz] / (1 + s);
        }
    } else {
        u[0] = u[0] / (1 + sc1);
        sc1 = 0;
    }
    if (bottom) {
        long b = nz - 1;
        sc1 = (real)(sc1 + DS(K[b] * irho[b]) * ddt / vz);
        u[b] = u[b] / (1 + sc1);
        long c = (long)(nx - 1) * nz + nz - 1;
        sc1 = (real)(DS(K[c] * irho[c]) * ddt / vz);
        for (int ix = 1; ix < nx - 1; ix++) {
            long i = (long)ix * nz + nz - 1;
            real s = (real)(DS(K[i] * irho[i]) * ddt / vz);
            u[i] = u[i] / (1 + s);
        }
    } else {
        u[nz - 1] = u[nz - 1] / (1 + sc1);
        sc1 = 0;
    }
    if (right) {
        long c = (long)(nx - 1) * nz + nz - 1;
        sc1 = (real)(sc1 + DS(K[c] * irho[c]) * ddt / vx);
        u[c] = u[c] / (1 + sc1);
        for (int iz = 1; iz < nz - 1; iz++) {
            long i = (long)(nx - 1) * nz + iz;
            real s = (real)(DS(K[i] * irho[i]) * ddt / vx);
            u[i] = u[i] / (1 + s);
        }
        long t = (long)(nx - 1) * nz;
        sc2 = (real)(sc2 + DS(K[t] * irho[t]) * ddt / vx);
        u[t] = u[t] / (1 + sc2);
    } else {
        long c = (long)(nx - 1) * nz + nz - 1;
        u[c] = u[c] / (1 + sc1);
        long t = (long)(nx - 1) * nz;
        u[t] = u[t] / (1 + sc2);
    }
}

/* ---------------------------------------------------------------------------
 * cos^2 taper (spatial_operators.cpp:523-549 + spatial_operators.ispc:47-68).
 * The z bands use single-precision cos (ISPC), the x bands double cos.
 * ------------------------------------------------------------------------- */
static void taper_band_z(real *u, int nx, int nz, int istart, int iend, real a)
{
    if (iend == istart) return;
    int lo = iend > istart ? istart : iend, hi = iend > istart ? iend : istart;
    real *val2 = (real *)malloc(sizeof(real) * (hi - lo + 1));
    for (int i = lo; i < hi; i++) {
        real v;
        if (iend > istart) v = R_COS(a * (real)0.5 * (real)M_PI * (real)(i - istart) / (real)(iend - istart));
        else v = R_COS(a * (real)0.5 * (real)M_PI * (real)(i + 1 - istart) / (real)(iend - istart));
        val2[i - lo] = v * v;
    }
    OMP_FOR
    for (int ix = 0; ix < nx; ix++)
        for (int i = lo; i < hi; i++) u[(long)ix * nz + i] *= val2[i - lo];
    free(val2);
}
static void taper_band_x(real *u, int nx, int nz, int istart, int iend, real a)
{
    if (iend == istart) return;
    int lo = iend > istart ? istart : iend, hi = iend > istart ? iend : istart;
    for (int ix = lo; ix < hi; ix++) {
        real v;
        if (iend > istart) v = (real)cos(a * 0.5 * M_PI * (ix - istart) / (iend - istart));
        else v = (real)cos(a * 0.5 * M_PI * (ix + 1 - istart) / (iend - istart));
        real v2 = v * v;
        real *p = u + (long)ix * nz;
        for (int iz = 0; iz < nz; iz++) p[iz] = v2 * p[iz];
    }
}
static void taper_all(real *u, int nx, int nz, const orc_param *par, int zt, int zb, int xl, int xr)
{
    real a = (real)par->taper_strength;
    if (zt) taper_band_z(u, nx, nz, par->taper_top, 0, a);
    if (zb) taper_band_z(u, nx, nz, nz - par->taper_bottom, nz, a);
    if (xl) taper_band_x(u, nx, nz, par->taper_left, 0, a);
    if (xr) taper_band_x(u, nx, nz, nx - par->taper_right, nx, a);
}

/* ---------------------------------------------------------------------------
 * Injectors (injector.cpp:3-239, misc.cpp:11-16).
 * ------------------------------------------------------------------------- */
static real hcoef_at(int n, int i)
{
    if (i < 4) return HC[i];
    if (i >= n - 4) return HC[n - 1 - i];
    return 1;
}

/* delta_m3 / ddelta_m3 ::findIndicesWeights.  xw, zw: [ntr][2][3] (type 0)
 * or [ntr][2][6] (type 1). */
void ORC(injector_weights)(int type, int ntr, const void *locx_, const void *locz_,
                           int nx, int nz, double dx_, double dz_, double ox_, double oz_,
                           int *xind, int *zind, void *xw_, void *zw_)
{
    init_tables();
    const real *locx = (const real *)locx_, *locz = (const real *)locz_;
    real *xw = (real *)xw_, *zw = (real *)zw_;
    const real dx = (real)dx_, dz = (real)dz_, ox = (real)ox_, oz = (real)oz_;
    const int w = type == 0 ? 3 : 6;
    for (int t = 0; t < ntr; t++) {
        int xi = (int)round((double)((locx[t] - ox) / dx));
        int zi = (int)round((double)((locz[t] - oz) / dz));
        if (xi == 0) xi = 1;
        if (xi == nx - 1) xi = nx - 2;
        if (zi == 0) zi = 1;
        if (zi == nz - 1) zi = nz - 2;
        for (int k = 0; k < 3; k++) { xind[t * 3 + k] = xi - 1 + k; zind[t * 3 + k] = zi - 1 + k; }
        real ax = (locx[t] - dx * (real)xi - ox) / dx;
        real az = (locz[t] - dz * (real)zi - oz) / dz;
        double ax2 = (double)ax * (double)ax, az2 = (double)az * (double)az;
        real *xi0 = xw + t * 2 * w, *xe = xi0 + w;
        real *zi0 = zw + t * 2 * w, *ze = zi0 + w;
        xi0[0] = (real)((ax2 - ax) / (double)(2 * dx * hcoef_at(nx, xi - 1)));
        xi0[1] = (real)((-ax2 + 1) / (double)(dx * hcoef_at(nx, xi)));
        xi0[2] = (real)((ax2 + ax) / (double)(2 * dx * hcoef_at(nx, xi + 1)));
        zi0[0] = (real)((az2 - az) / (double)(2 * dz * hcoef_at(nz, zi - 1)));
        zi0[1] = (real)((-az2 + 1) / (double)(dz * hcoef_at(nz, zi)));
        zi0[2] = (real)((az2 + az) / (double)(2 * dz * hcoef_at(nz, zi + 1)));
        xe[0] = (real)((ax2 - ax) / 2); xe[1] = (real)(-ax2 + 1); xe[2] = (real)((ax2 + ax) / 2);
        ze[0] = (real)((az2 - az) / 2); ze[1] = (real)(-az2 + 1); ze[2] = (real)((az2 + az) / 2);
        if (type == 1) {
            xi0[3] = (1 - 2 * ax) / (2 * dx * dx * hcoef_at(nx, xi - 1));
            xi0[4] = 2 * ax / (dx * dx * hcoef_at(nx, xi));
            xi0[5] = (-1 - 2 * ax) / (2 * dx * dx * hcoef_at(nx, xi + 1));
            zi0[3] = (1 - 2 * az) / (2 * dz * dz * hcoef_at(nz, zi - 1));
            zi0[4] = 2 * az / (dz * dz * hcoef_at(nz, zi));
            zi0[5] = (-1 - 2 * az) / (2 * dz * dz * hcoef_at(nz, zi + 1));
            xe[3] = (1 - 2 * ax) / (2 * dx); xe[4] = 2 * ax / dx; xe[5] = (-1 - 2 * ax) / (2 * dx);
            ze[3] = (1 - 2 * az) / (2 * dz); ze[4] = 2 * az / dz; ze[5] = (-1 - 2 * az) / (2 * dz);
        }
    }
}

/* inject one time sample; in0/in1 are [ntr][nt] trace blocks (in1 only for
 * the moment tensor).  add == 0 zeroes the touched cells first. */
static void inject(const orc_injector *J, int add, const real *in0, const real *in1, real *out, int nz, int nt, int it)
{
    const int w = J->type == 0 ? 3 : 6;
    const real *xw = (const real *)J->xw, *zw = (const real *)J->zw;
    if (!add)
        for (int t = 0; t < J->ntr; t++)
            for (int i = 0; i < 3; i++)
                for (int k = 0; k < 3; k++) out[(long)J->xind[t * 3 + i] * nz + J->zind[t * 3 + k]] = 0;
    for (int t = 0; t < J->ntr; t++) {
        const real *xi = xw + t * 2 * w, *zi = zw + t * 2 * w;
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++) {
                long c = (long)J->xind[t * 3 + i] * nz + J->zind[t * 3 + k];
                if (J->type == 0) out[c] += xi[i] * zi[k] * in0[(long)t * nt + it];
                else out[c] += (-xi[i + 3] * zi[k] * in0[(long)t * nt + it] - xi[i] * zi[k + 3] * in1[(long)t * nt + it]);
            }
    }
}

static void extract(const orc_injector *J, const real *in, real *out, int nz, int nt, int it)
{
    const real *xw = (const real *)J->xw, *zw = (const real *)J->zw;
    for (int t = 0; t < J->ntr; t++) {
        const real *xe = xw + t * 6 + 3, *ze = zw + t * 6 + 3;
        real o = out[(long)t * nt + it];
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++)
                o += xe[i] * ze[k] * in[(long)J->xind[t * 3 + i] * nz + J->zind[t * 3 + k]];
        out[(long)t * nt + it] = o;
    }
}

/* ---------------------------------------------------------------------------
 * Imaging conditions.
 * ------------------------------------------------------------------------- */
static real gdamp_weight(const orc_param *par, int it, real dtg)
{
    real t = it * dtg;
    real w = 1;
    real tmin = (real)par->gdamp_tmin, tmax = (real)par->gdamp_tmax, pw = (real)par->gdamp_power;
    if (tmax - t > 0 && t - tmin >= 0) w = (real)cos(pw * M_PI * (t - tmin) / (tmax - tmin));
    w *= w;
    return w;
}

/* Test switch, not the reference's behaviour: with g_exact_sum set, the
 * elastic / VTI imaging condition adds each time sample's terms (computed
 * exactly as below) into a double array, rounded to real once at the end of
 * the propagation: the exact sum of the same single-precision terms, against
 * which the tests measure the summation error of the device's plain and
 * compensated gradient accumulations.  Off by default. */
static int g_exact_sum = 0;
static double *g_xsum = NULL;   /* [3][nxz] while an exact-sum adjoint runs */

void ORC(set_exact_gradient_sum)(int on) { g_exact_sum = on != 0; }

/* g[i] += term in real arithmetic, or the term into the exact sum */
static inline void acc_r(real *g, double *x, long i, real term)
{
    if (x) x[i] += (double)term;
    else g[i] += term;
}
/* g[i] = (real)((double)g[i] + term), or the term into the exact sum */
static inline void acc_d(real *g, double *x, long i, double term)
{
    if (x) x[i] += term;
    else g[i] = (real)((double)g[i] + term);
}

/* nl_we_op_e::compute_gradients (we_op.cpp:505-562) and the VTI variant
 * (we_op.cpp:1478-1557).  m: converted model; ufull [nsnap][2][nxz]. */
static void grad_elastic(int vti, const real *m, const real *ufull, const real *adj, const real *ax, const real *az,
                         real *tmp, real *g, const orc_param *par, int nx, int nz, int it, real dx, real dz, real dtg)
{
    const long nxz = (long)nx * nz;
    const real *f0 = ufull + (long)it * 2 * nxz, *f1 = f0 + nxz;
    real *t0 = tmp, *t1 = tmp + nxz, *t2 = tmp + 2 * nxz, *t3 = tmp + 3 * nxz;
    Dx_(0, f0, t0, nx, nz, dx);
    Dz_(0, f1, t1, nx, nz, dz);
    Dx_(0, f1, t2, nx, nz, dx);
    Dz_(0, f0, t3, nx, nz, dz);
    const real w = gdamp_weight(par, it, dtg);
    const int last = par->nt / par->sub;
    const real *ax0 = ax, *ax1 = ax + nxz, *az0 = az, *az1 = az + nxz;
    const real *a0 = adj, *a1 = adj + nxz;
    const real *lam = m, *mu = m + nxz, *c13 = m + 3 * nxz, *eps = m + 4 * nxz;
    const real *fp0 = it + 1 <= last ? f0 + 2 * nxz : NULL, *fp1 = fp0 ? fp0 + nxz : NULL;
    const real *fm0 = it > 0 ? f0 - 2 * nxz : NULL, *fm1 = fm0 ? fm0 + nxz : NULL;
    real *g0 = g, *g1 = g + nxz, *g2 = g + 2 * nxz;
    double *x0 = g_xsum, *x1 = g_xsum ? g_xsum + nxz : NULL, *x2 = g_xsum ? g_xsum + 2 * nxz : NULL;
    OMP_FOR
    for (long i = 0; i < nxz; i++) {
        real dl, dm;
        if (!vti) {
            dl = (ax0[i] + az1[i]) * (t0[i] + t1[i]);
            dm = (az0[i] + ax1[i]) * (t2[i] + t3[i]) + 2 * ax0[i] * t0[i] + 2 * az1[i] * t1[i];
        } else {
            real del = ((c13[i] + mu[i]) * (c13[i] + mu[i]) - (lam[i] + mu[i]) * (lam[i] + mu[i])) / (2 * (lam[i] + mu[i]) * (lam[i] + 2 * mu[i]));
            real v1 = R_SQRT(2 * (lam[i] + 2 * mu[i]) * (lam[i] + mu[i]) * del + (lam[i] + mu[i]) * (lam[i] + mu[i]));
            real v2 = ((1 + 2 * del) * lam[i] + (1 + 3 * del) * mu[i]) / v1;
            real v3 = ((1 + 3 * del) * lam[i] + (1 + 4 * del) * mu[i]) / v1 - 1;
            dl = (1 + 2 * eps[i]) * ax0[i] * t0[i] + az1[i] * t1[i] + v2 * (ax0[i] * t1[i] + az1[i] * t0[i]);
            dm = (az0[i] + ax1[i]) * (t2[i] + t3[i]) + 2 * (1 + 2 * eps[i]) * ax0[i] * t0[i] + 2 * az1[i] * t1[i]
               + v3 * (ax0[i] * t1[i] + az1[i] * t0[i]);
        }
        if (it > 0 && it < last) {
            if (!vti) acc_r(g0, x0, i, w * dtg * (ax0[i] + az1[i]) * (t0[i] + t1[i]));
            else acc_r(g0, x0, i, w * dtg * dl);
            acc_r(g1, x1, i, w * dtg * dm);
            acc_d(g2, x2, i, (double)w * 1.0 / (double)dtg
                  * (double)(a0[i] * (fp0[i] - 2 * f0[i] + fm0[i]) + a1[i] * (fp1[i] - 2 * f1[i] + fm1[i])));
        } else if (it == 0) {
            acc_d(g0, x0, i, (double)w * 0.5 * (double)dtg * (double)(vti ? dl : (ax0[i] + az1[i])) * (double)(vti ? 1 : (t0[i] + t1[i])));
            acc_d(g1, x1, i, (double)w * 0.5 * (double)dtg * (double)dm);
            acc_d(g2, x2, i, (double)w * 1.0 / (double)dtg
                  * (double)(a0[i] * (fp0[i] - f0[i]) + a1[i] * (fp1[i] - f1[i])));
        } else {
            if (!vti) acc_r(g0, x0, i, w * dtg * (ax0[i] + az1[i]) * (t0[i] + t1[i]));
            else acc_r(g0, x0, i, w * dtg * dl);
            acc_r(g1, x1, i, w * dtg * dm);
            acc_d(g2, x2, i, (double)w * 1.0 / (double)dtg
                  * (double)(a0[i] * (-f0[i] + fm0[i]) + a1[i] * (-f1[i] + fm1[i])));
        }
    }
}

/* nl_we_op_a::compute_gradients (we_op.cpp:1883-1935).  m = (K, 1/rho). */
static void grad_acoustic(const real *m, const real *ufull, const real *adj, real *tmp, real *g,
                          const orc_param *par, int nx, int nz, int it, real dx, real dz, real dtg)
{
    const long nxz = (long)nx * nz;
    const real *f = ufull + (long)it * nxz;
    real *t0 = tmp, *t1 = tmp + nxz, *t2 = tmp + 2 * nxz, *t3 = tmp + 3 * nxz;
    Dx_(0, f, t0, nx, nz, dx);
    Dz_(0, f, t1, nx, nz, dz);
    Dx_(0, adj, t2, nx, nz, dx);
    Dz_(0, adj, t3, nx, nz, dz);
    const real w = gdamp_weight(par, it, dtg);
    const int last = par->nt / par->sub;
    const real *K = m;
    const real *fp = it + 1 <= last ? f + nxz : NULL, *fm = it > 0 ? f - nxz : NULL;
    real *g0 = g, *g1 = g + nxz;
    OMP_FOR
    for (long i = 0; i < nxz; i++) {
        double c = (double)w * 1.0 / (double)(dtg * K[i] * K[i]) * (double)adj[i];
        if (it > 0 && it < last) {
            g0[i] = (real)((double)g0[i] - c * (double)(fp[i] - 2 * f[i] + fm[i]));
            g1[i] += w * dtg * (t2[i] * t0[i] + t3[i] * t1[i]);
        } else if (it == 0) {
            g0[i] = (real)((double)g0[i] - c * (double)(fp[i] - f[i]));
            g1[i] = (real)((double)g1[i] + (double)w * 0.5 * (double)dtg * (double)(t2[i] * t0[i] + t3[i] * t1[i]));
        } else {
            g0[i] = (real)((double)g0[i] - c * (double)(-f[i] + fm[i]));
            g1[i] += w * dtg * (t2[i] * t0[i] + t3[i] * t1[i]);
        }
    }
}

/* ---------------------------------------------------------------------------
 * Elastic (iso / VTI) propagation: we_op.cpp:564-902 and 1559-1861.
 * model: converted [3][nx][nz] (lambda, mu, rho) or [5] (+ c13, eps).
 * src: [ncomp][ns][nt] (this shot's traces), rcv: [ncomp][nr][nt] (accumulated).
 * ------------------------------------------------------------------------- */
static void propagate_elastic(int vti, int adj, const real *model, const real *allsrc, real *allrcv,
                              const orc_injector *inj, const orc_injector *ext, real *full, real *grad,
                              const orc_param *par, int nx, int nz, real dx, real dz)
{
    const long nxz = (long)nx * nz;
    const int nt = par->nt, sub = par->sub;
    const real dt = (real)par->dt;
    real *u = (real *)calloc(6 * nxz, sizeof(real));
    real *dux = (real *)calloc(2 * nxz, sizeof(real));
    real *duz = (real *)calloc(2 * nxz, sizeof(real));
    real *tmp = (real *)calloc((grad ? 4 : 1) * nxz, sizeof(real));
    real *tmp1 = (real *)calloc(nxz, sizeof(real));
    real *prev = u, *curr = u + 2 * nxz, *next = u + 4 * nxz;
    const real *lam = model, *mu = model + nxz, *rho = model + 2 * nxz;
    const real *c13 = vti ? model + 3 * nxz : NULL, *eps = vti ? model + 4 * nxz : NULL;
    g_xsum = grad && g_exact_sum ? (double *)calloc(3 * nxz, sizeof(double)) : NULL;

    /* coefficient fields of the variable-coefficient operators */
    real *f2mu = (real *)malloc(nxz * sizeof(real));
    real *fxx = (real *)malloc(nxz * sizeof(real));     /* iso: 2mu, VTI: (1+2eps)2mu */
    real *lbis = vti ? (real *)malloc(nxz * sizeof(real)) : NULL;  /* (1+2eps)lambda */
    real *fimp_s = (real *)malloc(nxz * sizeof(real));  /* 1/2 sqrt(rho mu) */
    real *fimp_p = (real *)malloc(nxz * sizeof(real));  /* 1/2 sqrt(rho (lambda+2mu)) */
    real *fimp_px = vti ? (real *)malloc(nxz * sizeof(real)) : NULL; /* 1/2 sqrt(rho (1+2eps)(lambda+2mu)) */
    for (long i = 0; i < nxz; i++) {
        f2mu[i] = 2 * mu[i];
        fxx[i] = vti ? (1 + 2 * eps[i]) * 2 * mu[i] : 2 * mu[i];
        if (vti) lbis[i] = (1 + 2 * eps[i]) * lam[i];
        fimp_s[i] = (real)(0.5 * R_SQRT(mu[i] * rho[i]));
        fimp_p[i] = (real)(0.5 * R_SQRT((lam[i] + 2 * mu[i]) * rho[i]));
        if (vti) fimp_px[i] = (real)(0.5 * R_SQRT((1 + 2 * eps[i]) * (lam[i] + 2 * mu[i]) * rho[i]));
    }
    const real *c13f = vti ? c13 : lam;       /* coefficient of the cross term in the SAT */
    const real *fxxs = fxx;                   /* normal coefficient on left/right for next0 */
    const real *lamx = vti ? lbis : lam;      /* extra Dx SAT coefficient on left/right */
    const real *impx = vti ? fimp_px : fimp_p;

    int ns = par->ns, nr = par->nr;
    if (adj) { ns = par->nr; nr = par->ns; }
    const real *srcx0 = allsrc, *srcx1 = NULL, *srcz0 = allsrc + (long)ns * nt, *srcz1 = NULL;
    real *rcvx = allrcv, *rcvz = allrcv ? allrcv + (long)nr * nt : NULL;
    if (par->mt && !adj) {
        srcx1 = allsrc + 2L * ns * nt;
        srcz0 = allsrc + 2L * ns * nt;
        srcz1 = allsrc + (long)ns * nt;
    }

    inject(inj, 0, srcx0, srcx1, prev, nz, nt, 0);
    inject(inj, 0, srcz0, srcz1, prev + nxz, nz, nt, 0);
    for (long i = 0; i < nxz; i++) {
        prev[i] = (real)((double)prev[i] * (0.5 * (double)dt * (double)dt / (double)rho[i]));
        prev[nxz + i] = (real)((double)prev[nxz + i] * (0.5 * (double)dt * (double)dt / (double)rho[i]));
    }

    for (int it = 0; it < nt - 1; it++) {
        if (full && sub > 0 && it % sub == 0 && !grad) memcpy(full + (long)(it / sub) * 2 * nxz, curr, 2 * nxz * sizeof(real));
        if (!grad) {
            extract(ext, curr, rcvx, nz, nt, it);
            extract(ext, curr + nxz, rcvz, nz, nt, it);
        }
        if (grad && (nt - 1 - it) % sub == 0 && it != 0)
            grad_elastic(vti, model, full, curr, dux, duz, tmp, grad, par, nx, nz, (nt - 1 - it) / sub, dx, dz, sub * dt);

        real *c0 = curr, *c1 = curr + nxz, *n0 = next, *n1 = next + nxz, *p0 = prev, *p1 = prev + nxz;
        Dxxv_(0, c0, n0, nx, nz, dx, fxx);
        Dzzv_(0, c1, n1, nx, nz, dz, f2mu);
        Dxxv_(1, c1, n1, nx, nz, dx, mu);
        Dzzv_(1, c0, n0, nx, nz, dz, mu);
        Dx_(0, c0, dux, nx, nz, dx);
        Dz_(0, c1, duz + nxz, nx, nz, dz);
        if (!vti) {
            for (long i = 0; i < nxz; i++) tmp1[i] = dux[i] + duz[nxz + i];
            mDx_(tmp1, n0, nx, nz, dx, lam);
            mDz_(tmp1, n1, nx, nz, dz, lam);
        } else {
            for (long i = 0; i < nxz; i++) tmp1[i] = lbis[i] * dux[i] + c13[i] * duz[nxz + i];
            Dx_(1, tmp1, n0, nx, nz, dx);
            for (long i = 0; i < nxz; i++) tmp1[i] = lam[i] * duz[nxz + i] + c13[i] * dux[i];
            Dz_(1, tmp1, n1, nx, nz, dz);
        }
        Dx_(0, c1, dux + nxz, nx, nz, dx);
        Dz_(0, c0, duz, nx, nz, dz);
        mDx_(duz, n1, nx, nz, dx, mu);
        mDz_(dux + nxz, n0, nx, nz, dz, mu);

        inject(inj, 1, srcx0, srcx1, n0, nz, nt, it);
        inject(inj, 1, srcz0, srcz1, n1, nz, nt, it);

        /* boundary conditions: bc 1 traction free, 2 locally absorbing */
        int bcs[4] = {par->bc_top, par->bc_bottom, par->bc_left, par->bc_right};
        for (int side = 0; side < 4; side++) {
            int bc = bcs[side];
            if (bc != 1 && bc != 2) continue;
            int ab = bc == 2;
            if (side < 2) {
                esat_side(side, c1, c0, ab ? p0 : NULL, n0, nx, nz, dx, dz, dt, mu, mu, fimp_s);
                esat_side(side, c0, c1, ab ? p1 : NULL, n1, nx, nz, dx, dz, dt, c13f, f2mu, fimp_p);
                esat_normal_d1(side, c1, n1, nx, nz, dz, lam);
            } else {
                esat_side(side, c1, c0, ab ? p0 : NULL, n0, nx, nz, dx, dz, dt, c13f, fxxs, impx);
                esat_normal_d1(side, c0, n0, nx, nz, dx, lamx);
                esat_side(side, c0, c1, ab ? p1 : NULL, n1, nx, nz, dx, dz, dt, mu, mu, fimp_s);
            }
        }

        OMP_FOR
        for (long i = 0; i < nxz; i++) {
            n0[i] = dt * dt * n0[i] / rho[i] + 2 * c0[i] - p0[i];
            n1[i] = dt * dt * n1[i] / rho[i] + 2 * c1[i] - p1[i];
        }
        esat_scale(n0, n1, nx, nz, dx, dz, dt, lam, mu, rho, eps, par->bc_top == 2, par->bc_bottom == 2, par->bc_left == 2, par->bc_right == 2);

        taper_all(c0, nx, nz, par, 1, 1, 1, 1);
        taper_all(c1, nx, nz, par, 1, 1, 1, 1);
        taper_all(n0, nx, nz, par, 1, 1, 1, 1);
        taper_all(n1, nx, nz, par, 1, 1, 1, 1);

        real *b = prev; prev = curr; curr = next; next = b;
    }

    if (full && sub > 0 && (nt - 1) % sub == 0 && !grad) memcpy(full + (long)((nt - 1) / sub) * 2 * nxz, curr, 2 * nxz * sizeof(real));
    if (!grad) {
        extract(ext, curr, rcvx, nz, nt, nt - 1);
        extract(ext, curr + nxz, rcvz, nz, nt, nt - 1);
    }
    if (grad) grad_elastic(vti, model, full, curr, dux, duz, tmp, grad, par, nx, nz, 0, dx, dz, sub * dt);
    if (g_xsum) {
        for (long i = 0; i < 3 * nxz; i++) grad[i] = (real)((double)grad[i] + g_xsum[i]);
        free(g_xsum);
        g_xsum = NULL;
    }

    free(u); free(dux); free(duz); free(tmp); free(tmp1);
    free(f2mu); free(fxx); free(fimp_s); free(fimp_p);
    if (vti) { free(lbis); free(fimp_px); }
}

/* ---------------------------------------------------------------------------
 * Acoustic propagation: we_op.cpp:1937-2134.  model (K, 1/rho).
 * ------------------------------------------------------------------------- */
static void propagate_acoustic(int adj, const real *model, const real *allsrc, real *allrcv,
                               const orc_injector *inj, const orc_injector *ext, real *full, real *grad,
                               const orc_param *par, int nx, int nz, real dx, real dz)
{
    const long nxz = (long)nx * nz;
    const int nt = par->nt, sub = par->sub;
    const real dt = (real)par->dt;
    real *u = (real *)calloc(3 * nxz, sizeof(real));
    real *tmp = (real *)calloc(4 * nxz, sizeof(real));
    real *prev = u, *curr = u + nxz, *next = u + 2 * nxz;
    const real *K = model, *irho = model + nxz;
    const real alpha = (real)(0.2508560249 / (real)par->free_surface_stiffness);
    (void)adj;

    inject(inj, 0, allsrc, NULL, prev, nz, nt, 0);
    for (long i = 0; i < nxz; i++) prev[i] = (real)((double)prev[i] * (0.5 * (double)K[i] * (double)dt * (double)dt));

    for (int it = 0; it < nt - 1; it++) {
        if (full && sub > 0 && it % sub == 0 && !grad) memcpy(full + (long)(it / sub) * nxz, curr, nxz * sizeof(real));
        if (!grad) extract(ext, curr, allrcv, nz, nt, it);
        if (grad && (nt - 1 - it) % sub == 0 && it != 0)
            grad_acoustic(model, full, curr, tmp, grad, par, nx, nz, (nt - 1 - it) / sub, dx, dz, sub * dt);

        Dxxv_(0, curr, next, nx, nz, dx, irho);
        Dzzv_(1, curr, next, nx, nz, dz, irho);
        inject(inj, 1, allsrc, NULL, next, nz, nt, it);

        int bcs[4] = {par->bc_top, par->bc_bottom, par->bc_left, par->bc_right};
        for (int side = 0; side < 4; side++) {
            if (bcs[side] == 1) asat_dirichlet(side, curr, next, nx, nz, dx, dz, irho, alpha);
            else if (bcs[side] == 2) asat_nabs(side, curr, prev, next, nx, nz, dx, dz, dt, K, irho);
            else if (bcs[side] == 3) asat_nabs(side, curr, NULL, next, nx, nz, dx, dz, dt, K, irho);
        }
        OMP_FOR
        for (long i = 0; i < nxz; i++) next[i] = dt * dt * next[i] * K[i] + 2 * curr[i] - prev[i];
        asat_scale(next, nx, nz, dx, dz, dt, K, irho, par->bc_top == 2, par->bc_bottom == 2, par->bc_left == 2, par->bc_right == 2);
        taper_all(curr, nx, nz, par, 1, 1, 1, 1);
        taper_all(next, nx, nz, par, 1, 1, 1, 1);
        real *b = prev; prev = curr; curr = next; next = b;
    }
    if (full && sub > 0 && (nt - 1) % sub == 0 && !grad) memcpy(full + (long)((nt - 1) / sub) * nxz, curr, nxz * sizeof(real));
    if (!grad) extract(ext, curr, allrcv, nz, nt, nt - 1);
    if (grad) grad_acoustic(model, full, curr, tmp, grad, par, nx, nz, 0, dx, dz, sub * dt);
    free(u); free(tmp);
}

/* ---------------------------------------------------------------------------
 * Acoustic-elastic propagation: we_op.cpp:2137-2577.  A homogeneous water
 * layer of nza rows (grid nx x nza, same spacing) sits on the elastic grid;
 * its last row and the elastic first row share the interface depth.
 * inj/ext act on the elastic grid, inja/exta on the water grid.
 * ------------------------------------------------------------------------- */
static void propagate_ae(int adj, const real *model, const real *allsrc, real *allrcv,
                         const orc_injector *inj, const orc_injector *ext,
                         const orc_injector *inja, const orc_injector *exta, real *full, real *grad,
                         const orc_param *par, int nx, int nz, real dx, real dz)
{
    const long nxz = (long)nx * nz;
    const int nza = par->nza;
    const long nxza = (long)nx * nza;
    const int nt = par->nt, sub = par->sub;
    const real dt = (real)par->dt;
    real *u = (real *)calloc(6 * nxz, sizeof(real));
    real *dux = (real *)calloc(2 * nxz, sizeof(real));
    real *duz = (real *)calloc(2 * nxz, sizeof(real));
    real *phi = (real *)calloc(3 * nxza, sizeof(real));
    real *moda = (real *)malloc(2 * nxza * sizeof(real));
    real *tmp = (real *)calloc(4 * nxz, sizeof(real));
    real *prev = u, *curr = u + 2 * nxz, *next = u + 4 * nxz;
    real *preva = phi, *curra = phi + nxza, *nexta = phi + 2 * nxza;
    const real Kw = (real)par->water_density * (real)par->water_velocity * (real)par->water_velocity;
    const real rw = (real)par->water_density;
    for (long i = 0; i < nxza; i++) { moda[i] = Kw; moda[nxza + i] = (real)(1.0 / rw); }
    const real *Ka = moda, *irhoa = moda + nxza;
    const real *lam = model, *mu = model + nxz, *rho = model + 2 * nxz;
    const real alpha = (real)(0.2508560249 / (real)par->free_surface_stiffness);

    real *f2mu = (real *)malloc(nxz * sizeof(real));
    real *fimp_s = (real *)malloc(nxz * sizeof(real));
    real *fimp_p = (real *)malloc(nxz * sizeof(real));
    for (long i = 0; i < nxz; i++) {
        f2mu[i] = 2 * mu[i];
        fimp_s[i] = (real)(0.5 * R_SQRT(mu[i] * rho[i]));
        fimp_p[i] = (real)(0.5 * R_SQRT((lam[i] + 2 * mu[i]) * rho[i]));
    }

    int ns = par->ns, nr = par->nr;
    if (adj) { ns = par->nr; nr = par->ns; }
    const real *srcx = NULL, *srcz = NULL;
    real *rcvx = NULL, *rcvz = NULL;
    if (!adj) {
        rcvx = allrcv + (long)nr * nt;
        rcvz = allrcv + 2L * nr * nt;
        if (!par->acoustic_source) { srcx = allsrc; srcz = allsrc + (long)ns * nt; }
    } else {
        srcx = allsrc + (long)ns * nt;
        srcz = allsrc + 2L * ns * nt;
        if (!par->acoustic_source) { rcvx = allrcv; rcvz = allrcv ? allrcv + (long)nr * nt : NULL; }
    }
    const real *srca = allsrc;
    real *rcva = allrcv;

    if (!par->acoustic_source) {
        inject(inj, 0, srcx, NULL, prev, nz, nt, 0);
        inject(inj, 0, srcz, NULL, prev + nxz, nz, nt, 0);
        for (long i = 0; i < nxz; i++) {
            prev[i] = (real)((double)prev[i] * (0.5 * (double)dt * (double)dt / (double)rho[i]));
            prev[nxz + i] = (real)((double)prev[nxz + i] * (0.5 * (double)dt * (double)dt / (double)rho[i]));
        }
    } else {
        inject(inja, 0, srca, NULL, preva, nza, nt, 0);
        for (long i = 0; i < nxza; i++) preva[i] = (real)((double)preva[i] * (0.5 * (double)Ka[i] * (double)dt * (double)dt));
    }

    for (int it = 0; it < nt - 1; it++) {
        if (full && sub > 0 && it % sub == 0 && !grad) memcpy(full + (long)(it / sub) * 2 * nxz, curr, 2 * nxz * sizeof(real));
        if (!grad) {
            if (!adj) {
                extract(ext, curr, rcvx, nz, nt, it);
                extract(ext, curr + nxz, rcvz, nz, nt, it);
                extract(exta, curra, rcva, nza, nt, it);
            } else {
                if (!par->acoustic_source) {
                    extract(ext, curr, rcvx, nz, nt, it);
                    extract(ext, curr + nxz, rcvz, nz, nt, it);
                } else extract(exta, curra, rcva, nza, nt, it);
            }
        }
        if (grad && (nt - 1 - it) % sub == 0 && it != 0)
            grad_elastic(0, model, full, curr, dux, duz, tmp, grad, par, nx, nz, (nt - 1 - it) / sub, dx, dz, sub * dt);

        real *c0 = curr, *c1 = curr + nxz, *n0 = next, *n1 = next + nxz, *p0 = prev, *p1 = prev + nxz;
        Dxxv_(0, curra, nexta, nx, nza, dx, irhoa);
        Dzzv_(1, curra, nexta, nx, nza, dz, irhoa);
        Dxxv_(0, c0, n0, nx, nz, dx, f2mu);
        Dzzv_(0, c1, n1, nx, nz, dz, f2mu);
        Dxxv_(1, c1, n1, nx, nz, dx, mu);
        Dzzv_(1, c0, n0, nx, nz, dz, mu);
        Dx_(0, c0, dux, nx, nz, dx);
        Dz_(0, c1, duz + nxz, nx, nz, dz);
        mDx_(dux, n0, nx, nz, dx, lam);
        mDz_(duz + nxz, n1, nx, nz, dz, lam);
        mDx_(duz + nxz, n0, nx, nz, dx, lam);
        mDz_(dux, n1, nx, nz, dz, lam);
        Dx_(0, c1, dux + nxz, nx, nz, dx);
        Dz_(0, c0, duz, nx, nz, dz);
        mDx_(duz, n1, nx, nz, dx, mu);
        mDz_(dux + nxz, n0, nx, nz, dz, mu);

        if (adj) {
            inject(inj, 1, srcx, NULL, n0, nz, nt, it);
            inject(inj, 1, srcz, NULL, n1, nz, nt, it);
            inject(inja, 1, srca, NULL, nexta, nza, nt, it);
        } else if (!par->acoustic_source) {
            inject(inj, 1, srcx, NULL, n0, nz, nt, it);
            inject(inj, 1, srcz, NULL, n1, nz, nt, it);
        } else {
            inject(inja, 1, srca, NULL, nexta, nza, nt, it);
        }

        /* water top */
        if (par->bc_top == 1) asat_dirichlet(0, curra, nexta, nx, nza, dx, dz, irhoa, alpha);
        else if (par->bc_top == 2) asat_nabs(0, curra, preva, nexta, nx, nza, dx, dz, dt, Ka, irhoa);
        else if (par->bc_top == 3) asat_nabs(0, curra, NULL, nexta, nx, nza, dx, dz, dt, Ka, irhoa);
        /* elastic bottom */
        if (par->bc_bottom == 1 || par->bc_bottom == 2) {
            int ab = par->bc_bottom == 2;
            esat_side(1, c1, c0, ab ? p0 : NULL, n0, nx, nz, dx, dz, dt, mu, mu, fimp_s);
            esat_side(1, c0, c1, ab ? p1 : NULL, n1, nx, nz, dx, dz, dt, lam, f2mu, fimp_p);
            esat_normal_d1(1, c1, n1, nx, nz, dz, lam);
        }
        for (int side = 2; side < 4; side++) {
            int bc = side == 2 ? par->bc_left : par->bc_right;
            if (bc == 1) {
                asat_dirichlet(side, curra, nexta, nx, nza, dx, dz, irhoa, alpha);
            } else if (bc == 2) {
                asat_nabs(side, curra, preva, nexta, nx, nza, dx, dz, dt, Ka, irhoa);
            }
            if (bc == 1 || bc == 2) {
                int ab = bc == 2;
                esat_side(side, c1, c0, ab ? p0 : NULL, n0, nx, nz, dx, dz, dt, lam, f2mu, fimp_p);
                esat_normal_d1(side, c0, n0, nx, nz, dx, lam);
                esat_side(side, c0, c1, ab ? p1 : NULL, n1, nx, nz, dx, dz, dt, mu, mu, fimp_s);
            }
        }
        /* interface, uncoupled parts */
        asat_nabs(1, curra, NULL, nexta, nx, nza, dx, dz, dt, Ka, irhoa);
        esat_side(0, c1, c0, NULL, n0, nx, nz, dx, dz, dt, mu, mu, fimp_s);
        esat_side(0, c0, c1, NULL, n1, nx, nz, dx, dz, dt, lam, f2mu, fimp_p);
        esat_normal_d1(0, c1, n1, nx, nz, dz, lam);

        OMP_FOR
        for (long i = 0; i < nxza; i++) nexta[i] = dt * dt * nexta[i] * Ka[i] + 2 * curra[i] - preva[i];
        OMP_FOR
        for (long i = 0; i < nxz; i++) {
            n0[i] = dt * dt * n0[i] / rho[i] + 2 * c0[i] - p0[i];
            n1[i] = dt * dt * n1[i] / rho[i] + 2 * c1[i] - p1[i];
        }
        asat_scale(nexta, nx, nza, dx, dz, dt, Ka, irhoa, par->bc_top == 2, 0, par->bc_left == 2, par->bc_right == 2);
        esat_scale(n0, n1, nx, nz, dx, dz, dt, lam, mu, rho, NULL, 0, par->bc_bottom == 2, par->bc_left == 2, par->bc_right == 2);

        /* implicit coupling at the interface */
        {
            const int sign = 1 - 2 * adj;
            const real h = (real)((double)dz * (17.0 / 48));
            const real val0 = dt / (2 * h);
            for (int ix = 0; ix < nx; ix++) {
                long ie = (long)ix * nz, ia = (long)ix * nza + nza - 1;
                real v1 = Kw * val0 * (n1[ie] - p1[ie] + sign * val0 / rho[ie] * preva[ia]);
                real v2 = 1 + val0 * val0 * Kw / rho[ie];
                nexta[ia] = (nexta[ia] + sign * v1) / v2;
                n1[ie] = n1[ie] - sign * val0 / rho[ie] * (nexta[ia] - preva[ia]);
            }
        }

        taper_all(curra, nx, nza, par, 1, 0, 1, 1);
        taper_all(nexta, nx, nza, par, 1, 0, 1, 1);
        taper_all(c0, nx, nz, par, 0, 1, 1, 1);
        taper_all(c1, nx, nz, par, 0, 1, 1, 1);
        taper_all(n0, nx, nz, par, 0, 1, 1, 1);
        taper_all(n1, nx, nz, par, 0, 1, 1, 1);

        real *ba = preva; preva = curra; curra = nexta; nexta = ba;
        real *b = prev; prev = curr; curr = next; next = b;
    }
    if (full && sub > 0 && (nt - 1) % sub == 0 && !grad) memcpy(full + (long)((nt - 1) / sub) * 2 * nxz, curr, 2 * nxz * sizeof(real));
    if (!grad) {
        if (!adj) {
            extract(ext, curr, rcvx, nz, nt, nt - 1);
            extract(ext, curr + nxz, rcvz, nz, nt, nt - 1);
            extract(exta, curra, rcva, nza, nt, nt - 1);
        } else {
            if (!par->acoustic_source) {
                extract(ext, curr, rcvx, nz, nt, nt - 1);
                extract(ext, curr + nxz, rcvz, nz, nt, nt - 1);
            } else extract(exta, curra, rcva, nza, nt, nt - 1);
        }
    }
    /* the reference adds no final-sample gradient for this propagator */
    free(u); free(dux); free(duz); free(phi); free(moda); free(tmp);
    free(f2mu); free(fimp_s); free(fimp_p);
}

/* ---------------------------------------------------------------------------
 * Exported entry point.
 * kind: 0 elastic, 1 VTI, 2 acoustic, 3 acoustic-elastic.
 * Returns 0 on success, negative on invalid arguments.
 * ------------------------------------------------------------------------- */
int ORC(propagate)(int kind, int adj, const void *model, const void *allsrc, void *allrcv,
                   const orc_injector *inj, const orc_injector *ext,
                   const orc_injector *inja, const orc_injector *exta,
                   void *full_wfld, void *grad, const orc_param *par,
                   int nx, int nz, double dx, double dz)
{
    init_tables();
    if (nx < 12 || nz < 12 || par->nt < 2) return -1;
    if (par->sub <= 0 && grad) return -2;
    if (kind == 0 || kind == 1)
        propagate_elastic(kind == 1, adj, (const real *)model, (const real *)allsrc, (real *)allrcv, inj, ext,
                          (real *)full_wfld, (real *)grad, par, nx, nz, (real)dx, (real)dz);
    else if (kind == 2)
        propagate_acoustic(adj, (const real *)model, (const real *)allsrc, (real *)allrcv, inj, ext,
                           (real *)full_wfld, (real *)grad, par, nx, nz, (real)dx, (real)dz);
    else if (kind == 3) {
        if (par->nza < 12) return -3;
        propagate_ae(adj, (const real *)model, (const real *)allsrc, (real *)allrcv, inj, ext, inja, exta,
                     (real *)full_wfld, (real *)grad, par, nx, nz, (real)dx, (real)dz);
    } else return -4;
    return 0;
}

/* Model conversions (we_op.cpp:476-494, 1441-1462, 1863-1881), in place on
 * [npar][n]. */
void ORC(convert_model)(int kind, void *m_, int n, int forward)
{
    real *m = (real *)m_;
    real *p0 = m, *p1 = m + n, *p2 = m + 2L * n, *p3 = m + 3L * n;
    for (int i = 0; i < n; i++) {
        if (kind == 2) {
            if (forward) { p0[i] = p1[i] * p0[i] * p0[i]; p1[i] = (real)(1.0 / p1[i]); }
            else { p0[i] = R_SQRT(p0[i] * p1[i]); p1[i] = (real)(1.0 / p1[i]); }
        } else if (forward) {
            p0[i] = p2[i] * (p0[i] * p0[i] - 2 * p1[i] * p1[i]);
            p1[i] = p2[i] * p1[i] * p1[i];
            if (kind == 1)
                p3[i] = (real)(DS(2 * (p0[i] + 2 * p1[i]) * (p0[i] + p1[i]) * p3[i] + (p0[i] + p1[i]) * (p0[i] + p1[i])) - p1[i]);
        } else {
            if (kind == 1)
                p3[i] = ((p3[i] + p1[i]) * (p3[i] + p1[i]) - (p0[i] + p1[i]) * (p0[i] + p1[i])) / (2 * (p0[i] + p1[i]) * (p0[i] + 2 * p1[i]));
            p0[i] = R_SQRT((p0[i] + 2 * p1[i]) / p2[i]);
            p1[i] = R_SQRT(p1[i] / p2[i]);
        }
    }
}

int ORC(real_size)(void) { return (int)sizeof(real); }

/* ---------------------------------------------------------------------------
 * Time resampling (src/cpp/operator.cpp:755-856): the windowed-sinc and the
 * linear resampler between a domain time axis (nm samples at dm) and a range
 * axis (np samples at dp), both from t = 0, on ntr traces, add = false.
 *   adjoint = 0: in [ntr][nm] -> out [ntr][np]   (apply_forward, interpolation)
 *   adjoint = 1: in [ntr][np] -> out [ntr][nm]   (apply_adjoint, decimation)
 * Same operation order and promotions: the sinc argument and the cosine
 * window are formed in double from single-precision times (M_PI is a double),
 * sinc(x) = sin(x)/x with x rounded to the sample type and sin evaluated in
 * double (the reference's unqualified sin of a float resolves to ::sin(double)),
 * and each product pmod*sinc (sample type) times the window (double) is added
 * in double to the output sample.  The window is a + (1-a) cos(pi (itm - t/dm)
 * / hl) with a = 1/2 (sinc_resampler's default alpha).
 * ------------------------------------------------------------------------- */
static real sinc_(real x)
{
    if (x == 0.0) return 1.0;
    return (real)(sin((double)x) / (double)x);
}

int ORC(resample)(int linear, int adjoint, int hl, int ntr, int nm, double dm_, int np, double dp_,
                   const void *in_, void *out_)
{
    const real *in = (const real *)in_;
    real *out = (real *)out_;
    const real dm = (real)dm_, dp = (real)dp_, a = (real)0.5;
    if (adjoint) memset(out, 0, (size_t)ntr * nm * sizeof(real));
    OMP_FOR
    for (int ix = 0; ix < ntr; ix++) {
        const real *pm = adjoint ? NULL : in + (size_t)ix * nm;
        const real *pd = adjoint ? in + (size_t)ix * np : NULL;
        real *om = adjoint ? out + (size_t)ix * nm : NULL;
        real *od = adjoint ? NULL : out + (size_t)ix * np;
        for (int itd = 0; itd < np; itd++) {
            if (linear) {
                const real x = itd * dp / dm;
                int i = (int)floor(x), j = (int)ceil(x);
                if (i > nm - 1) i = nm - 1;
                if (j > nm - 1) j = nm - 1;
                const real wj = (itd * dp - i * dm) / dm, wi = 1 - wj;
                if (!adjoint) od[itd] = wi * pm[i] + wj * pm[j];
                else {
                    om[i] += wi * pd[itd];
                    om[j] += wj * pd[itd];
                }
                continue;
            }
            const real t = itd * dp;
            const int itm0 = (int)floor(t / dm);
            const int lo = itm0 - hl + 1 > 0 ? itm0 - hl + 1 : 0;
            const int hi = itm0 + hl < nm - 1 ? itm0 + hl : nm - 1;
            if (!adjoint) od[itd] = 0;
            for (int itm = lo; itm <= hi; itm++) {
                const real s = sinc_((real)(M_PI * (t - itm * dm) / dm));
                const double w = a + (1 - a) * cos(M_PI * (itm - t / dm) / hl);
                if (!adjoint) od[itd] = (real)(od[itd] + (double)(pm[itm] * s) * w);
                else om[itm] = (real)(om[itm] + (double)(pd[itd] * s) * w);
            }
        }
    }
    return 0;
}
