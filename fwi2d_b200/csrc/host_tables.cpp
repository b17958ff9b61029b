#include "host_tables.h"
#include "../../include/fwi2d_b200.h"
#include <algorithm>
#include <cmath>
#include <cstring>

namespace fwi2d {

namespace {
struct Q { int r, j, k; long long num, den; };

// Nonzero entries of the 4x6 first-derivative closure (spatial_operators.cpp:102).
const Q kD1[] = {
    {0, 0, 0, -24, 17}, {0, 0, 1, 59, 34}, {0, 0, 2, -4, 17}, {0, 0, 3, -3, 34},
    {0, 1, 0, -1, 2}, {0, 1, 2, 1, 2},
    {0, 2, 0, 4, 43}, {0, 2, 1, -59, 86}, {0, 2, 3, 59, 86}, {0, 2, 4, -4, 43},
    {0, 3, 0, 3, 98}, {0, 3, 2, -59, 98}, {0, 3, 4, 32, 49}, {0, 3, 5, -4, 49},
};

// Nonzero entries of the 6x8x8 variable-coefficient second-derivative closure
// (spatial_operators.hpp:34-41): row r, column j, coefficient sample k.
const Q kD2[] = {
#include "d2_closure.inc"
};

SbpTables make_tables()
{
    SbpTables t;
    std::memset(&t, 0, sizeof(t));
    for (const Q &q : kD1) t.b1[q.j][q.k] = (float)((double)q.num / (double)q.den);
    for (const Q &q : kD2) t.b2[q.r][q.j][q.k] = (float)((double)q.num / (double)q.den);
    const double c2[10] = {-3.0 / 4, -5.0 / 6, -1.0 / 24, 1.0 / 6, 1.0 / 2, 1.0 / 2, 1.0 / 6, -1.0 / 8, 1.0 / 6, -1.0 / 8};
    for (int i = 0; i < 10; i++) t.c2[i] = (float)c2[i];
    t.c1[0] = (float)(2.0 / 3);
    t.c1[1] = (float)(-1.0 / 12);
    t.sc[0] = (float)(11.0 / 6); t.sc[1] = -3.f; t.sc[2] = 1.5f; t.sc[3] = (float)(-1.0 / 3);
    t.hc[0] = (float)(17.0 / 48); t.hc[1] = (float)(59.0 / 48); t.hc[2] = (float)(43.0 / 48); t.hc[3] = (float)(49.0 / 48);
    t.h0 = (float)(17.0 / 48);
    return t;
}
}  // namespace

const SbpTables &sbp_tables()
{
    static const SbpTables t = make_tables();
    return t;
}

void taper_factors(int nx, int nz, int t_top, int t_bottom, int t_left, int t_right, float a,
                   bool use_top, bool use_bottom, bool use_left, bool use_right,
                   std::vector<float> &tz, std::vector<float> &tx)
{
    tz.resize(nz);
    tx.resize(nx);
    taper_factors_into(nx, nz, t_top, t_bottom, t_left, t_right, a, use_top, use_bottom, use_left, use_right,
                       tz.data(), tx.data());
}

void taper_factors_into(int nx, int nz, int t_top, int t_bottom, int t_left, int t_right, float a,
                        bool use_top, bool use_bottom, bool use_left, bool use_right, float *tz, float *tx)
{
    std::fill(tz, tz + nz, 1.f);
    std::fill(tx, tx + nx, 1.f);
    const float pi = (float)M_PI, half = 0.5f;
    if (use_top && t_top > 0) {
        const int istart = t_top, iend = 0;
        for (int i = 0; i < istart; i++) {
            float v = std::cos(a * half * pi * (float)(i + 1 - istart) / (float)(iend - istart));
            tz[i] = tz[i] * (v * v);
        }
    }
    if (use_bottom && t_bottom > 0) {
        const int istart = nz - t_bottom, iend = nz;
        for (int i = istart; i < iend; i++) {
            float v = std::cos(a * half * pi * (float)(i - istart) / (float)(iend - istart));
            tz[i] = tz[i] * (v * v);
        }
    }
    if (use_left && t_left > 0) {
        const int istart = t_left, iend = 0;
        for (int i = 0; i < istart; i++) {
            float v = (float)std::cos(a * 0.5 * M_PI * (i + 1 - istart) / (iend - istart));
            tx[i] = tx[i] * (v * v);
        }
    }
    if (use_right && t_right > 0) {
        const int istart = nx - t_right, iend = nx;
        for (int i = istart; i < iend; i++) {
            float v = (float)std::cos(a * 0.5 * M_PI * (i - istart) / (iend - istart));
            tx[i] = tx[i] * (v * v);
        }
    }
}

// The reference evaluates each scaler with the double sqrt on float
// arguments and rounds once to float: DS() restates that.
static inline double DS(float x) { return std::sqrt((double)x); }

void elastic_scale_divisors(int nx, int nz, float dx, float dz, float dt, const float *lam, const float *mu,
                            const float *rho, const float *eps, long long ld, bool top, bool bottom, bool left,
                            bool right, std::vector<float> &den)
{
    den.resize(2 * (2 * nx + 2 * nz));
    elastic_scale_divisors_into(nx, nz, dx, dz, dt, lam, mu, rho, eps, ld, top, bottom, left, right, den.data());
}

void elastic_scale_divisors_into(int nx, int nz, float dx, float dz, float dt, const float *lam, const float *mu,
                                 const float *rho, const float *eps, long long ld, bool top, bool bottom, bool left,
                                 bool right, float *den)
{
    const int per = 2 * nx + 2 * nz;
    std::fill(den, den + 2 * per, 1.f);
    auto T = [&](int ix) -> float * { return &den[ix]; };
    auto B = [&](int ix) -> float * { return &den[nx + ix]; };
    auto L = [&](int iz) -> float * { return &den[2 * nx + iz]; };
    auto R = [&](int iz) -> float * { return &den[2 * nx + nz + iz]; };
    auto set = [&](float *p0, float s0, float s1) { p0[0] = 1 + s0; p0[per] = 1 + s1; };
    auto at = [&](int ix, int iz) { return (long long)ix * ld + iz; };
    auto cxx = [&](long long i) -> float {
        return eps ? (1 + 2 * eps[i]) * (lam[i] + 2 * mu[i]) : (lam[i] + 2 * mu[i]);
    };
    const float h0 = sbp_tables().h0;
    const double ddt = (double)dt, vz = (double)(2 * dz * h0), vx = (double)(2 * dx * h0);
    float sc1x = 0, sc1z = 0, sc2x = 0, sc2z = 0;
    if (top) {
        long long c0 = at(0, 0), c1 = at(nx - 1, 0);
        sc1x = (float)(DS(mu[c0] / rho[c0]) * ddt / vz);
        sc1z = (float)(sc1x * DS((lam[c0] + 2 * mu[c0]) / mu[c0]));
        sc2x = (float)(DS(mu[c1] / rho[c1]) * ddt / vz);
        sc2z = (float)(sc1x * DS((lam[c1] + 2 * mu[c1]) / mu[c1]));
        for (int ix = 1; ix < nx - 1; ix++) {
            long long i = at(ix, 0);
            float sx = (float)(DS(mu[i] / rho[i]) * ddt / vz);
            float sz = (float)(sx * DS((lam[i] + 2 * mu[i]) / mu[i]));
            set(T(ix), sx, sz);
        }
    }
    if (left) {
        long long c0 = at(0, 0), b = at(0, nz - 1);
        sc1x = (float)(sc1x + DS(cxx(c0) / rho[c0]) * ddt / vx);
        sc1z = (float)(sc1z + DS(mu[c0] / rho[c0]) * ddt / vx);
        set(T(0), sc1x, sc1z);
        sc1x = (float)(DS(cxx(b) / rho[b]) * ddt / vx);
        sc1z = (float)(sc1x * DS(mu[b] / cxx(b)));
        for (int iz = 1; iz < nz - 1; iz++) {
            long long i = at(0, iz);
            float sx = (float)(DS(cxx(i) / rho[i]) * ddt / vx);
            float sz = (float)(sx * DS(mu[i] / cxx(i)));
            set(L(iz), sx, sz);
        }
    } else {
        set(T(0), sc1x, sc1z);
        sc1x = 0;
        sc1z = 0;
    }
    if (bottom) {
        long long b = at(0, nz - 1), c = at(nx - 1, nz - 1);
        sc1x = (float)(sc1x + DS(mu[b] / rho[b]) * ddt / vz);
        sc1z = (float)(sc1z + DS((lam[b] + 2 * mu[b]) / rho[b]) * ddt / vz);
        set(B(0), sc1x, sc1z);
        sc1x = (float)(DS(mu[c] / rho[c]) * ddt / vz);
        sc1z = (float)(sc1x * DS((lam[c] + 2 * mu[c]) / mu[c]));
        for (int ix = 1; ix < nx - 1; ix++) {
            long long i = at(ix, nz - 1);
            float sx = (float)(DS(mu[i] / rho[i]) * ddt / vz);
            float sz = (float)(sx * DS((lam[i] + 2 * mu[i]) / mu[i]));
            set(B(ix), sx, sz);
        }
    } else {
        set(B(0), sc1x, sc1z);
        sc1x = 0;
        sc1z = 0;
    }
    if (right) {
        long long c = at(nx - 1, nz - 1), t = at(nx - 1, 0);
        sc1x = (float)(sc1x + DS(cxx(c) / rho[c]) * ddt / vx);
        sc1z = (float)(sc1z + DS(mu[c] / rho[c]) * ddt / vx);
        set(B(nx - 1), sc1x, sc1z);
        for (int iz = 1; iz < nz - 1; iz++) {
            long long i = at(nx - 1, iz);
            float sx = (float)(DS(cxx(i) / rho[i]) * ddt / vx);
            float sz = (float)(sx * DS(mu[i] / cxx(i)));
            set(R(iz), sx, sz);
        }
        sc2x = (float)(sc2x + DS(cxx(t) / rho[t]) * ddt / vx);
        sc2z = (float)(sc2z + DS(mu[t] / rho[t]) * ddt / vx);
        set(T(nx - 1), sc2x, sc2z);
    } else {
        set(B(nx - 1), sc1x, sc1z);
        set(T(nx - 1), sc2x, sc2z);
    }
}

void acoustic_scale_divisors(int nx, int nz, float dx, float dz, float dt, const float *K, const float *irho,
                             long long ld, bool top, bool bottom, bool left, bool right, std::vector<float> &den)
{
    const int per = 2 * nx + 2 * nz;
    den.assign(per, 1.f);
    auto at = [&](int ix, int iz) { return (long long)ix * ld + iz; };
    const float h0 = sbp_tables().h0;
    const double ddt = (double)dt, vz = (double)(2 * dz * h0), vx = (double)(2 * dx * h0);
    float sc1 = 0, sc2 = 0;
    if (top) {
        long long c0 = at(0, 0), t = at(nx - 1, 0);
        sc1 = (float)(DS(K[c0] * irho[c0]) * ddt / vz);
        sc2 = (float)(DS(K[t] * irho[t]) * ddt / vz);
        for (int ix = 1; ix < nx - 1; ix++) {
            long long i = at(ix, 0);
            den[ix] = 1 + (float)(DS(K[i] * irho[i]) * ddt / vz);
        }
    }
    if (left) {
        long long c0 = at(0, 0), b = at(0, nz - 1);
        sc1 = (float)(sc1 + DS(K[c0] * irho[c0]) * ddt / vx);
        den[0] = 1 + sc1;
        sc1 = (float)(DS(K[b] * irho[b]) * ddt / vx);
        for (int iz = 1; iz < nz - 1; iz++) {
            long long i = at(0, iz);
            den[2 * nx + iz] = 1 + (float)(DS(K[i] * irho[i]) * ddt / vx);
        }
    } else {
        den[0] = 1 + sc1;
        sc1 = 0;
    }
    if (bottom) {
        long long b = at(0, nz - 1), c = at(nx - 1, nz - 1);
        sc1 = (float)(sc1 + DS(K[b] * irho[b]) * ddt / vz);
        den[nx] = 1 + sc1;
        sc1 = (float)(DS(K[c] * irho[c]) * ddt / vz);
        for (int ix = 1; ix < nx - 1; ix++) {
            long long i = at(ix, nz - 1);
            den[nx + ix] = 1 + (float)(DS(K[i] * irho[i]) * ddt / vz);
        }
    } else {
        den[nx] = 1 + sc1;
        sc1 = 0;
    }
    if (right) {
        long long c = at(nx - 1, nz - 1), t = at(nx - 1, 0);
        sc1 = (float)(sc1 + DS(K[c] * irho[c]) * ddt / vx);
        den[nx + nx - 1] = 1 + sc1;
        for (int iz = 1; iz < nz - 1; iz++) {
            long long i = at(nx - 1, iz);
            den[2 * nx + nz + iz] = 1 + (float)(DS(K[i] * irho[i]) * ddt / vx);
        }
        sc2 = (float)(sc2 + DS(K[t] * irho[t]) * ddt / vx);
        den[nx - 1] = 1 + sc2;
    } else {
        den[nx + nx - 1] = 1 + sc1;
        den[nx - 1] = 1 + sc2;
    }
}

static float hcoef_at(int n, int i)
{
    const float *hc = sbp_tables().hc;
    if (i < 4) return hc[i];
    if (i >= n - 4) return hc[n - 1 - i];
    return 1.f;
}

// dipole_m3::findIndicesWeights (injector.cpp:241-326): the two ends lie at
// loc -/+ gl/2 (cos dip, sin dip).  The end positions, pivots and alphas are
// formed in double (the reference's cos / sin of a float resolve to the
// double functions) and the alphas rounded to single precision; the weights
// are the delta_m3 formulas in double from the single-precision alphas.
void dipole_weights(int ntr, const float *locx, const float *locz, const float *dip, float gl, int nx, int nz,
                    float dx, float dz, float ox, float oz, int *xind, int *zind, float *xw, float *zw)
{
    const float h = gl / 2;
    auto pivot = [](double g, int n) {
        int i = (int)std::round(g);
        if (i == 0) i = 1;
        if (i == n - 1) i = n - 2;
        return i;
    };
    for (int t = 0; t < ntr; t++) {
        const double c = std::cos((double)dip[t]), s = std::sin((double)dip[t]);
        const double gx[2] = {((double)locx[t] - h * c - ox) / dx, ((double)locx[t] + h * c - ox) / dx};
        const double gz[2] = {((double)locz[t] - h * s - oz) / dz, ((double)locz[t] + h * s - oz) / dz};
        int *xi = xind + 6 * t, *zi = zind + 6 * t;
        float *xi0 = xw + 12 * t, *xe = xi0 + 6, *zi0 = zw + 12 * t, *ze = zi0 + 6;
        for (int e = 0; e < 2; e++) {
            const int px = pivot(gx[e], nx), pz = pivot(gz[e], nz);
            for (int k = 0; k < 3; k++) {
                xi[3 * e + k] = px - 1 + k;
                zi[3 * e + k] = pz - 1 + k;
            }
            const float ax = (float)(gx[e] - px), az = (float)(gz[e] - pz);
            const double ax2 = (double)ax * (double)ax, az2 = (double)az * (double)az;
            float *wx = xi0 + 3 * e, *vx = xe + 3 * e, *wz = zi0 + 3 * e, *vz = ze + 3 * e;
            wx[0] = (float)((ax2 - ax) / (double)(2 * dx * hcoef_at(nx, px - 1)));
            wx[1] = (float)((-ax2 + 1) / (double)(dx * hcoef_at(nx, px)));
            wx[2] = (float)((ax2 + ax) / (double)(2 * dx * hcoef_at(nx, px + 1)));
            wz[0] = (float)((az2 - az) / (double)(2 * dz * hcoef_at(nz, pz - 1)));
            wz[1] = (float)((-az2 + 1) / (double)(dz * hcoef_at(nz, pz)));
            wz[2] = (float)((az2 + az) / (double)(2 * dz * hcoef_at(nz, pz + 1)));
            vx[0] = (float)((ax2 - ax) / 2);
            vx[1] = (float)(-ax2 + 1);
            vx[2] = (float)((ax2 + ax) / 2);
            vz[0] = (float)((az2 - az) / 2);
            vz[1] = (float)(-az2 + 1);
            vz[2] = (float)((az2 + az) / 2);
        }
    }
}

void injector_weights(int type, int ntr, const float *locx, const float *locz, int nx, int nz, float dx, float dz,
                      float ox, float oz, int *xind, int *zind, float *xw, float *zw)
{
    const int w = type == 0 ? 3 : 6;
    for (int t = 0; t < ntr; t++) {
        int xi = (int)std::round((locx[t] - ox) / dx);
        int zi = (int)std::round((locz[t] - oz) / dz);
        if (xi == 0) xi = 1;
        if (xi == nx - 1) xi = nx - 2;
        if (zi == 0) zi = 1;
        if (zi == nz - 1) zi = nz - 2;
        for (int k = 0; k < 3; k++) {
            xind[t * 3 + k] = xi - 1 + k;
            zind[t * 3 + k] = zi - 1 + k;
        }
        const float ax = (locx[t] - dx * (float)xi - ox) / dx;
        const float az = (locz[t] - dz * (float)zi - oz) / dz;
        const double ax2 = (double)ax * (double)ax, az2 = (double)az * (double)az;
        float *xi0 = xw + t * 2 * w, *xe = xi0 + w;
        float *zi0 = zw + t * 2 * w, *ze = zi0 + w;
        xi0[0] = (float)((ax2 - ax) / (double)(2 * dx * hcoef_at(nx, xi - 1)));
        xi0[1] = (float)((-ax2 + 1) / (double)(dx * hcoef_at(nx, xi)));
        xi0[2] = (float)((ax2 + ax) / (double)(2 * dx * hcoef_at(nx, xi + 1)));
        zi0[0] = (float)((az2 - az) / (double)(2 * dz * hcoef_at(nz, zi - 1)));
        zi0[1] = (float)((-az2 + 1) / (double)(dz * hcoef_at(nz, zi)));
        zi0[2] = (float)((az2 + az) / (double)(2 * dz * hcoef_at(nz, zi + 1)));
        xe[0] = (float)((ax2 - ax) / 2);
        xe[1] = (float)(-ax2 + 1);
        xe[2] = (float)((ax2 + ax) / 2);
        ze[0] = (float)((az2 - az) / 2);
        ze[1] = (float)(-az2 + 1);
        ze[2] = (float)((az2 + az) / 2);
        if (type == 1) {
            xi0[3] = (1 - 2 * ax) / (2 * dx * dx * hcoef_at(nx, xi - 1));
            xi0[4] = 2 * ax / (dx * dx * hcoef_at(nx, xi));
            xi0[5] = (-1 - 2 * ax) / (2 * dx * dx * hcoef_at(nx, xi + 1));
            zi0[3] = (1 - 2 * az) / (2 * dz * dz * hcoef_at(nz, zi - 1));
            zi0[4] = 2 * az / (dz * dz * hcoef_at(nz, zi));
            zi0[5] = (-1 - 2 * az) / (2 * dz * dz * hcoef_at(nz, zi + 1));
            xe[3] = (1 - 2 * ax) / (2 * dx);
            xe[4] = 2 * ax / dx;
            xe[5] = (-1 - 2 * ax) / (2 * dx);
            ze[3] = (1 - 2 * az) / (2 * dz);
            ze[4] = 2 * az / dz;
            ze[5] = (-1 - 2 * az) / (2 * dz);
        }
    }
}


// analyzeModel (src/cpp/we_op.cpp:267-474), single precision as the
// reference's FP32 build: the delta admissibility bound and the Vs fix are
// formed in double where the reference's literals are doubles (-0.5, 2.0,
// 0.9999, sqrt(2), sqrt(2.0001)), and the VTI horizontal velocity
// vp sqrt(1 + 2 eps) takes the double square root of the single-precision
// 1 + 2 eps.  Clips are max(lo, min(hi, v)) (vecReg::clip).
void analyze_model(int npar, float *m, int nx, int nz, float dx, float dz, int data_nt, float data_dt,
                   fwi2d_model_check &c)
{
    const long n = (long)nx * nz;
    auto lo = [&](int k) { return *std::min_element(m + k * n, m + (k + 1) * n); };
    auto hi = [&](int k) { return *std::max_element(m + k * n, m + (k + 1) * n); };
    auto clip = [&](int k, float a, float b) {
        for (long i = k * n; i < (k + 1) * n; i++) m[i] = std::max(a, std::min(b, m[i]));
    };
    if (npar >= 3) {
        float vpmax = hi(0), vsmin = lo(1);
        if (npar == 5) {
            // Thomsen delta inside -0.5 (1 - vs^2/vp^2) < delta < 2 / (vp^2/vs^2 - 1) (we_op.cpp:296-316)
            const float *vp = m, *vs = m + n;
            float *del = m + 3 * n;
            for (long i = 0; i < n; i++) {
                const float v1 = (float)(-0.5 * (1 - vs[i] * vs[i] / (vp[i] * vp[i])));
                const float v2 = (float)(2.0 / (vp[i] * vp[i] / (vs[i] * vs[i]) - 1));
                if (del[i] < v1) del[i] = (float)(0.9999 * v1);
                else if (del[i] > v2) del[i] = (float)(0.9999 * v2);
            }
        }
        if (!c.soft_clip) {
            clip(0, c.vpmin, c.vpmax);
            clip(1, c.vsmin, c.vsmax);
            clip(2, c.rhomin, c.rhomax);
            if (npar == 5) {
                clip(3, c.deltamin, c.deltamax);
                clip(4, c.epsilonmin, c.epsilonmax);
            }
            // Vs <= Vp / sqrt(2) (we_op.cpp:352-361)
            for (long i = 0; i < n; i++)
                if ((double)m[i] < std::sqrt(2.0) * (double)m[n + i]) m[n + i] = (float)((double)m[i] / std::sqrt(2.0001));
            vpmax = hi(0);
            vsmin = lo(1);
        }
        c.vmax = vpmax;
        c.vmin = vsmin;
        if (npar == 5) {
            float h = 0.f;
            for (long i = 0; i < n; i++) {
                const float v = (float)((double)m[i] * std::sqrt((double)(1 + 2 * m[4 * n + i])));
                h = i == 0 ? v : std::max(h, v);
            }
            c.vmax = std::max(h, c.vmax);
        }
        if (c.acoustic_elastic) {
            c.vmax = std::max(c.vmax, c.water_velocity);
            c.vmin = std::min(c.vmin, c.water_velocity);
        }
    } else {
        clip(0, c.vpmin, c.vpmax);
        clip(1, c.rhomin, c.rhomax);
        c.vmax = hi(0);
        c.vmin = lo(0);
    }
    // time axis (we_op.cpp:436-472)
    const float tmax = (data_nt - 1) * data_dt;
    const float h = std::min(dx, dz);
    if (c.dt == 0.f) {
        c.dt = c.courant * h / c.vmax;
    } else if (c.dt > 0.f) {
        c.dt = std::min(c.dt, data_dt);
        c.courant = c.dt * c.vmax / h;
    } else {
        c.dt = c.courant * h / c.vmax;
        if (data_dt > c.dt) c.dt = data_dt / std::ceil(data_dt / c.dt);
        else c.dt = data_dt;
        c.courant = c.dt * c.vmax / h;
    }
    c.nt = (int)std::round(tmax / c.dt) + 1;
    c.tmax = (c.nt - 1) * c.dt;
    if (c.sub < 0) c.sub = (int)std::round(data_dt / c.dt);
}

}  // namespace fwi2d
