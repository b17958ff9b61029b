// Host-side tables that the kernels consume, each computed with the
// reference's own arithmetic so that the device results match it sample for
// sample.
#pragma once
#include <vector>
#include <cstdint>

struct fwi2d_model_check;   // include/fwi2d_b200.h

namespace fwi2d {

// SBP constants as the reference's initialisers produce them (double rational
// rounded to float): spatial_operators.hpp:34-41, spatial_operators.cpp:102-129.
struct SbpTables {
    float b1[4][6];
    float b2[6][8][8];
    float c2[10];
    float c1[2];
    float sc[4];
    float hc[4];
    float h0;
};
const SbpTables &sbp_tables();

// cos^2 taper factors per z row and per x column (spatial_operators.cpp:523-549
// with the z bands in single precision as the ISPC loop, the x bands in double).
// Bands are applied only where enabled (the acoustic-elastic grids taper a
// subset of their sides).
void taper_factors(int nx, int nz, int t_top, int t_bottom, int t_left, int t_right, float strength,
                   bool use_top, bool use_bottom, bool use_left, bool use_right,
                   std::vector<float> &tz, std::vector<float> &tx);
// The same into caller arrays tz[nz], tx[nx] (no allocation).
void taper_factors_into(int nx, int nz, int t_top, int t_bottom, int t_left, int t_right, float strength,
                        bool use_top, bool use_bottom, bool use_left, bool use_right, float *tz, float *tx);

// Divisors of the implicit absorbing scaling at every boundary sample, laid out
// [ncomp][top nx | bottom nx | left nz | right nz]; 1 where nothing divides.
// Elastic / VTI: esat_scale_boundaries / vtisat_scale_boundaries
// (spatial_operators.cpp:307-521); acoustic: asat_scale_boundaries (:779-860).
void elastic_scale_divisors(int nx, int nz, float dx, float dz, float dt, const float *lam, const float *mu,
                            const float *rho, const float *eps, long long ld, bool top, bool bottom, bool left,
                            bool right, std::vector<float> &den);
// The same into a caller array den[2 * (2*nx + 2*nz)] (no allocation).
void elastic_scale_divisors_into(int nx, int nz, float dx, float dz, float dt, const float *lam, const float *mu,
                                 const float *rho, const float *eps, long long ld, bool top, bool bottom, bool left,
                                 bool right, float *den);
void acoustic_scale_divisors(int nx, int nz, float dx, float dz, float dt, const float *K, const float *irho,
                             long long ld, bool top, bool bottom, bool left, bool right, std::vector<float> &den);

// delta_m3 / ddelta_m3::findIndicesWeights (injector.cpp:3-64, 114-187).
// xw, zw: [ntr][2][3] (type 0) or [ntr][2][6] (type 1).
// analyzeModel (we_op.cpp:267-474) on a raw model [npar][nx][nz], in place.
void analyze_model(int npar, float *model, int nx, int nz, float dx, float dz, int data_nt, float data_dt,
                   fwi2d_model_check &c);

// dipole_m3::findIndicesWeights (injector.cpp:241-326).
void dipole_weights(int ntr, const float *locx, const float *locz, const float *dip, float gl, int nx, int nz,
                    float dx, float dz, float ox, float oz, int *xind, int *zind, float *xw, float *zw);

void injector_weights(int type, int ntr, const float *locx, const float *locz, int nx, int nz, float dx, float dz,
                      float ox, float oz, int *xind, int *zind, float *xw, float *zw);

}  // namespace fwi2d
