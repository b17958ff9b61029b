// Device-side data structures shared by the propagation kernels and the host
// engine.  Layouts follow the reference (src/cpp/we_op.cpp:564-902): every
// 2-D array is x-major with z contiguous, a[ix*ldz + iz]; ldz is nz rounded
// up to a multiple of 32 so that each x-row starts on a 128-byte boundary.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fwi2d {

enum Kind { KIND_ELASTIC = 0, KIND_VTI = 1, KIND_ACOUSTIC = 2, KIND_AE = 3 };
enum SnapPrec { SNAP_FP32 = 0, SNAP_BF16 = 1, SNAP_FP16 = 2 };

// One injection contribution to one cell.  delta_m3: out += wa*S[ia];
// ddelta_m3 (moment tensor): out += wa*S[ia] - wb*S[ib]  (injector.cpp:91-112, 214-239).
struct InjEntry {
    int gx, gz;       // cell on the shot's grid
    int comp;         // field component (0: x / potential, 1: z)
    int mt;           // 1 for the moment-tensor form
    int ia, ib;       // rows of the time-major source block
    float wa, wb;     // xw*zw products (reference order)
};

// One receiver sample: o = sum_{i,k} w[3i+k] * u[gx0+i][gz0+k]  (injector.cpp:68-89).
struct ExtEntry {
    int row;          // output row in the time-major trace block
    int comp;         // field component read
    int gx0, gz0;     // first of the 3x3 cells
    float w[9];
};

// Initial "prev" of the leapfrog (we_op.cpp:657-663): the cell accumulates its
// injection entries idx[i0..i1) at time sample 0 in the reference's order,
// then is scaled in double by `factor` (dt^2/(2 rho), or K dt^2/2 acoustic).
struct InitCell {
    int gx, gz, comp, i0, i1, pad;
    double factor;
};

// One row of a marching unit: its source entries [e0, e1) (sorted by z,
// spanning [zlo, zhi]), its receivers [r0, r1) and its taper factor.  32 bytes,
// fetched by one bulk copy per row.
struct MarchRow {
    int e0, e1, zlo, zhi, r0, r1;
    float tx;
    int pad;
};

struct ShotDev {
    int nx, nz, ldz;      // shot grid (nz == model nz)
    int x0;               // first model column of this shot's grid
    int nt;               // time samples of this shot
    float *u[2];          // two field buffers, each [ncomp][nx][ldz]
    const float *src;     // time-major injection traces [nt][nsrc]
    int nsrc;
    float *rcv;           // time-major extraction output [nt][nrcv]
    int nrcv;
    const InjEntry *inj;  // grouped by work unit; march units sorted by (x, z), reference order per cell
    const int *inj_off;   // [units+1]
    const ExtEntry *ext;  // grouped by the unit owning the pivot; march units sorted by pivot row
    const int *ext_off;   // [units+1]
    int n_ext;
    const struct MarchRow *mrow;   // per march unit and row (MarchRef::roff + row - xb)
    const float *den;     // absorbing-boundary divisors: [ncomp][2*nx + 2*nz] (top, bottom, left, right)
    const float *tz;      // taper factor along z [nz]
    const float *tx;      // taper factor along x [nx]
    void *snap;           // snapshots [nslot][ncomp][nx][ldz] in fp32/bf16/fp16
    long long snap_slot;  // elements per slot
    float *snap_inv;      // per-slot dequantisation factor (16-bit snapshots)
    unsigned *snap_amax;  // per-slot max |u| bits (16-bit snapshots)
    float *grad;          // [3 or 2][nx][ldz] gradient accumulator of this shot
    float *gcomp;         // compensated accumulation: running sum pair hi [3 or 2][nx][ldz], then lo; or nullptr
    float *halo_save;     // interface scratch (acoustic-elastic) or nullptr
    const float *gwt;     // gradient time-damping weight per snapshot index
    float *ckpt;          // checkpoints [k][2][ncomp][nx][ldz] (checkpoint-and-recompute) or nullptr
};

// Model on the full grid; shots index it at column x0 + ix.
struct ModelDev {
    int nx, nz, ldz;
    const float *p0, *p1, *p2;   // elastic: lambda, mu, rho.  acoustic: K, 1/rho
    const float *c13, *eps;      // VTI
    const float *fxx;            // VTI: (1+2eps)*2mu ; elastic: unused
    const float *lbis;           // VTI: (1+2eps)*lambda
    const float *gv2, *gv3;      // VTI gradient: dC13/dlambda, dC13/dmu
};

// Scalars of one propagation, each computed on the host exactly as the
// reference computes it (float arithmetic unless noted).
struct StepConst {
    float dt, dt2;               // dt, dt*dt
    float inv_d2x, inv_d2z;      // 1/(dx*dx), 1/(dz*dz)       (Dxx_var/Dzz_var a/d2)
    float adx, adz;              // 1/dx, 1/dz                 (mult_Dx/mult_Dz a/d)
    float sdx, sdz;              // (float)(1.0/(double)d)     (Dx/Dz interior scale)
    float dx, dz;
    float d2x, d2z;              // dx*dx, dz*dz
    float sat_x, sat_z;          // 1/(dx*h0), 1/(dz*h0)       (esat_* a/(d*h0))
    float nsat_x, nsat_z;        // 1/(dx*dx*h0), 1/(dz*dz*h0) (esat_D* a/(d*d*h0))
    float alpha;                 // acoustic free-surface stiffness factor
    int bc[4];                   // top, bottom, left, right
    int sub;
    int snap_prec;
    int nslot;
    int spin;                    // poll limit of each bounded device wait (marching kernel)
};

// Work unit of the tile kernel: a TX x TZ window of one shot grid starting
// at (wx0, wz0) that writes the cells of [ox0, ox1) x [oz0, oz1).
struct TileRef {
    int shot, unit;
    int wx0, ox0, ox1;
    int wz0, oz0, oz1;
};

// Work unit of the x-marching kernel: rows [xb, xe) (all clear of the x
// boundary bands) of a z window of 2*blockDim.x cells starting at za (even,
// -2 for the first window) that writes the cells of [oz0, oz1).  roff is the
// first of this unit's (xe - xb + 1) per-row offsets and row records.
struct MarchRef {
    int shot, unit;
    int xb, xe;
    int za, oz0, oz1;
    int roff;
};

// Work unit of the top / bottom band kernel: rows [xb, xe) of one shot's
// top (side 0: z < 6) or bottom (side 1: z >= nz-6) band; roff as MarchRef.
struct BandRef {
    int shot, unit;
    int xb, xe;
    int side, roff;
};

// Tile k of an axis of n samples with tiles of T (n == T or n >= T + 8):
// the window [min(kT, n-T), +T) owns the cells up to the next window, the
// last window is flush with the far boundary.
inline void tile_window_host(int k, int ntile, int n, int T, int &w0, int &o0, int &o1)
{
    auto w = [&](int i) { return i * T < n - T ? i * T : n - T; };
    w0 = w(k);
    o0 = k == 0 ? 0 : w(k);
    o1 = k == ntile - 1 ? n : w(k + 1);
}

}  // namespace fwi2d
