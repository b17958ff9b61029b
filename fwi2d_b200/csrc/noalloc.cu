// fwi2d_propagate_noalloc: the elastic forward propagation of one shot with
// no device or host memory allocation.
//
// Some callers cannot allocate device memory: plug-ins loaded into a host
// process that owns the device allocator (a framework's caching pool that must
// account for every byte on the device), and real-time loops that forbid
// allocation after start-up (cudaMalloc and cudaFree can synchronise the
// device and take unbounded time).  For them this entry point keeps every device-side buffer of the
// propagation -- the pitched model, the two wavefield buffers, the time-major
// traces and the injection / extraction / boundary tables -- in one
// file-scope static __device__ array of FWI2D_NOALLOC_SCRATCH_BYTES (64 MiB),
// and its host-side tables in fixed-size static host arrays.  A GPU holds
// the 64 MiB from the first call on it until the process exits.
//
// Contract:
// * inputs and outputs are host buffers with the reference's propagate
//   layout (as fwi2d_propagate with adj = 0, sub = 0): the receivers are
//   accumulated into allrcv;
// * the problem must fit the scratch array and the static tables (at most
//   FWI2D_NOALLOC_MAX_* of each); larger ones are rejected with
//   FWI2D_ERR_ARG and a message naming the limit;
// * all calls in a process share the scratch array of the current device,
//   which keeps the last call's contents; everything that must start at zero
//   is cleared at the start of each call;
// * every call runs on the legacy default stream (stream 0), not on a stream
//   given to fwi2d_set_stream, so it waits for, and holds up, the work of
//   every blocking stream on the device; it returns only after its GPU work
//   has finished;
// * calls that overlapped on the GPU would race on the shared array; a host
//   mutex serialises the calls of a process and each call finishes its GPU
//   work before it returns, so they never overlap.  Each process (each CUDA
//   context) has its own copy of the array: other processes do not share it;
// * the CUDA runtime loads the module that holds the array lazily (the
//   default since CUDA 12), so the 64 MiB are reserved on a device by the
//   first call on it, which also looks up the array's device address
//   (cudaGetSymbolAddress) with that device current and may synchronise the
//   device.  Make that first call at start-up, before any real-time loop or
//   stream capture; later calls allocate nothing.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "engine.h"
#include "host_tables.h"
#include "launch.h"
#include "../../include/fwi2d_b200.h"

namespace fwi2d {
namespace noalloc {

constexpr size_t kScratchBytes = FWI2D_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxN = FWI2D_NOALLOC_MAX_AXIS;            // samples along x or z
constexpr int kMaxSrc = FWI2D_NOALLOC_MAX_SOURCES;       // source traces
constexpr int kMaxRcv = FWI2D_NOALLOC_MAX_RECEIVERS;     // receiver traces
constexpr int kMaxTiles = 65536;
constexpr int kMaxInj = 2 * 9 * kMaxSrc;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// device address of g_scratch per device, looked up once per device
static unsigned char *g_addr[64];
static std::mutex g_mutex;

// fixed-size host tables
static InjEntry h_inj_raw[kMaxInj], h_inj[kMaxInj];
static int h_inj_tile[kMaxInj];
static ExtEntry h_ext_raw[2 * kMaxRcv], h_ext[2 * kMaxRcv];
static int h_ext_tile[2 * kMaxRcv];
static int h_inj_off[kMaxTiles + 1], h_ext_off[kMaxTiles + 1], h_cnt[kMaxTiles + 1];
static float h_den[2 * (4 * kMaxN)], h_tz[kMaxN], h_tx[kMaxN];
static TileRef h_tiles[kMaxTiles];
static InitCell h_cells[kMaxInj];
static int h_idx[kMaxInj];

static thread_local char g_msg[256];

static int fail(int code, const char *msg)
{
    std::snprintf(g_msg, sizeof(g_msg), "%s", msg);
    return code;
}

static size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

static int owner(int g, int n, int T)
{
    if (g >= n - T) return (n + T - 1) / T - 1;
    return g / T;
}

// stable grouping of entries by tile (counting sort into fixed arrays)
template <class E>
static void group_by_tile(const E *in, const int *tile, int n, int ntiles, E *out, int *off)
{
    for (int t = 0; t <= ntiles; t++) h_cnt[t] = 0;
    for (int i = 0; i < n; i++) h_cnt[tile[i] + 1]++;
    off[0] = 0;
    for (int t = 0; t < ntiles; t++) off[t + 1] = off[t] + h_cnt[t + 1];
    for (int t = 0; t <= ntiles; t++) h_cnt[t] = off[t];
    for (int i = 0; i < n; i++) out[h_cnt[tile[i]]++] = in[i];
}

__global__ void k_add_from_time_major(const float *__restrict__ tm, float *__restrict__ raw, int rows, int nt)
{
    const long long n = (long long)rows * nt;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / nt, t = i - r * nt;
        raw[i] = raw[i] + tm[t * rows + r];
    }
}

}  // namespace noalloc
}  // namespace fwi2d

using namespace fwi2d;
using namespace fwi2d::noalloc;

#define NA_CK(x)                                                                 \
    do {                                                                         \
        cudaError_t e_ = (x);                                                    \
        if (e_ != cudaSuccess) {                                                 \
            (void)cudaGetLastError();                                            \
            return fail(FWI2D_ERR_CUDA, cudaGetErrorString(e_));                 \
        }                                                                        \
    } while (0)

extern "C" const char *fwi2d_noalloc_last_error(void) { return g_msg; }

extern "C" int fwi2d_propagate_noalloc(const float *model, const float *allsrc, float *allrcv,
                                       const fwi2d_injector *inj, const fwi2d_injector *ext,
                                       const fwi2d_params *par, int ns, int nr, int nx, int nz, float dx, float dz)
{
    std::lock_guard<std::mutex> lock(g_mutex);
    g_msg[0] = 0;
    if (!model || !allsrc || !allrcv || !inj || !ext || !par) return fail(FWI2D_ERR_ARG, "null argument");
    const fwi2d_params &p = *par;
    if (nx < 12 || nz < 12 || nx > kMaxN || nz > kMaxN)
        return fail(FWI2D_ERR_ARG, "grid axes must have 12 to FWI2D_NOALLOC_MAX_AXIS samples");
    if (p.nt < 2 || p.dt <= 0 || dx <= 0 || dz <= 0) return fail(FWI2D_ERR_ARG, "invalid nt, dt or spacing");
    if (p.mt || inj->type != FWI2D_INJ_DELTA || ext->type != FWI2D_INJ_DELTA)
        return fail(FWI2D_ERR_UNSUPPORTED, "the allocation-free entry takes point-force sources (delta injectors)");
    if (inj->ntr < 1 || inj->ntr > kMaxSrc) return fail(FWI2D_ERR_ARG, "1 to FWI2D_NOALLOC_MAX_SOURCES source traces");
    if (ext->ntr < 1 || ext->ntr > kMaxRcv) return fail(FWI2D_ERR_ARG, "1 to FWI2D_NOALLOC_MAX_RECEIVERS receivers");
    if (ns < inj->ntr || nr < ext->ntr) return fail(FWI2D_ERR_ARG, "ns / nr smaller than the injector trace counts");
    for (int i = 0; i < 4; i++) {
        const int bc = (&p.bc_top)[i];
        if (bc != 1 && bc != 2) return fail(FWI2D_ERR_ARG, "boundary conditions must be 1 or 2");
    }
    if (p.taper_top < 0 || p.taper_bottom < 0 || p.taper_left < 0 || p.taper_right < 0 ||
        p.taper_top + p.taper_bottom > nz || p.taper_left + p.taper_right > nx)
        return fail(FWI2D_ERR_ARG, "invalid or overlapping tapers");
    for (const fwi2d_injector *J : {inj, ext})
        if (!J->xind || !J->zind || !J->xw || !J->zw) return fail(FWI2D_ERR_ARG, "incomplete injector tables");
    for (const fwi2d_injector *J : {inj, ext})
        for (int t = 0; t < J->ntr; t++)
            for (int k = 0; k < 3; k++)
                if (J->xind[t * 3 + k] < 0 || J->xind[t * 3 + k] >= nx || J->zind[t * 3 + k] < 0 ||
                    J->zind[t * 3 + k] >= nz)
                    return fail(FWI2D_ERR_ARG, "injector index outside the grid");

    // tile shape: the first that tiles the grid
    int shape = -1, TZ = 0, TX = 0;
    for (int i = 0; i < elastic_tile_count() && shape < 0; i++) {
        int tz, tx;
        elastic_tile_shape(i, &tz, &tx);
        if ((nz == tz || nz >= tz + 8) && (nx == tx || nx >= tx + 8)) {
            shape = i;
            TZ = tz;
            TX = tx;
        }
    }
    if (shape < 0) return fail(FWI2D_ERR_ARG, "no tile shape fits the grid");
    const int tiles_x = (nx + TX - 1) / TX, tiles_z = (nz + TZ - 1) / TZ, ntiles = tiles_x * tiles_z;
    if (ntiles > kMaxTiles) return fail(FWI2D_ERR_ARG, "grid too large for the allocation-free entry");

    const int nt = p.nt, ldz = (nz + 31) / 32 * 32;
    const int nsrc = 2 * inj->ntr, nrcv = 2 * ext->ntr;
    const size_t fld = (size_t)nx * ldz * sizeof(float);
    // scratch layout
    size_t o = 0;
    const size_t o_model = o; o += align256(3 * fld);
    const size_t o_u0 = o; o += align256(2 * fld);
    const size_t o_u1 = o; o += align256(2 * fld);
    const size_t o_src_raw = o; o += align256((size_t)nsrc * nt * sizeof(float));
    const size_t o_src = o; o += align256((size_t)nsrc * nt * sizeof(float));
    const size_t o_rcv = o; o += align256((size_t)nrcv * nt * sizeof(float));
    const size_t o_rcv_raw = o; o += align256((size_t)nrcv * nt * sizeof(float));
    const size_t o_inj = o; o += align256(kMaxInj * sizeof(InjEntry));
    const size_t o_inj_off = o; o += align256((ntiles + 1) * sizeof(int));
    const size_t o_ext = o; o += align256((size_t)nrcv * sizeof(ExtEntry));
    const size_t o_ext_off = o; o += align256((ntiles + 1) * sizeof(int));
    const size_t o_den = o; o += align256((size_t)2 * (2 * nx + 2 * nz) * sizeof(float));
    const size_t o_tz = o; o += align256(nz * sizeof(float));
    const size_t o_tx = o; o += align256(nx * sizeof(float));
    const size_t o_gwt = o; o += align256(sizeof(float));
    const size_t o_shot = o; o += align256(sizeof(ShotDev));
    const size_t o_tiles = o; o += align256((size_t)ntiles * sizeof(TileRef));
    const size_t o_cells = o; o += align256(kMaxInj * sizeof(InitCell));
    const size_t o_idx = o; o += align256(kMaxInj * sizeof(int));
    const size_t o_ioff = o; o += align256(2 * sizeof(int));
    if (o > kScratchBytes) {
        std::snprintf(g_msg, sizeof(g_msg),
                      "problem needs %zu bytes of device scratch; the static scratch holds %zu (FWI2D_NOALLOC_SCRATCH_BYTES)",
                      o, kScratchBytes);
        return FWI2D_ERR_ARG;
    }

    int dev = 0;
    NA_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(FWI2D_ERR_ARG, "device index beyond 63");
    if (!g_addr[dev]) {
        // once per device: the SBP coefficient tables the step kernels read
        // (copies into the kernels' constant memory, no allocation), then the
        // scratch array's device address
        const SbpTables &t = sbp_tables();
        upload_sbp_tables(&t.b1[0][0], &t.b2[0][0][0], t.c2, t.c1, t.sc, t.hc);
        NA_CK(cudaGetLastError());
        void *ptr = nullptr;
        NA_CK(cudaGetSymbolAddress(&ptr, g_scratch));
        g_addr[dev] = (unsigned char *)ptr;
    }
    unsigned char *S = g_addr[dev];
    cudaStream_t st = 0;

    // model: lambda, mu, rho pitched to ldz
    for (int k = 0; k < 3; k++)
        NA_CK(cudaMemcpy2DAsync(S + o_model + k * fld, ldz * sizeof(float), model + (size_t)k * nx * nz,
                                nz * sizeof(float), nz * sizeof(float), nx, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemsetAsync(S + o_u0, 0, 2 * fld, st));
    NA_CK(cudaMemsetAsync(S + o_u1, 0, 2 * fld, st));
    // source traces: component blocks of stride ns*nt -> [2*ntr][nt] -> time-major
    for (int c = 0; c < 2; c++)
        NA_CK(cudaMemcpyAsync(S + o_src_raw + (size_t)c * inj->ntr * nt * sizeof(float), allsrc + (size_t)c * ns * nt,
                              (size_t)inj->ntr * nt * sizeof(float), cudaMemcpyHostToDevice, st));
    launch_to_time_major((const float *)(S + o_src_raw), (float *)(S + o_src), nsrc, nt, st);
    NA_CK(cudaGetLastError());

    // injection entries (reference order: component, trace, x, z), grouped by tile
    int ninj = 0;
    for (int c = 0; c < 2; c++)
        for (int t = 0; t < inj->ntr; t++)
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    InjEntry &e = h_inj_raw[ninj];
                    e.gx = inj->xind[t * 3 + a];
                    e.gz = inj->zind[t * 3 + b];
                    e.comp = c;
                    e.mt = 0;
                    e.ia = c * inj->ntr + t;
                    e.ib = 0;
                    e.wa = inj->xw[t * 6 + a] * inj->zw[t * 6 + b];
                    e.wb = 0.f;
                    h_inj_tile[ninj] = owner(e.gz, nz, TZ) * tiles_x + owner(e.gx, nx, TX);
                    ninj++;
                }
    group_by_tile(h_inj_raw, h_inj_tile, ninj, ntiles, h_inj, h_inj_off);
    // receivers
    int next = 0;
    for (int c = 0; c < 2; c++)
        for (int t = 0; t < ext->ntr; t++) {
            ExtEntry &e = h_ext_raw[next];
            e.row = c * ext->ntr + t;
            e.comp = c;
            e.gx0 = ext->xind[t * 3];
            e.gz0 = ext->zind[t * 3];
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) e.w[a * 3 + b] = ext->xw[t * 6 + 3 + a] * ext->zw[t * 6 + 3 + b];
            h_ext_tile[next] = owner(ext->zind[t * 3 + 1], nz, TZ) * tiles_x + owner(ext->xind[t * 3 + 1], nx, TX);
            next++;
        }
    group_by_tile(h_ext_raw, h_ext_tile, next, ntiles, h_ext, h_ext_off);

    // initial state cells (we_op.cpp:657-663)
    int ncell = 0, nidx = 0;
    const float *lam = model, *mu = model + (size_t)nx * nz, *rho = model + 2 * (size_t)nx * nz;
    for (int i = 0; i < ninj; i++) {
        const InjEntry &e = h_inj[i];
        int k = 0;
        while (k < ncell && !(h_cells[k].gx == e.gx && h_cells[k].gz == e.gz && h_cells[k].comp == e.comp)) k++;
        if (k == ncell) {
            std::memset(&h_cells[k], 0, sizeof(InitCell));
            h_cells[k].gx = e.gx;
            h_cells[k].gz = e.gz;
            h_cells[k].comp = e.comp;
            h_cells[k].factor = 0.5 * (double)p.dt * (double)p.dt / (double)rho[(size_t)e.gx * nz + e.gz];
            ncell++;
        }
    }
    for (int k = 0; k < ncell; k++) {
        h_cells[k].i0 = nidx;
        for (int i = 0; i < ninj; i++)
            if (h_inj[i].gx == h_cells[k].gx && h_inj[i].gz == h_cells[k].gz && h_inj[i].comp == h_cells[k].comp)
                h_idx[nidx++] = i;
        h_cells[k].i1 = nidx;
    }
    const int ioff[2] = {0, ncell};

    // the regular path's table helpers, writing into the static host arrays
    elastic_scale_divisors_into(nx, nz, dx, dz, p.dt, lam, mu, rho, nullptr, nz, p.bc_top == 2, p.bc_bottom == 2,
                                p.bc_left == 2, p.bc_right == 2, h_den);
    taper_factors_into(nx, nz, p.taper_top, p.taper_bottom, p.taper_left, p.taper_right, p.taper_strength, true,
                       true, true, true, h_tz, h_tx);
    for (int tzi = 0, k = 0; tzi < tiles_z; tzi++)
        for (int txi = 0; txi < tiles_x; txi++, k++) {
            TileRef &r = h_tiles[k];
            r.shot = 0;
            r.unit = k;
            tile_window_host(txi, tiles_x, nx, TX, r.wx0, r.ox0, r.ox1);
            tile_window_host(tzi, tiles_z, nz, TZ, r.wz0, r.oz0, r.oz1);
        }
    const float one = 1.f;

    ShotDev sd;
    std::memset(&sd, 0, sizeof(sd));
    sd.nx = nx;
    sd.nz = nz;
    sd.ldz = ldz;
    sd.x0 = 0;
    sd.nt = nt;
    sd.n_ext = next;
    sd.u[0] = (float *)(S + o_u0);
    sd.u[1] = (float *)(S + o_u1);
    sd.src = (const float *)(S + o_src);
    sd.nsrc = nsrc;
    sd.rcv = (float *)(S + o_rcv);
    sd.nrcv = nrcv;
    sd.inj = (const InjEntry *)(S + o_inj);
    sd.inj_off = (const int *)(S + o_inj_off);
    sd.ext = (const ExtEntry *)(S + o_ext);
    sd.ext_off = (const int *)(S + o_ext_off);
    sd.den = (const float *)(S + o_den);
    sd.tz = (const float *)(S + o_tz);
    sd.tx = (const float *)(S + o_tx);
    sd.gwt = (const float *)(S + o_gwt);

    NA_CK(cudaMemcpyAsync(S + o_inj, h_inj, ninj * sizeof(InjEntry), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_inj_off, h_inj_off, (ntiles + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_ext, h_ext, next * sizeof(ExtEntry), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_ext_off, h_ext_off, (ntiles + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_den, h_den, (size_t)2 * (2 * nx + 2 * nz) * sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_tz, h_tz, nz * sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_tx, h_tx, nx * sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_gwt, &one, sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_shot, &sd, sizeof(ShotDev), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_tiles, h_tiles, (size_t)ntiles * sizeof(TileRef), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_cells, h_cells, ncell * sizeof(InitCell), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_idx, h_idx, nidx * sizeof(int), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(S + o_ioff, ioff, 2 * sizeof(int), cudaMemcpyHostToDevice, st));

    ModelDev md;
    std::memset(&md, 0, sizeof(md));
    md.nx = nx;
    md.nz = nz;
    md.ldz = ldz;
    md.p0 = (const float *)(S + o_model);
    md.p1 = (const float *)(S + o_model + fld);
    md.p2 = (const float *)(S + o_model + 2 * fld);

    StepConst C;
    std::memset(&C, 0, sizeof(C));
    const float h0 = sbp_tables().h0;
    C.dt = p.dt;
    C.dt2 = p.dt * p.dt;
    C.dx = dx;
    C.dz = dz;
    C.d2x = dx * dx;
    C.d2z = dz * dz;
    C.inv_d2x = 1.f / C.d2x;
    C.inv_d2z = 1.f / C.d2z;
    C.adx = 1.f / dx;
    C.adz = 1.f / dz;
    C.sdx = (float)(1.0 / (double)dx);
    C.sdz = (float)(1.0 / (double)dz);
    C.sat_x = 1.f / (dx * h0);
    C.sat_z = 1.f / (dz * h0);
    C.nsat_x = 1.f / (dx * dx * h0);
    C.nsat_z = 1.f / (dz * dz * h0);
    C.bc[0] = p.bc_top;
    C.bc[1] = p.bc_bottom;
    C.bc[2] = p.bc_left;
    C.bc[3] = p.bc_right;
    C.sub = 1;
    C.snap_prec = FWI2D_SNAP_FP32;
    C.spin = 1 << 20;

    const ShotDev *shots = (const ShotDev *)(S + o_shot);
    launch_init_state(shots, 1, (const InitCell *)(S + o_cells), (const int *)(S + o_ioff), (const int *)(S + o_idx),
                      st);
    for (int it = 0; it < nt - 1; it++)
        launch_elastic_step(shape, false, shots, (const TileRef *)(S + o_tiles), ntiles, md, C, it, STEP_EXTRACT,
                            p.dt, st);
    launch_finalize(shots, 1, C, 2, STEP_EXTRACT, st);
    NA_CK(cudaGetLastError());

    // receivers: accumulate into the caller's blocks (stride nr*nt per component)
    for (int c = 0; c < 2; c++)
        NA_CK(cudaMemcpyAsync(S + o_rcv_raw + (size_t)c * ext->ntr * nt * sizeof(float), allrcv + (size_t)c * nr * nt,
                              (size_t)ext->ntr * nt * sizeof(float), cudaMemcpyHostToDevice, st));
    k_add_from_time_major<<<296, 256, 0, st>>>((const float *)(S + o_rcv), (float *)(S + o_rcv_raw), nrcv, nt);
    NA_CK(cudaGetLastError());
    for (int c = 0; c < 2; c++)
        NA_CK(cudaMemcpyAsync(allrcv + (size_t)c * nr * nt, S + o_rcv_raw + (size_t)c * ext->ntr * nt * sizeof(float),
                              (size_t)ext->ntr * nt * sizeof(float), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    return FWI2D_OK;
}
