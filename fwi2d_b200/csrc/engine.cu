// Host engine and C ABI of fwi2d_b200.
//
// A context owns one device stream, one model and one batch plan.  The plan
// holds every per-shot device buffer (two field buffers, time-major traces,
// injection / extraction tables, boundary and taper tables, snapshots and the
// gradient accumulator) and two CUDA graphs: the forward time loop and the
// adjoint time loop, each a chain of one fused kernel per time step.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.h"
#include "host_tables.h"
#include "launch.h"
#include "resample.cuh"
#include "../../include/fwi2d_b200.h"

namespace fwi2d {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                                              \
    do {                                                                                                   \
        cudaError_t e_ = (x);                                                                              \
        if (e_ != cudaSuccess) {                                                                           \
            (void)cudaGetLastError();                                                                      \
            throw Error(e_ == cudaErrorMemoryAllocation ? FWI2D_ERR_OOM : FWI2D_ERR_CUDA,                  \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                                  \
        }                                                                                                  \
    } while (0)
#define REQ(c, msg)                                      \
    do {                                                 \
        if (!(c)) throw Error(FWI2D_ERR_ARG, (msg));     \
    } while (0)

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t bytes)
    {
        release();
        if (bytes) {
            CK(cudaMalloc(&p, bytes));
            n = bytes;
        }
    }
    template <class T> T *as() const { return (T *)p; }
    // (re)allocates only when the size changes, so device pointers captured
    // in a CUDA graph stay valid across same-size updates
    void ensure(size_t bytes)
    {
        if (bytes != n || !p) alloc(bytes);
    }
    template <class T> void upload(const std::vector<T> &v, cudaStream_t st)
    {
        ensure(std::max<size_t>(v.size(), 1) * sizeof(T));
        if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    }
};

static int round_up(int a, int b) { return (a + b - 1) / b * b; }

// ---------------------------------------------------------------------------
// layout kernels
// ---------------------------------------------------------------------------
__global__ void k_to_time_major(const float *__restrict__ in, float *__restrict__ out, int rows, int nt)
{
    __shared__ float t[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        int r = r0 + j, c = c0 + threadIdx.x;
        if (r < rows && c < nt) t[j][threadIdx.x] = in[(long long)r * nt + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        int c = c0 + j, r = r0 + threadIdx.x;
        if (r < rows && c < nt) out[(long long)c * rows + r] = t[threadIdx.x][j];
    }
}
__global__ void k_from_time_major(const float *__restrict__ in, float *__restrict__ out, int rows, int nt)
{
    __shared__ float t[32][33];
    const int c0 = blockIdx.y * 32, r0 = blockIdx.x * 32;   // in is [nt][rows]
    for (int j = threadIdx.y; j < 32; j += 8) {
        int c = c0 + j, r = r0 + threadIdx.x;
        if (r < rows && c < nt) t[j][threadIdx.x] = in[(long long)c * rows + r];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        int r = r0 + j, c = c0 + threadIdx.x;
        if (r < rows && c < nt) out[(long long)r * nt + c] = t[threadIdx.x][j];
    }
}
__global__ void k_add_subgrid(float *__restrict__ full, const float *__restrict__ part, int ncomp, int x0, int nx,
                              int ldz, long long full_comp)
{
    const long long n = (long long)ncomp * nx * ldz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long c = i / ((long long)nx * ldz);
        const long long r = i - c * nx * ldz;
        full[c * full_comp + (long long)x0 * ldz + r] += part[i];
    }
}
__global__ void k_pitch(const float *__restrict__ in, float *__restrict__ out, long long rows, int nz, int ldz)
{
    const long long n = rows * ldz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / ldz;
        const int z = (int)(i - r * ldz);
        out[i] = z < nz ? in[r * nz + z] : 0.f;
    }
}
__global__ void k_unpitch(const float *__restrict__ in, float *__restrict__ out, long long rows, int nz, int ldz)
{
    const long long n = rows * nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / nz;
        const int z = (int)(i - r * nz);
        out[i] = in[r * ldz + z];
    }
}

// Compensated (two-level) gradient accumulation.  The step kernels add each
// time sample's imaging term into the FP32 accumulator `grad` in the
// reference's order, so that `grad` holds the sum over the last few adjoint
// steps only; every kCompWindow steps this kernel adds it into a running sum
// held as an unevaluated pair (hi, lo) with Neumaier's compensated summation
// (hi + lo carries the sum to about twice the FP32 precision) and clears it.
// final: the last partial window is added and `grad` receives hi + lo.
static const int kCompWindow = 8;
__global__ void k_grad_flush(const ShotDev *__restrict__ shots, int ncompg, int final)
{
    const ShotDev &S = shots[blockIdx.y];
    const long long n = (long long)ncompg * S.nx * S.ldz;
    float *__restrict__ g = S.grad;
    float *__restrict__ hi = S.gcomp;
    float *__restrict__ lo = S.gcomp + n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float w = g[i], h = hi[i];
        const float t = h + w;
        const float c = lo[i] + (fabsf(h) >= fabsf(w) ? (h - t) + w : (w - t) + h);
        if (final) {
            g[i] = t + c;
        } else {
            hi[i] = t;
            lo[i] = c;
            g[i] = 0.f;
        }
    }
}

void launch_to_time_major(const float *in, float *out, int rows, int nt, cudaStream_t st)
{
    dim3 g((nt + 31) / 32, (rows + 31) / 32), b(32, 8);
    k_to_time_major<<<g, b, 0, st>>>(in, out, rows, nt);
}
void launch_from_time_major(const float *in, float *out, int rows, int nt, cudaStream_t st)
{
    dim3 g((rows + 31) / 32, (nt + 31) / 32), b(32, 8);
    k_from_time_major<<<g, b, 0, st>>>(in, out, rows, nt);
}
void launch_add_subgrid(float *full, const float *part, int ncomp, int x0, int nx, int ldz, long long full_comp,
                        cudaStream_t st)
{
    k_add_subgrid<<<592, 256, 0, st>>>(full, part, ncomp, x0, nx, ldz, full_comp);
}

// ---------------------------------------------------------------------------
// model
// ---------------------------------------------------------------------------
struct ModelState {
    int kind = -1, nx = 0, nz = 0, ldz = 0, npar = 0;
    float dx = 0, dz = 0;
    std::vector<float> host;   // converted model as given, [npar][nx][nz]
    DevBuf p0, p1, p2, c13, eps, fxx, lbis, gv2, gv3;
    DevBuf stage;              // unpitched upload staging, [nx][nz]
    ModelDev dev() const
    {
        ModelDev m;
        m.nx = nx;
        m.nz = nz;
        m.ldz = ldz;
        m.p0 = p0.as<float>();
        m.p1 = p1.as<float>();
        m.p2 = p2.as<float>();
        m.c13 = c13.as<float>();
        m.eps = eps.as<float>();
        m.fxx = fxx.as<float>();
        m.lbis = lbis.as<float>();
        m.gv2 = gv2.as<float>();
        m.gv3 = gv3.as<float>();
        return m;
    }
    const float *hp(int i) const { return host.data() + (size_t)i * nx * nz; }
};

static int npar_of(int kind)
{
    switch (kind) {
    case KIND_ELASTIC: return 3;
    case KIND_VTI: return 5;
    case KIND_ACOUSTIC: return 2;
    case KIND_AE: return 3;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
struct ShotPlan {
    int x0 = 0, nx = 0, nt = 0;
    int ncomp = 2;                 // field components
    int ncomp_src = 2, ntr_src = 0, nr = 0;
    int nsrc_rows = 0, nrcv_rows = 0;
    int nslot = 0;                 // snapshot time slots of the shot (1 + nt/sub)
    int nbuf = 0;                  // slots held on the device (nslot, or the replay window)
    size_t snap_need = 0;          // bytes of its snapshot store
    int u_t0 = 0, u_m0 = 0, u_b0 = 0, u_i0 = 0;   // first tile / marching / band / interior unit in the plan
    int u_w0 = 0;                                 // acoustic-elastic: first fluid-layer tile in the plan
    void *snap_base = nullptr;     // its snapshot store: `snap`, or its place in the plan's wave pool
    std::vector<InjEntry> inj_f, inj_a;
    std::vector<int> inj_f_off, inj_a_off, inj_f_roff, inj_a_roff;
    std::vector<ExtEntry> ext_f;
    std::vector<int> ext_f_off, ext_none_off, ext_f_roff;
    std::vector<MarchRow> mrow_f, mrow_a;
    DevBuf u0, u1, src_f, rcv_f, src_a;
    DevBuf d_inj_f, d_inj_f_off, d_inj_a, d_inj_a_off, d_ext_f, d_ext_f_off, d_ext_none_off;
    DevBuf d_mrow_f, d_mrow_a;
    DevBuf den, tz, tx, snap, amax, grad, gwt;
    DevBuf gcomp;                  // compensated accumulation: running sum pair (hi, lo) of the gradient
    DevBuf r0, r1, ckpt;           // checkpoint-and-recompute: replay fields and checkpoints
    DevBuf halo;                   // acoustic-elastic: prev of the interface row [nx]
    std::unique_ptr<ShotPlan> fluid;   // acoustic-elastic: the fluid layer's grid (nx x nza)
};

struct Plan {
    fwi2d_params par;
    int kind = 0;
    int shape = 0;                 // index into the shape list (tile shapes, then marching shapes)
    int tshape = 0, TZ = 32, TX = 16;   // tile shape of the tile kernel's units
    bool march = false;            // interior rows on the marching kernel
    bool framed = false;           // interior on the tile kernel's interior path, frame on the band kernels
    bool band_split = false;       // frame on the band kernels that split a cell's components over two warps
    int ishape = 0;                // framed: tile shape of the interior tiles
    int nth = 0, lx = 0;           // marching: threads (z window) per unit, rows per unit
    int nt_max = 0;
    int ncompg = 3;
    std::vector<std::unique_ptr<ShotPlan>> shots;
    std::vector<TileRef> tiles;
    std::vector<MarchRef> marches;
    std::vector<BandRef> bands;
    std::vector<TileRef> itiles;   // framed: interior tiles
    DevBuf d_tiles, d_march, d_bands, d_itiles, d_shots_f, d_shots_a;
    // Waves: contiguous runs of shots whose snapshots fit the device together.
    // A plan whose snapshots all fit has one wave.  Each wave has its own
    // forward-with-snapshots and adjoint graphs over its shots' units; the
    // waves share one snapshot pool (snap_pool), so a gradient runs wave by
    // wave.  `all` spans every shot and unit (forward without snapshots,
    // autotuning).
    struct Wave {
        int s0 = 0, s1 = 0, nt_max = 0;
        int t0 = 0, t1 = 0, m0 = 0, m1 = 0, b0 = 0, b1 = 0, i0 = 0, i1 = 0;   // unit ranges
        int w0 = 0, w1 = 0;                                                   // fluid-layer tiles
        cudaGraphExec_t graph[2] = {nullptr, nullptr};                        // forward + snapshots, adjoint
        cudaEvent_t ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
        long long launches[2] = {0, 0};
    };
    std::vector<Wave> waves;
    Wave all;
    DevBuf snap_pool;
    bool fwd_waves = false;        // the last forward timing is the sum over the waves' events
    // checkpoint-and-recompute: every `ckpt` steps; cuts[k] is the first
    // imaging time of segment k (cuts.back() = nt - 1); per-segment shot
    // tables of the replay (forward with snapshot store) and of the adjoint
    int ckpt = 0;
    std::vector<int> cuts;
    DevBuf d_shots_r, d_shots_c;
    // acoustic-elastic: fluid layer of nza rows (pitch ldzw) with the constant
    // model (K, 1/rho) of the water, its tiles, shot tables and step constants
    bool ae = false, ae_src_fluid = false;
    int nza = 0, ldzw = 0, nx_max = 0;
    float Kw = 0.f, val0 = 0.f;
    StepConst Cw;
    DevBuf wK, wIR;
    std::vector<TileRef> wtiles;
    DevBuf d_wtiles, d_wshots_f, d_wshots_a;
    std::vector<InitCell> wicells[2];
    std::vector<int> wioff[2], wiidx[2];
    DevBuf d_wicells[2], d_wioff[2], d_wiidx[2];
    ModelDev wdev() const
    {
        ModelDev m;
        std::memset(&m, 0, sizeof(m));
        m.nz = nza;
        m.ldz = ldzw;
        m.p0 = wK.as<float>();
        m.p1 = wIR.as<float>();
        return m;
    }
    // initial-state cells per mode (0 forward, 1 adjoint)
    std::vector<InitCell> icells[2];
    std::vector<int> ioff[2], iidx[2];
    DevBuf d_icells[2], d_ioff[2], d_iidx[2];
    // FWI gradient: observed data, misfit partial sums
    DevBuf d_obs, d_misfit, d_part;
    // data time axis of fwi2d_fwi_gradient (fwi2d_set_data_axis): dd > 0 when
    // sources and data are sampled at dd and resampled to dt; nd per shot;
    // d_rs0 / d_rs1 hold one shot's trace block in the trace pipeline
    float dd = 0.f;
    int rs_linear = 0, rs_hl = 11;
    std::vector<int> nd;
    DevBuf d_rs0, d_rs1;
    DevBuf d_grad_full, d_stage;
    StepConst C;
    float dtg = 0;
    bool have_snapshots = false;
    bool snapshots_valid = false;
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};   // forward, forward+store, adjoint
    cudaEvent_t ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [forward|adjoint][start|end]
    bool timed[2] = {false, false};
    long long launches[3] = {0, 0, 0};
    long long snap_bytes = 0;
    // device status word of the bounded waits (launch_take_timeout after each
    // pass) and its pinned host copy, read after the pass has finished
    DevBuf d_status;
    int *h_status = nullptr;
    ~Plan()
    {
        if (h_status) cudaFreeHost(h_status);
        for (auto &w : waves) {
            for (auto &g : w.graph)
                if (g) cudaGraphExecDestroy(g);
            for (auto &a : w.ev)
                for (auto &e : a)
                    if (e) cudaEventDestroy(e);
        }
        for (auto &g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto &a : ev)
            for (auto &e : a)
                if (e) cudaEventDestroy(e);
    }
};

}  // namespace fwi2d

struct fwi2d_ctx {
    int device = 0;
    cudaStream_t st = nullptr;      // stream all work is ordered on
    cudaStream_t own = nullptr;     // the context's own stream
    cudaStream_t side = nullptr;    // boundary-band kernels run here and on side2, overlapping the core kernel
    cudaStream_t side2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr;
    fwi2d::ModelState M;
    std::unique_ptr<fwi2d::Plan> plan;
};

namespace fwi2d {

static void set_device(fwi2d_ctx *ctx) { CK(cudaSetDevice(ctx->device)); }

// ---- model upload -----------------------------------------------------------
static void upload_model_values(fwi2d_ctx *ctx, const float *model);

static void set_model(fwi2d_ctx *ctx, int kind, int nx, int nz, float dx, float dz, const float *model)
{
    REQ(kind >= 0 && kind <= 3, "unknown propagator kind");
    REQ(nx >= 12 && nz >= 12, "the model must have at least 12 samples along each axis");
    REQ(dx > 0 && dz > 0, "grid spacings must be positive");
    REQ(model != nullptr, "null model");
    set_device(ctx);
    ModelState &M = ctx->M;
    ctx->plan.reset();
    M.kind = kind;
    M.nx = nx;
    M.nz = nz;
    M.ldz = round_up(nz, 32);
    M.dx = dx;
    M.dz = dz;
    M.npar = npar_of(kind);
    upload_model_values(ctx, model);
}

// New values for the current model geometry (device arrays, host copy).
static void upload_model_values(fwi2d_ctx *ctx, const float *model)
{
    ModelState &M = ctx->M;
    const int kind = M.kind, nx = M.nx, nz = M.nz;
    const size_t nxz = (size_t)nx * nz;
    M.host.assign(model, model + nxz * M.npar);
    for (size_t i = 0; i < M.host.size(); i++) REQ(std::isfinite(M.host[i]), "model holds a non-finite value");
    const size_t pitched = (size_t)nx * M.ldz;
    M.stage.ensure(nxz * sizeof(float));
    // every upload goes through the one staging buffer, in stream order; the
    // sources stay valid until the synchronisation at the end
    auto up = [&](DevBuf &dst, const float *src) {
        dst.ensure(pitched * sizeof(float));
        CK(cudaMemcpyAsync(M.stage.p, src, nxz * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
        k_pitch<<<592, 256, 0, ctx->st>>>(M.stage.as<float>(), dst.as<float>(), nx, nz, M.ldz);
        CK(cudaGetLastError());
    };
    // device copies straight from the caller's array (which may be pinned)
    up(M.p0, model);
    up(M.p1, model + nxz);
    if (kind != KIND_ACOUSTIC) up(M.p2, model + 2 * nxz);
    else M.p2.release();
    M.c13.release();
    M.eps.release();
    M.fxx.release();
    M.lbis.release();
    M.gv2.release();
    M.gv3.release();
    if (kind == KIND_VTI) {
        const float *lam = M.hp(0), *mu = M.hp(1), *c13 = M.hp(3), *eps = M.hp(4);
        std::vector<float> fxx(nxz), lbis(nxz), v2(nxz), v3(nxz);
        for (size_t i = 0; i < nxz; i++) {
            fxx[i] = (1 + 2 * eps[i]) * 2 * mu[i];           // vtiexpr7b, we_op.cpp:1473
            lbis[i] = (1 + 2 * eps[i]) * lam[i];             // mod_bis, we_op.cpp:1590
            const float l = lam[i], m = mu[i], c = c13[i];   // we_op.cpp:1499-1504
            const float del = ((c + m) * (c + m) - (l + m) * (l + m)) / (2 * (l + m) * (l + 2 * m));
            const float val1 = std::sqrt(2 * (l + 2 * m) * (l + m) * del + (l + m) * (l + m));
            v2[i] = ((1 + 2 * del) * l + (1 + 3 * del) * m) / val1;
            v3[i] = ((1 + 3 * del) * l + (1 + 4 * del) * m) / val1 - 1;
        }
        up(M.c13, c13);
        up(M.eps, eps);
        up(M.fxx, fxx.data());
        up(M.lbis, lbis.data());
        up(M.gv2, v2.data());
        up(M.gv3, v3.data());
    }
    CK(cudaStreamSynchronize(ctx->st));
}

// ---- plan construction -------------------------------------------------------
static int owner_tile(int g, int n, int T)
{
    if (g >= n - T) return (n + T - 1) / T - 1;
    return g / T;
}

static void check_injector(const fwi2d_injector &J, int nx, int nz, const char *what)
{
    if (J.ntr == 0) return;
    REQ(J.ntr > 0 && J.xind && J.zind && J.xw && J.zw, std::string(what) + ": incomplete injector tables");
    REQ(J.type == FWI2D_INJ_DELTA || J.type == FWI2D_INJ_DDELTA, std::string(what) + ": unknown injector type");
    for (int t = 0; t < J.ntr; t++)
        for (int k = 0; k < 3; k++) {
            REQ(J.xind[t * 3 + k] >= 0 && J.xind[t * 3 + k] < nx, std::string(what) + ": x index outside the shot grid");
            REQ(J.zind[t * 3 + k] >= 0 && J.zind[t * 3 + k] < nz, std::string(what) + ": z index outside the shot grid");
        }
}

// ---- work decomposition ---------------------------------------------------------
// A plan runs either the tile kernel over the whole of every shot grid, or the
// marching kernel over the cells clear of the four boundary bands
// (6 <= x < nx-6, 6 <= z < nz-6), the tile kernel (full-height tiles of
// kBandTile) on the x bands and the band kernel on the top and bottom bands.
struct MarchShape {
    int nth, lx;
};
static const MarchShape kMarchShapes[] = {{224, 64}, {256, 64}, {192, 64}, {128, 64},
                                          {224, 32}, {256, 32}, {192, 32}, {128, 32},
                                          {128, 16}, {224, 16}};
static const int kNumMarch = sizeof(kMarchShapes) / sizeof(kMarchShapes[0]);
static const int kBandTile = 3;    // (TZ, TX) = (32, 8): band windows of 8 columns own 6
static const int kBand = 6;
// Framed tile plans: the tile kernel's interior path on windows of one of
// these tile shapes over the cells clear of all four boundary bands, and the
// band kernels of the marching plans on the frame.  Shape indices follow the
// marching shapes.
static const int kFramedShapes[] = {3, 2, 1, 0};
static const int kNumFramed = sizeof(kFramedShapes) / sizeof(kFramedShapes[0]);

// The band kernels of framed and marching plans come in two forms: one
// thread per cell, or the two field components of a cell in two warps
// (split), which halves the serial closure chain of a thread.  The frame's
// few CTAs set the time of a step when the plan has few band windows (one
// 401 x 801 shot on B200, same interior shape: forward 17 % and adjoint 4 %
// faster);
// with many, the split kernels' larger CTAs take registers from the interior
// kernel on their SMs (eight such shots: 3-6 % slower per gradient).  So the
// split form is taken up to kSplitMaxBandWindows x-band windows (32 rows of
// one side of one shot each); FWI2D_BAND_SPLIT=0 or 1 forces either form.
static const int kSplitMaxBandWindows = 32;
static bool band_split_for(int nshots, int nz)
{
    const char *e = std::getenv("FWI2D_BAND_SPLIT");
    if (e && *e) return std::atoi(e) != 0;
    return (long long)nshots * 2 * ((nz + 31) / 32) <= kSplitMaxBandWindows;
}

static int shape_count() { return elastic_tile_count() + kNumMarch + kNumFramed; }
static bool is_march_shape(int s) { return s >= elastic_tile_count() && s < elastic_tile_count() + kNumMarch; }
static bool is_framed_shape(int s) { return s >= elastic_tile_count() + kNumMarch && s < shape_count(); }
static int framed_tile_shape(int s) { return kFramedShapes[s - elastic_tile_count() - kNumMarch]; }

// Work units of one shot.  Units are numbered per shot: tiles first, then
// marching units (segment-major, then z window).
struct ShotUnits {
    bool march = false;            // marching plan: x-band tiles, bands, marching units
    bool framed = false;           // framed tile plan: x-band tiles, bands, interior tiles
    int nx = 0, nz = 0;
    int TX = 0, TZ = 0, tiles_x = 0, tiles_z = 0;
    int lx = 0, nseg = 0, nwin = 0;
    int ITX = 0, ITZ = 0, itiles_x = 0;   // framed: interior tile shape and tiles along x
    int zrows = 64;                        // rows per top / bottom band unit (zband_rows)
    int itiles_z = 0, izlast = 0;          // framed: tiles along z, first row of the last (interior coordinates)
    std::vector<int> zo;           // marching: owned z starts of the core windows, plus nz - 6
    std::vector<TileRef> tiles;    // marching and framed plans: the x-band tiles
    std::vector<BandRef> bands;    // top / bottom band units (two per run of rows)
    std::vector<MarchRef> marches;
    std::vector<TileRef> itiles;   // framed: tiles of the interior [6, nx-6) x [6, nz-6)
    int nunits() const { return (int)(tiles.size() + bands.size() + marches.size() + itiles.size()); }
    int unit_of(int x, int z) const
    {
        if (!march && !framed) return owner_tile(z, nz, TZ) * tiles_x + owner_tile(x, nx, TX);
        if (x < kBand) return owner_tile(z, nz, TZ);
        if (x >= nx - kBand) return tiles_z + owner_tile(z, nz, TZ);
        const int nt = (int)tiles.size();
        if (z < kBand || z >= nz - kBand) return nt + 2 * ((x - kBand) / zrows) + (z < kBand ? 0 : 1);
        if (framed) {
            const int zi = z - kBand;
            const int kz = zi >= izlast ? itiles_z - 1 : zi / ITZ;
            return nt + (int)bands.size() + kz * itiles_x + owner_tile(x - kBand, nx - 2 * kBand, ITX);
        }
        const int seg = (x - kBand) / lx;
        const int k = (int)(std::upper_bound(zo.begin(), zo.end(), z) - zo.begin()) - 1;
        return nt + (int)bands.size() + seg * nwin + k;
    }
    // units whose entries are sorted by row and indexed by per-row records
    // (band and marching units)
    bool row_sorted(int u) const
    {
        return u >= (int)tiles.size() && u < (int)(tiles.size() + bands.size() + marches.size());
    }
    struct RowUnit {
        int unit, xb, xe, roff;
    };
    std::vector<RowUnit> row_units() const
    {
        std::vector<RowUnit> r;
        for (const BandRef &b : bands) r.push_back({b.unit, b.xb, b.xe, b.roff});
        for (const MarchRef &m : marches) r.push_back({m.unit, m.xb, m.xe, m.roff});
        return r;
    }
};

static bool axis_fits(int T, int n) { return n == T || n >= T + 8; }

// Core z windows of the marching kernel for nth threads: window k owns
// [zo[k], zo[k+1]) within [6, nz-6) and covers [za, za + nth), two cells
// beyond its owned range on each side (the last one flush with nz-4, or
// starting at 4 when one window covers the whole core), so every cell it
// evaluates lies in [4, nz-4) where the stencils take their interior form.
static void march_windows(int nz, int nth, std::vector<int> &zo, std::vector<int> &za)
{
    const int w = nth - 4, lo = kBand, hi = nz - kBand;
    const int K = (hi - lo + w - 1) / w;
    zo.assign(K + 1, 0);
    for (int k = 0; k < K; k++) zo[k] = lo + k * w;
    zo[K] = hi;
    za.assign(K, 0);
    for (int k = 0; k < K; k++) za[k] = zo[k] - 2;
    if (K > 1) za[K - 1] = std::max(lo - 2, std::min(zo[K - 1] - 2, hi + 2 - nth));
}

// Whether a shape can run a shot grid of nx x nz.
static bool shape_fits(int shape, int nx, int nz)
{
    if (shape < 0 || shape >= shape_count()) return false;
    int tz, tx;
    if (shape < elastic_tile_count()) {
        elastic_tile_shape(shape, &tz, &tx);
        return axis_fits(tz, nz) && axis_fits(tx, nx);
    }
    elastic_tile_shape(kBandTile, &tz, &tx);
    const bool frame = axis_fits(tz, nz) && nx >= 2 * tx && nx > 2 * kBand && nz >= 40;
    if (is_framed_shape(shape)) {
        int itz, itx;
        elastic_tile_shape(framed_tile_shape(shape), &itz, &itx);
        return frame && axis_fits(itz, nz - 2 * kBand) && axis_fits(itx, nx - 2 * kBand);
    }
    return frame && march_threads_ok(kMarchShapes[shape - elastic_tile_count()].nth);
}

static ShotUnits make_units(int shape, int shot, int nx, int nz, bool band_split)
{
    ShotUnits U;
    U.nx = nx;
    U.nz = nz;
    U.zrows = zband_rows(band_split);
    const bool framed = is_framed_shape(shape);
    const bool march = is_march_shape(shape);
    U.march = march;
    U.framed = framed;
    elastic_tile_shape(march || framed ? kBandTile : shape, &U.TZ, &U.TX);
    U.tiles_z = (nz + U.TZ - 1) / U.TZ;
    if (!march && !framed) {
        U.tiles_x = (nx + U.TX - 1) / U.TX;
        for (int tzi = 0; tzi < U.tiles_z; tzi++)
            for (int txi = 0; txi < U.tiles_x; txi++) {
                TileRef r;
                r.shot = shot;
                r.unit = (int)U.tiles.size();
                tile_window_host(txi, U.tiles_x, nx, U.TX, r.wx0, r.ox0, r.ox1);
                tile_window_host(tzi, U.tiles_z, nz, U.TZ, r.wz0, r.oz0, r.oz1);
                U.tiles.push_back(r);
            }
        return U;
    }
    for (int side = 0; side < 2; side++)
        for (int tzi = 0; tzi < U.tiles_z; tzi++) {
            TileRef r;
            r.shot = shot;
            r.unit = (int)U.tiles.size();
            r.wx0 = side == 0 ? 0 : nx - U.TX;
            r.ox0 = side == 0 ? 0 : nx - kBand;
            r.ox1 = side == 0 ? kBand : nx;
            tile_window_host(tzi, U.tiles_z, nz, U.TZ, r.wz0, r.oz0, r.oz1);
            U.tiles.push_back(r);
        }
    int roff = 0;
    for (int a = kBand; a < nx - kBand; a += U.zrows)
        for (int side = 0; side < 2; side++) {
            BandRef b;
            b.shot = shot;
            b.unit = (int)(U.tiles.size() + U.bands.size());
            b.xb = a;
            b.xe = std::min(a + U.zrows, nx - kBand);
            b.side = side;
            b.roff = roff;
            roff += b.xe - b.xb + 1;
            U.bands.push_back(b);
        }
    if (framed) {
        // interior windows, tiled as the tile plans tile a whole grid, offset by
        // the band; along z every window starts on an even row (the kernel's
        // z-pairs), so the last one may reach one row into the bottom band,
        // which it does not own: its owned cells' stencils stay interior and
        // its halo inside the grid
        elastic_tile_shape(framed_tile_shape(shape), &U.ITZ, &U.ITX);
        const int ni_x = nx - 2 * kBand, ni_z = nz - 2 * kBand;
        U.itiles_x = (ni_x + U.ITX - 1) / U.ITX;
        const int itiles_z = (ni_z + U.ITZ - 1) / U.ITZ;
        const int T = U.ITZ;
        auto zw = [&](int i) {
            const int v = i * T < ni_z - T ? i * T : ni_z - T;
            return v + (v & 1);
        };
        U.itiles_z = itiles_z;
        U.izlast = zw(itiles_z - 1);
        for (int tzi = 0; tzi < itiles_z; tzi++)
            for (int txi = 0; txi < U.itiles_x; txi++) {
                TileRef r;
                r.shot = shot;
                r.unit = (int)(U.tiles.size() + U.bands.size() + U.itiles.size());
                tile_window_host(txi, U.itiles_x, ni_x, U.ITX, r.wx0, r.ox0, r.ox1);
                r.wz0 = zw(tzi);
                r.oz0 = tzi == 0 ? 0 : zw(tzi);
                r.oz1 = tzi == itiles_z - 1 ? ni_z : zw(tzi + 1);
                r.wx0 += kBand;
                r.ox0 += kBand;
                r.ox1 += kBand;
                r.wz0 += kBand;
                r.oz0 += kBand;
                r.oz1 += kBand;
                U.itiles.push_back(r);
            }
        return U;
    }
    const MarchShape ms = kMarchShapes[shape - elastic_tile_count()];
    std::vector<int> za;
    march_windows(nz, ms.nth, U.zo, za);
    U.nwin = (int)za.size();
    U.lx = ms.lx;
    const int rows = nx - 2 * kBand;
    U.nseg = (rows + U.lx - 1) / U.lx;
    for (int sg = 0; sg < U.nseg; sg++)
        for (int k = 0; k < U.nwin; k++) {
            MarchRef m;
            m.shot = shot;
            m.unit = (int)(U.tiles.size() + U.bands.size() + U.marches.size());
            m.xb = kBand + sg * U.lx;
            m.xe = std::min(m.xb + U.lx, nx - kBand);
            m.za = za[k];
            m.oz0 = U.zo[k];
            m.oz1 = U.zo[k + 1];
            m.roff = roff;
            roff += m.xe - m.xb + 1;
            U.marches.push_back(m);
        }
    return U;
}

// Group entries by unit (stable: the reference's order survives within a
// cell); within a marching unit order them by row (then z for injection).
// off: [units+1] offsets; roff: per marching unit and row, the first entry of
// the row (absolute), plus the end.
template <class E>
static void group_entries(const ShotUnits &U, const std::vector<E> &ent, const std::vector<int> &unit,
                          const std::vector<int> &row, const std::vector<int> &zkey, std::vector<E> &out,
                          std::vector<int> &off, std::vector<int> &roff)
{
    const int nu = U.nunits();
    std::vector<size_t> idx(ent.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
        if (unit[a] != unit[b]) return unit[a] < unit[b];
        if (!U.row_sorted(unit[a])) return false;
        if (row[a] != row[b]) return row[a] < row[b];
        return zkey[a] < zkey[b];
    });
    out.clear();
    off.assign(nu + 1, 0);
    for (size_t i : idx) {
        out.push_back(ent[i]);
        off[unit[i] + 1]++;
    }
    for (int t = 0; t < nu; t++) off[t + 1] += off[t];
    const std::vector<ShotUnits::RowUnit> rus = U.row_units();
    int nro = 0;
    for (const auto &m : rus) nro += m.xe - m.xb + 1;
    roff.assign(std::max(nro, 1), 0);
    for (const auto &m : rus) {
        int e = off[m.unit];
        for (int r = m.xb; r <= m.xe; r++) {
            while (e < off[m.unit + 1] && row[idx[e]] < r) e++;
            roff[m.roff + r - m.xb] = e;
        }
    }
}

// Injection entries of one injector into a field, in the reference's order
// (component, trace, x, z), grouped by owning unit.
static void build_inj(const fwi2d_injector &J, int ncomp, const int *rowbase_a, const int *rowbase_b,
                      const ShotUnits &U, std::vector<InjEntry> &out, std::vector<int> &off, std::vector<int> &roff)
{
    std::vector<InjEntry> ent;
    const int w = J.type == FWI2D_INJ_DELTA ? 3 : 6;
    for (int c = 0; c < ncomp; c++)
        for (int t = 0; t < J.ntr; t++) {
            const float *xi = J.xw + (size_t)t * 2 * w, *zi = J.zw + (size_t)t * 2 * w;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    InjEntry e;
                    e.gx = J.xind[t * 3 + a];
                    e.gz = J.zind[t * 3 + b];
                    e.comp = c;
                    if (J.type == FWI2D_INJ_DELTA) {
                        e.mt = 0;
                        e.ia = rowbase_a[c] + t;
                        e.ib = 0;
                        e.wa = xi[a] * zi[b];
                        e.wb = 0.f;
                    } else {
                        e.mt = 1;
                        e.ia = rowbase_a[c] + t;
                        e.ib = rowbase_b[c] + t;
                        e.wa = -xi[a + 3] * zi[b];
                        e.wb = xi[a] * zi[b + 3];
                    }
                    ent.push_back(e);
                }
        }
    std::vector<int> unit(ent.size()), row(ent.size()), zk(ent.size());
    for (size_t i = 0; i < ent.size(); i++) {
        unit[i] = U.unit_of(ent[i].gx, ent[i].gz);
        row[i] = ent[i].gx;
        zk[i] = ent[i].gz;
    }
    group_entries(U, ent, unit, row, zk, out, off, roff);
}

// Receiver entries, owned by the unit of the pivot cell (the middle of the 3x3).
static void build_ext(const fwi2d_injector &J, int ncomp, const ShotUnits &U, std::vector<ExtEntry> &out,
                      std::vector<int> &off, std::vector<int> &roff, int row0 = 0)
{
    std::vector<ExtEntry> ent;
    std::vector<int> unit, row, zk;
    for (int c = 0; c < ncomp; c++)
        for (int t = 0; t < J.ntr; t++) {
            ExtEntry e;
            e.row = row0 + c * J.ntr + t;
            e.comp = c;
            e.gx0 = J.xind[t * 3];
            e.gz0 = J.zind[t * 3];
            const float *xe = J.xw + (size_t)t * 6 + 3, *ze = J.zw + (size_t)t * 6 + 3;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) e.w[a * 3 + b] = xe[a] * ze[b];
            ent.push_back(e);
            unit.push_back(U.unit_of(J.xind[t * 3 + 1], J.zind[t * 3 + 1]));
            row.push_back(J.xind[t * 3 + 1]);
            zk.push_back(J.zind[t * 3 + 1]);
        }
    group_entries(U, ent, unit, row, zk, out, off, roff);
}

// Row records of the marching units from the per-row entry offsets.
static void build_march_rows(const ShotUnits &U, const std::vector<InjEntry> &inj, const std::vector<int> &iroff,
                             const std::vector<int> *eroff, const std::vector<float> &tx, std::vector<MarchRow> &out)
{
    out.clear();
    for (const auto &m : U.row_units())
        for (int r = m.xb; r <= m.xe; r++) {   // one spare record per unit keeps the roff layout
            MarchRow R;
            std::memset(&R, 0, sizeof(R));
            const int k = m.roff + r - m.xb;
            if (r == m.xe) {
                out.push_back(R);
                continue;
            }
            R.e0 = iroff[k];
            R.e1 = iroff[k + 1];
            R.zlo = R.e1 > R.e0 ? inj[R.e0].gz : 0;
            R.zhi = R.e1 > R.e0 ? inj[R.e1 - 1].gz : -1;
            R.r0 = eroff ? (*eroff)[k] : 0;
            R.r1 = eroff ? (*eroff)[k + 1] : 0;
            R.tx = tx[r];
            out.push_back(R);
        }
    if (out.empty()) out.resize(1);
}

static StepConst make_const(const fwi2d_params &p, float dx, float dz)
{
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
    C.alpha = (float)(0.2508560249 / p.free_surface_stiffness);
    C.bc[0] = p.bc_top;
    C.bc[1] = p.bc_bottom;
    C.bc[2] = p.bc_left;
    C.bc[3] = p.bc_right;
    C.sub = p.sub > 0 ? p.sub : 1;
    C.snap_prec = p.snapshot_precision;
    // poll limit of the marching kernel's bounded waits: FWI2D_SPIN_LIMIT
    // (read when a plan is built) or 2^20 polls
    C.spin = 1 << 20;
    if (const char *e = std::getenv("FWI2D_SPIN_LIMIT")) {
        const long v = std::strtol(e, nullptr, 10);
        if (v >= 0 && v <= (1L << 30)) C.spin = (int)v;
    }
    return C;
}

static void shot_dev(const Plan &P, const ShotPlan &s, const ModelState &M, bool adjoint, ShotDev &d)
{
    std::memset(&d, 0, sizeof(d));
    d.nx = s.nx;
    d.nz = M.nz;
    d.ldz = M.ldz;
    d.x0 = s.x0;
    d.nt = s.nt;
    d.u[0] = s.u0.as<float>();
    d.u[1] = s.u1.as<float>();
    if (!adjoint) {
        d.src = s.src_f.as<float>();
        d.nsrc = s.nsrc_rows;
        d.rcv = s.rcv_f.as<float>();
        d.nrcv = s.nrcv_rows;
        d.inj = s.d_inj_f.as<InjEntry>();
        d.inj_off = s.d_inj_f_off.as<int>();
        d.ext = s.d_ext_f.as<ExtEntry>();
        d.ext_off = s.d_ext_f_off.as<int>();
        d.n_ext = (int)s.ext_f.size();
        d.mrow = s.d_mrow_f.as<MarchRow>();
    } else {
        d.src = s.src_a.as<float>();
        d.nsrc = s.nrcv_rows;
        d.rcv = nullptr;
        d.nrcv = 0;
        d.inj = s.d_inj_a.as<InjEntry>();
        d.inj_off = s.d_inj_a_off.as<int>();
        d.ext = nullptr;
        d.ext_off = s.d_ext_none_off.as<int>();
        d.n_ext = 0;
        d.mrow = s.d_mrow_a.as<MarchRow>();
    }
    d.den = s.den.as<float>();
    d.tz = s.tz.as<float>();
    d.tx = s.tx.as<float>();
    d.snap = s.snap_base;
    d.snap_slot = (long long)s.ncomp * s.nx * M.ldz;
    d.snap_amax = s.amax.as<unsigned>();
    d.grad = s.grad.as<float>();
    d.gcomp = s.gcomp.as<float>();
    d.gwt = s.gwt.as<float>();
    d.halo_save = s.halo.as<float>();
    (void)P;
}

// Tables of the fluid layer of an acoustic-elastic shot: its own grid, fields,
// injector tables and boundary factors; its traces are the fluid rows of the
// shot's trace buffers (rows [0, nr) of every time sample).
static void shot_dev_fluid(const Plan &P, const ShotPlan &s, bool adjoint, ShotDev &d)
{
    const ShotPlan &w = *s.fluid;
    std::memset(&d, 0, sizeof(d));
    d.nx = w.nx;
    d.nz = P.nza;
    d.ldz = P.ldzw;
    d.x0 = w.x0;
    d.nt = w.nt;
    d.u[0] = w.u0.as<float>();
    d.u[1] = w.u1.as<float>();
    if (!adjoint) {
        d.src = s.src_f.as<float>();
        d.nsrc = s.nsrc_rows;
        d.rcv = s.rcv_f.as<float>();
        d.nrcv = s.nrcv_rows;
        d.inj = w.d_inj_f.as<InjEntry>();
        d.inj_off = w.d_inj_f_off.as<int>();
        d.ext = w.d_ext_f.as<ExtEntry>();
        d.ext_off = w.d_ext_f_off.as<int>();
        d.n_ext = (int)w.ext_f.size();
    } else {
        d.src = s.src_a.as<float>();
        d.nsrc = s.nrcv_rows;
        d.inj = w.d_inj_a.as<InjEntry>();
        d.inj_off = w.d_inj_a_off.as<int>();
        d.ext_off = w.d_ext_none_off.as<int>();
    }
    d.den = w.den.as<float>();
    d.tz = w.tz.as<float>();
    d.tx = w.tx.as<float>();
    d.halo_save = w.halo.as<float>();
}

// Cells touched by the injection at time sample 0, with their entries in
// the reference's order and the double-precision scale of we_op.cpp:657-663.
static void init_factors(const ModelState &M, Plan &P)
{
    const double dt = P.par.dt;
    for (int mode = 0; mode < 2; mode++)
        for (size_t s = 0; s < P.shots.size(); s++) {
            const ShotPlan &S = *P.shots[s];
            for (int c = P.ioff[mode][s]; c < P.ioff[mode][s + 1]; c++) {
                InitCell &q = P.icells[mode][c];
                const size_t mi = (size_t)(S.x0 + q.gx) * M.nz + q.gz;
                if (M.kind == KIND_ACOUSTIC) q.factor = 0.5 * (double)M.host[mi] * dt * dt;
                else q.factor = 0.5 * dt * dt / (double)M.host[2 * (size_t)M.nx * M.nz + mi];
            }
        }
}

static void collect_init_cells(const Plan &P, bool fluid, std::vector<InitCell> *icells, std::vector<int> *iidx,
                               std::vector<int> *ioff)
{
    for (int mode = 0; mode < 2; mode++) {
        icells[mode].clear();
        iidx[mode].clear();
        ioff[mode].assign(P.shots.size() + 1, 0);
        for (size_t s = 0; s < P.shots.size(); s++) {
            const ShotPlan &SP = fluid ? *P.shots[s]->fluid : *P.shots[s];
            const std::vector<InjEntry> &inj = mode ? SP.inj_a : SP.inj_f;
            std::vector<std::vector<int>> lists;
            std::vector<InitCell> cells;
            for (size_t i = 0; i < inj.size(); i++) {
                const InjEntry &e = inj[i];
                size_t k = 0;
                for (; k < cells.size(); k++)
                    if (cells[k].gx == e.gx && cells[k].gz == e.gz && cells[k].comp == e.comp) break;
                if (k == cells.size()) {
                    InitCell q;
                    std::memset(&q, 0, sizeof(q));
                    q.gx = e.gx;
                    q.gz = e.gz;
                    q.comp = e.comp;
                    cells.push_back(q);
                    lists.emplace_back();
                }
                lists[k].push_back((int)i);
            }
            for (size_t k = 0; k < cells.size(); k++) {
                cells[k].i0 = (int)iidx[mode].size();
                iidx[mode].insert(iidx[mode].end(), lists[k].begin(), lists[k].end());
                cells[k].i1 = (int)iidx[mode].size();
                icells[mode].push_back(cells[k]);
            }
            ioff[mode][s + 1] = (int)icells[mode].size();
        }
    }
}

static void build_init_cells(const ModelState &M, Plan &P)
{
    collect_init_cells(P, false, P.icells, P.iidx, P.ioff);
    init_factors(M, P);
    if (P.ae) {
        // the fluid layer's initial state: 0.5 K dt^2 in double (we_op.cpp:2230-2236)
        collect_init_cells(P, true, P.wicells, P.wiidx, P.wioff);
        const double dt = P.par.dt;
        for (int mode = 0; mode < 2; mode++)
            for (auto &q : P.wicells[mode]) q.factor = 0.5 * (double)P.Kw * dt * dt;
    }
}

static void upload_init_cells(Plan &P, cudaStream_t st)
{
    for (int mode = 0; mode < 2; mode++) {
        if (P.ae) {
            P.d_wicells[mode].upload(P.wicells[mode], st);
            P.d_wioff[mode].upload(P.wioff[mode], st);
            P.d_wiidx[mode].upload(P.wiidx[mode], st);
        }
        P.d_icells[mode].upload(P.icells[mode], st);
        P.d_ioff[mode].upload(P.ioff[mode], st);
        P.d_iidx[mode].upload(P.iidx[mode], st);
    }
}

// Snapshot stores and waves.  All shots in one wave when their snapshots fit
// the device (less a reserve for the rest of the work), each shot with its
// own store.  Otherwise contiguous runs of shots, each as large as the
// budget takes, that share one pool as large as the largest run.
// FWI2D_SNAPSHOT_BUDGET (bytes) replaces the budget.  Elastic and VTI plans
// only: checkpointed plans (their replay windows are small), acoustic and
// acoustic-elastic plans keep one wave.
static void plan_waves(Plan &P, bool one_wave)
{
    const int n = (int)P.shots.size();
    size_t total = 0, largest = 0;
    for (auto &S : P.shots) {
        total += S->snap_need;
        largest = std::max(largest, S->snap_need);
    }
    size_t budget = 0;
    if (const char *e = std::getenv("FWI2D_SNAPSHOT_BUDGET")) {
        budget = (size_t)std::strtoull(e, nullptr, 10);
    } else {
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t reserve = (size_t)2 << 30;
        budget = free_b > reserve ? free_b - reserve : 0;
        budget -= budget / 20;
    }
    auto range = [&](Plan::Wave &w, int s0, int s1) {
        w.s0 = s0;
        w.s1 = s1;
        w.nt_max = 0;
        for (int s = s0; s < s1; s++) w.nt_max = std::max(w.nt_max, P.shots[s]->nt);
        const ShotPlan &a = *P.shots[s0];
        w.t0 = a.u_t0;
        w.m0 = a.u_m0;
        w.b0 = a.u_b0;
        w.i0 = a.u_i0;
        w.w0 = a.u_w0;
        if (s1 < n) {
            const ShotPlan &b = *P.shots[s1];
            w.t1 = b.u_t0;
            w.m1 = b.u_m0;
            w.b1 = b.u_b0;
            w.i1 = b.u_i0;
            w.w1 = b.u_w0;
        } else {
            w.t1 = (int)P.tiles.size();
            w.m1 = (int)P.marches.size();
            w.b1 = (int)P.bands.size();
            w.i1 = (int)P.itiles.size();
            w.w1 = (int)P.wtiles.size();
        }
    };
    P.waves.clear();
    range(P.all, 0, n);
    if (one_wave || total <= budget || total == 0) {
        P.waves.push_back(P.all);
        for (auto &S : P.shots) {
            S->snap.alloc(S->snap_need);
            S->snap_base = S->snap.p;
        }
        return;
    }
    if (largest > budget)
        throw Error(FWI2D_ERR_OOM, "the snapshots of one shot exceed the device memory: use checkpoint_every");
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t pool = 0;
    for (int s0 = 0; s0 < n;) {
        size_t bytes = 0;
        int s1 = s0;
        while (s1 < n && (s1 == s0 || bytes + al(P.shots[s1]->snap_need) <= budget))
            bytes += al(P.shots[s1++]->snap_need);
        Plan::Wave w;
        range(w, s0, s1);
        P.waves.push_back(w);
        pool = std::max(pool, bytes);
        s0 = s1;
    }
    P.snap_pool.alloc(pool);
    P.snap_bytes = P.snap_bytes - total + pool;
    for (const auto &w : P.waves) {
        size_t off = 0;
        for (int s = w.s0; s < w.s1; s++) {
            ShotPlan &S = *P.shots[s];
            S.snap.release();
            S.snap_base = (char *)P.snap_pool.p + off;
            off += (S.snap_need + 255) & ~(size_t)255;
        }
    }
}

static void set_shots_impl(fwi2d_ctx *ctx, const fwi2d_params *par, int nshots, const fwi2d_shot *shots)
{
    ModelState &M = ctx->M;
    if (M.kind < 0) throw Error(FWI2D_ERR_STATE, "fwi2d_set_model must be called first");
    REQ(par != nullptr && shots != nullptr && nshots > 0, "no shots");
    const fwi2d_params &p = *par;
    REQ(p.nt >= 2, "nt must be at least 2");
    REQ(p.dt > 0, "dt must be positive");
    REQ(p.sub >= 0, "sub must be >= 0");
    REQ(p.snapshot_precision >= 0 && p.snapshot_precision <= 2, "unknown snapshot precision");
    REQ(p.taper_top >= 0 && p.taper_bottom >= 0 && p.taper_left >= 0 && p.taper_right >= 0, "negative taper");
    const bool ae = M.kind == KIND_AE;
    // acoustic-elastic: the top boundary and its taper belong to the fluid layer
    REQ((ae ? 0 : p.taper_top) + p.taper_bottom <= M.nz, "top and bottom tapers overlap");
    for (int i = 0; i < 4; i++) {
        int bc = (&p.bc_top)[i];
        REQ(bc >= 1 && bc <= 3, "boundary condition must be 1, 2 or 3");
        if (M.kind != KIND_ACOUSTIC && !(ae && i == 0))
            REQ(bc <= 2, "the elastic propagators take boundary conditions 1 or 2");
    }
    if (ae) {
        REQ(p.nza >= 12, "acoustic-elastic: the fluid layer needs nza >= 12 rows");
        REQ(p.water_velocity > 0 && p.water_density > 0, "acoustic-elastic: water velocity and density must be positive");
        REQ(p.taper_top <= p.nza, "acoustic-elastic: the top taper is longer than the fluid layer");
        REQ(!p.mt, "acoustic-elastic: point sources only (mt = 0)");
        REQ(p.checkpoint_every == 0, "acoustic-elastic: checkpoint-and-recompute is not available");
    }
    const bool acoustic = M.kind == KIND_ACOUSTIC;
    REQ(!(acoustic && p.mt), "the acoustic propagator takes point sources only (mt = 0)");
    REQ(p.checkpoint_every >= 0, "checkpoint_every must be >= 0");
    if (p.checkpoint_every > 0) {
        REQ(p.sub == 1, "checkpoint-and-recompute needs sub = 1");
        for (int s = 1; s < nshots; s++)
            if (shots[s].nt != shots[0].nt)
                throw Error(FWI2D_ERR_UNSUPPORTED,
                            "checkpoint-and-recompute needs every shot of the plan to have the same nt");
    }
    set_device(ctx);

    auto P = std::make_unique<Plan>();
    P->par = p;
    P->kind = M.kind;
    P->ncompg = M.kind == KIND_ACOUSTIC ? 2 : 3;
    P->C = make_const(p, M.dx, M.dz);
    P->dtg = (float)(P->C.sub) * p.dt;
    if (ae) {
        // elastic grid: its top edge is the fluid interface (traction-free SAT);
        // fluid layer: the reference's top, left and right conditions and a
        // Neumann interface at its bottom (we_op.cpp:2400-2480)
        P->C.bc[0] = 1;
        P->Cw = make_const(p, M.dx, M.dz);
        P->Cw.bc[1] = 3;
        P->ae = true;
        P->ae_src_fluid = p.acoustic_source != 0;
        P->nza = p.nza;
        P->ldzw = round_up(p.nza, 32);
        const float rw = p.water_density;
        P->Kw = rw * p.water_velocity * p.water_velocity;
        const float h = (float)((double)M.dz * (17.0 / 48));   // interface row weight, we_op.cpp:2490
        P->val0 = p.dt / (2 * h);
        std::vector<float> wk((size_t)M.nx * P->ldzw, P->Kw), wir((size_t)M.nx * P->ldzw, (float)(1.0 / rw));
        P->wK.upload(wk, ctx->st);
        P->wIR.upload(wir, ctx->st);
    }

    // shape: the requested one, else the marching kernel where it has enough
    // units to fill the GPU, else the first tile shape that fits every shot
    auto shape_ok = [&](int i) {
        if ((acoustic || ae) && !acoustic_shape_ok(i)) return false;
        for (int s = 0; s < nshots; s++)
            if (!shape_fits(i, shots[s].nx, M.nz)) return false;
        return true;
    };
    int shape = p.tile_shape;
    if (shape < 0 || shape >= shape_count()) {
        shape = -1;
        const int m0 = elastic_tile_count();
        if (!acoustic && !ae && shape_ok(m0)) {
            long long units = 0;
            for (int s = 0; s < nshots; s++)
                units += (long long)make_units(m0, s, shots[s].nx, M.nz, false).marches.size();
            if (units >= 148) shape = m0;
        }
        for (int i = 0; i < elastic_tile_count() && shape < 0; i++)
            if (shape_ok(i)) shape = i;
        REQ(shape >= 0, "no tile shape fits the grid (an axis needs n == T or n >= T + 8)");
    }
    REQ(shape_ok(shape), "the requested tile shape does not fit a shot grid");
    P->shape = shape;
    P->march = is_march_shape(shape);
    P->framed = is_framed_shape(shape);
    P->tshape = P->march || P->framed ? kBandTile : shape;
    if (P->framed) P->ishape = framed_tile_shape(shape);
    P->band_split = (P->march || P->framed) && band_split_for(nshots, M.nz);
    elastic_tile_shape(P->tshape, &P->TZ, &P->TX);
    if (P->march) {
        P->nth = kMarchShapes[shape - elastic_tile_count()].nth;
        P->lx = kMarchShapes[shape - elastic_tile_count()].lx;
    }

    const bool vti = M.kind == KIND_VTI;
    long long total_bytes = 0;
    for (int s = 0; s < nshots; s++) {
        const fwi2d_shot &sh = shots[s];
        REQ(sh.x0 >= 0 && sh.nx >= 12 && sh.x0 + sh.nx <= M.nx, "shot grid outside the model");
        REQ(sh.nt >= 2 && sh.nt <= p.nt, "shot nt must be in [2, params.nt]");
        REQ(p.taper_left + p.taper_right <= sh.nx, "left and right tapers overlap");
        const bool src_fluid = ae && p.acoustic_source;
        const fwi2d_injector none = {FWI2D_INJ_DELTA, 0, nullptr, nullptr, nullptr, nullptr};
        const fwi2d_injector &esrc = src_fluid ? none : sh.src;
        REQ((src_fluid ? sh.src_water.ntr : sh.src.ntr) > 0, "shot without source");
        REQ(sh.rcv.ntr > 0 && sh.rcv.type == FWI2D_INJ_DELTA, "shot receivers must be a delta injector");
        if (!src_fluid)
            REQ((sh.src.type == FWI2D_INJ_DDELTA) == (p.mt != 0), "source injector type must match params.mt");
        check_injector(esrc, sh.nx, M.nz, "source");
        check_injector(sh.rcv, sh.nx, M.nz, "receivers");
        if (ae) {
            REQ(sh.rcv_water.ntr == sh.rcv.ntr && sh.rcv_water.type == FWI2D_INJ_DELTA,
                "acoustic-elastic: the fluid receivers must be a delta injector with as many traces as the elastic ones");
            check_injector(sh.rcv_water, sh.nx, p.nza, "fluid receivers");
            if (src_fluid) {
                REQ(sh.src_water.type == FWI2D_INJ_DELTA, "acoustic-elastic: the fluid source must be a delta injector");
                check_injector(sh.src_water, sh.nx, p.nza, "fluid source");
            }
        }
        auto S = std::make_unique<ShotPlan>();
        S->x0 = sh.x0;
        S->nx = sh.nx;
        S->nt = sh.nt;
        S->ncomp = acoustic ? 1 : 2;
        const ShotUnits U = make_units(shape, s, sh.nx, M.nz, P->band_split);
        const int nunits = U.nunits();
        S->ntr_src = src_fluid ? sh.src_water.ntr : sh.src.ntr;
        S->ncomp_src = acoustic || src_fluid ? 1 : (p.mt ? 3 : 2);
        S->nr = sh.rcv.ntr;
        S->nsrc_rows = S->ncomp_src * S->ntr_src;
        // acoustic-elastic traces: [fluid, x, z] blocks of nr rows (we_op.cpp:2199-2214)
        S->nrcv_rows = (ae ? 3 : S->ncomp) * S->nr;
        // forward sources: force -> rows c*ntr ; moment tensor blocks (mxx, mzz, mxz)
        int ra[2], rb[2];
        if (!p.mt) {
            ra[0] = 0;
            ra[1] = S->ntr_src;
            rb[0] = rb[1] = 0;
        } else {
            ra[0] = 0;                  // next0: inx = mxx, inz = mxz  (we_op.cpp:618-621)
            rb[0] = 2 * S->ntr_src;
            ra[1] = 2 * S->ntr_src;     // next1: inx = mxz, inz = mzz
            rb[1] = S->ntr_src;
        }
        build_inj(esrc, S->ncomp, ra, rb, U, S->inj_f, S->inj_f_off, S->inj_f_roff);
        const int r0 = ae ? S->nr : 0;   // first elastic row of the traces
        int qa[2] = {r0, r0 + S->nr}, qb[2] = {0, 0};
        build_inj(sh.rcv, S->ncomp, qa, qb, U, S->inj_a, S->inj_a_off, S->inj_a_roff);
        build_ext(sh.rcv, S->ncomp, U, S->ext_f, S->ext_f_off, S->ext_f_roff, r0);
        S->ext_none_off.assign(nunits + 1, 0);

        // boundary divisors and taper on this shot's window of the model
        std::vector<float> den, tz, tx;
        if (acoustic) {
            const float *K = M.hp(0) + (size_t)sh.x0 * M.nz, *irho = M.hp(1) + (size_t)sh.x0 * M.nz;
            acoustic_scale_divisors(sh.nx, M.nz, M.dx, M.dz, p.dt, K, irho, M.nz, p.bc_top == 2, p.bc_bottom == 2,
                                    p.bc_left == 2, p.bc_right == 2, den);
        } else {
            const float *lam = M.hp(0) + (size_t)sh.x0 * M.nz, *mu = M.hp(1) + (size_t)sh.x0 * M.nz,
                        *rho = M.hp(2) + (size_t)sh.x0 * M.nz;
            const float *eps = vti ? M.hp(4) + (size_t)sh.x0 * M.nz : nullptr;
            elastic_scale_divisors(sh.nx, M.nz, M.dx, M.dz, p.dt, lam, mu, rho, eps, M.nz, !ae && p.bc_top == 2,
                                   p.bc_bottom == 2, p.bc_left == 2, p.bc_right == 2, den);
        }
        taper_factors(sh.nx, M.nz, ae ? 0 : p.taper_top, p.taper_bottom, p.taper_left, p.taper_right,
                      p.taper_strength, true, true, true, true, tz, tx);
        if (ae) {
            // the fluid layer's grid of this shot: same columns, nza rows
            auto W = std::make_unique<ShotPlan>();
            W->x0 = sh.x0;
            W->nx = sh.nx;
            W->nt = sh.nt;
            W->ncomp = 1;
            W->nr = sh.rcv_water.ntr;
            const ShotUnits UW = make_units(shape, s, sh.nx, p.nza, P->band_split);
            int wa[2] = {0, 0}, wb[2] = {0, 0};
            build_inj(src_fluid ? sh.src_water : none, 1, wa, wb, UW, W->inj_f, W->inj_f_off, W->inj_f_roff);
            build_inj(sh.rcv_water, 1, wa, wb, UW, W->inj_a, W->inj_a_off, W->inj_a_roff);
            build_ext(sh.rcv_water, 1, UW, W->ext_f, W->ext_f_off, W->ext_f_roff, 0);
            W->ext_none_off.assign(UW.nunits() + 1, 0);
            std::vector<float> wk((size_t)sh.nx * p.nza, P->Kw), wir((size_t)sh.nx * p.nza, (float)(1.0 / p.water_density));
            std::vector<float> wden, wtz, wtx;
            acoustic_scale_divisors(sh.nx, p.nza, M.dx, M.dz, p.dt, wk.data(), wir.data(), p.nza, p.bc_top == 2, false,
                                    p.bc_left == 2, p.bc_right == 2, wden);
            taper_factors(sh.nx, p.nza, p.taper_top, 0, p.taper_left, p.taper_right, p.taper_strength, true, true,
                          true, true, wtz, wtx);
            const size_t wfield = (size_t)sh.nx * P->ldzw;
            W->u0.alloc(wfield * sizeof(float));
            W->u1.alloc(wfield * sizeof(float));
            W->halo.alloc((size_t)sh.nx * sizeof(float));
            W->d_inj_f.upload(W->inj_f, ctx->st);
            W->d_inj_f_off.upload(W->inj_f_off, ctx->st);
            W->d_inj_a.upload(W->inj_a, ctx->st);
            W->d_inj_a_off.upload(W->inj_a_off, ctx->st);
            W->d_ext_f.upload(W->ext_f, ctx->st);
            W->d_ext_f_off.upload(W->ext_f_off, ctx->st);
            W->d_ext_none_off.upload(W->ext_none_off, ctx->st);
            W->den.upload(wden, ctx->st);
            W->tz.upload(wtz, ctx->st);
            W->tx.upload(wtx, ctx->st);
            S->u_w0 = (int)P->wtiles.size();
            P->wtiles.insert(P->wtiles.end(), UW.tiles.begin(), UW.tiles.end());
            S->halo.alloc((size_t)sh.nx * sizeof(float));
            S->fluid = std::move(W);
            P->nx_max = std::max(P->nx_max, sh.nx);
        }
        S->nslot = p.sub > 0 ? 1 + sh.nt / p.sub : 0;
        std::vector<float> gw(std::max(S->nslot, 1), 1.f);
        for (int i = 0; i < S->nslot; i++) {
            float t = i * P->dtg;
            float w = 1;
            if (p.gdamp_tmax - t > 0 && t - p.gdamp_tmin >= 0)
                w = (float)std::cos(p.gdamp_power * M_PI * (t - p.gdamp_tmin) / (p.gdamp_tmax - p.gdamp_tmin));
            w *= w;
            gw[i] = w;
        }

        const size_t field = (size_t)S->ncomp * sh.nx * M.ldz;
        S->u0.alloc(field * sizeof(float));
        S->u1.alloc(field * sizeof(float));
        S->src_f.alloc((size_t)sh.nt * S->nsrc_rows * sizeof(float));
        S->rcv_f.alloc((size_t)sh.nt * S->nrcv_rows * sizeof(float));
        S->src_a.alloc((size_t)sh.nt * S->nrcv_rows * sizeof(float));
        S->d_inj_f.upload(S->inj_f, ctx->st);
        S->d_inj_f_off.upload(S->inj_f_off, ctx->st);
        S->d_inj_a.upload(S->inj_a, ctx->st);
        S->d_inj_a_off.upload(S->inj_a_off, ctx->st);
        S->d_ext_f.upload(S->ext_f, ctx->st);
        S->d_ext_f_off.upload(S->ext_f_off, ctx->st);
        S->d_ext_none_off.upload(S->ext_none_off, ctx->st);
        build_march_rows(U, S->inj_f, S->inj_f_roff, &S->ext_f_roff, tx, S->mrow_f);
        build_march_rows(U, S->inj_a, S->inj_a_roff, nullptr, tx, S->mrow_a);
        S->d_mrow_f.upload(S->mrow_f, ctx->st);
        S->d_mrow_a.upload(S->mrow_a, ctx->st);
        S->den.upload(den, ctx->st);
        S->tz.upload(tz, ctx->st);
        S->tx.upload(tx, ctx->st);
        S->gwt.upload(gw, ctx->st);
        S->grad.alloc((size_t)P->ncompg * sh.nx * M.ldz * sizeof(float));
        if (p.compensated && p.sub > 0) S->gcomp.alloc(2 * S->grad.n);
        else S->gcomp.release();
        if (S->nslot > 0) {
            const size_t esz = p.snapshot_precision == FWI2D_SNAP_FP32 ? 4 : 2;
            const int K = p.checkpoint_every;
            // checkpointing: a replay window of K + 2 slots (times cuts[k]-1 .. cuts[k+1])
            S->nbuf = K > 0 ? std::min(S->nslot, K + 2) : S->nslot;
            size_t bytes = (size_t)S->nbuf * field * esz;
            S->snap_need = bytes;   // allocated below, once the waves are known
            S->amax.alloc((size_t)S->nslot * sizeof(unsigned));
            if (K > 0) {
                const int nseg = (sh.nt - 1 + K - 1) / K;
                S->r0.alloc(field * sizeof(float));
                S->r1.alloc(field * sizeof(float));
                if (nseg > 1) S->ckpt.alloc((size_t)(nseg - 1) * 2 * field * sizeof(float));
                bytes += S->r0.n + S->r1.n + S->ckpt.n;
            }
            P->snap_bytes += bytes;
            total_bytes += bytes;
        }
        P->nt_max = std::max(P->nt_max, sh.nt);
        S->u_t0 = (int)P->tiles.size();
        S->u_m0 = (int)P->marches.size();
        S->u_b0 = (int)P->bands.size();
        S->u_i0 = (int)P->itiles.size();
        P->tiles.insert(P->tiles.end(), U.tiles.begin(), U.tiles.end());
        P->marches.insert(P->marches.end(), U.marches.begin(), U.marches.end());
        P->bands.insert(P->bands.end(), U.bands.begin(), U.bands.end());
        P->itiles.insert(P->itiles.end(), U.itiles.begin(), U.itiles.end());
        P->shots.push_back(std::move(S));
    }
    P->have_snapshots = p.sub > 0;
    plan_waves(*P, p.checkpoint_every > 0);
    P->d_tiles.upload(P->tiles, ctx->st);
    P->d_march.upload(P->marches, ctx->st);
    P->d_bands.upload(P->bands, ctx->st);
    P->d_itiles.upload(P->itiles, ctx->st);
    std::vector<ShotDev> sf(nshots), sa(nshots);
    for (int s = 0; s < nshots; s++) {
        shot_dev(*P, *P->shots[s], M, false, sf[s]);
        shot_dev(*P, *P->shots[s], M, true, sa[s]);
    }
    for (int s = 0; s < nshots; s++) sf[s].ckpt = P->shots[s]->ckpt.as<float>();
    P->d_shots_f.upload(sf, ctx->st);
    P->d_shots_a.upload(sa, ctx->st);
    if (ae) {
        std::vector<ShotDev> wf(nshots), wa(nshots);
        for (int s = 0; s < nshots; s++) {
            shot_dev_fluid(*P, *P->shots[s], false, wf[s]);
            shot_dev_fluid(*P, *P->shots[s], true, wa[s]);
        }
        P->d_wshots_f.upload(wf, ctx->st);
        P->d_wshots_a.upload(wa, ctx->st);
        P->d_wtiles.upload(P->wtiles, ctx->st);
    }
    if (p.checkpoint_every > 0) {
        const int K = p.checkpoint_every, nt = P->nt_max;
        P->ckpt = K;
        P->cuts.clear();
        for (int t = 0; t < nt - 1; t += K) P->cuts.push_back(t);
        P->cuts.push_back(nt - 1);
        const int nseg = (int)P->cuts.size() - 1;
        const size_t esz = p.snapshot_precision == FWI2D_SNAP_FP32 ? 4 : 2;
        std::vector<ShotDev> sr((size_t)nseg * nshots), sc((size_t)nseg * nshots);
        for (int k = 0; k < nseg; k++) {
            // slot t of segment k lives at window index t - base (base = cuts[k] - 1, or -1 for
            // segment 0): the tables carry the window's address shifted by -base slots, so the
            // kernels index it with the absolute time; only slots of the window are accessed
            const long long base = k == 0 ? -1 : P->cuts[k] - 1;
            for (int s = 0; s < nshots; s++) {
                ShotPlan &S = *P->shots[s];
                char *win = (char *)S.snap_base - base * (long long)sf[s].snap_slot * (long long)esz;
                ShotDev r = sf[s];
                r.u[0] = S.r0.as<float>();
                r.u[1] = S.r1.as<float>();
                r.rcv = nullptr;
                r.nrcv = 0;
                r.snap = win;
                ShotDev a = sa[s];
                a.snap = win;
                sr[(size_t)k * nshots + s] = r;
                sc[(size_t)k * nshots + s] = a;
            }
        }
        P->d_shots_r.upload(sr, ctx->st);
        P->d_shots_c.upload(sc, ctx->st);
    }
    build_init_cells(M, *P);
    upload_init_cells(*P, ctx->st);
    P->d_grad_full.alloc((size_t)P->ncompg * M.nx * M.ldz * sizeof(float));
    P->d_status.alloc(sizeof(int));
    CK(cudaMemsetAsync(P->d_status.p, 0, sizeof(int), ctx->st));
    CK(cudaMallocHost((void **)&P->h_status, sizeof(int)));
    *P->h_status = 0;
    CK(cudaStreamSynchronize(ctx->st));
    ctx->plan = std::move(P);
}

// After a pass has finished (its stream synchronised): a bounded device wait
// that gave up during it makes the pass's results invalid.  Clears the status
// and reports FWI2D_ERR_TIMEOUT.
static void check_timeout(fwi2d_ctx *ctx)
{
    if (!ctx->plan || !ctx->plan->h_status) return;
    Plan &P = *ctx->plan;
    const int v = *P.h_status;
    if (v == 0) return;
    *P.h_status = 0;
    CK(cudaMemsetAsync(P.d_status.p, 0, sizeof(int), ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    P.snapshots_valid = false;
    throw Error(FWI2D_ERR_TIMEOUT, "a bounded device wait of the marching kernel reached its limit (row " +
                                       std::to_string(v - 1) + "); the results of this pass are not trusted");
}

// Queue the move of the device timeout flag into the plan's status word and
// its copy to the host (read by check_timeout once the stream has finished).
static void queue_timeout_check(fwi2d_ctx *ctx, Plan &P)
{
    launch_take_timeout(P.d_status.as<int>(), ctx->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(P.h_status, P.d_status.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
}

// One time step of every shot.  Tile-only plans: one launch.  Marching
// plans: the marching kernel on `st` while the tile kernel computes the
// boundary bands on the context's side stream; the two branches write
// disjoint cells and join before the next step.  Returns the number of
// launches.
static int launch_step(fwi2d_ctx *ctx, const Plan &P, const ShotDev *shots, const ModelDev &md, int it, int flags,
                       cudaStream_t st, const Plan::Wave *wave = nullptr)
{
    // the units of the wave's shots (the kernels index the shot tables by the
    // units' own shot numbers)
    const Plan::Wave &R = wave ? *wave : P.all;
    const TileRef *tiles = P.d_tiles.as<TileRef>() + R.t0;
    const int ntiles = R.t1 - R.t0;
    int n = 0;
    if (P.ae) {
        // fluid layer, elastic grid, then the implicit interface coupling
        const bool adj = (flags & STEP_GRAD) != 0;
        const ShotDev *wshots = (adj ? P.d_wshots_a : P.d_wshots_f).as<ShotDev>();
        launch_ae_fluid_step(P.tshape, wshots, P.d_wtiles.as<TileRef>() + R.w0, R.w1 - R.w0, P.wdev(), P.Cw, it,
                             flags & STEP_EXTRACT, st);
        launch_ae_elastic_step(P.tshape, shots, tiles, ntiles, md, P.C, it, flags, P.dtg, st);
        launch_ae_couple(shots + R.s0, wshots + R.s0, R.s1 - R.s0, P.nx_max, md, P.C, it, flags, P.dtg, P.Kw, P.val0,
                         adj ? -1 : 1, st);
        return 3;
    }
    if (P.kind == KIND_ACOUSTIC) {
        launch_acoustic_step(P.tshape, shots, tiles, ntiles, md, P.C, it, flags, P.dtg, st);
        return 1;
    }
    if (!P.march && !P.framed) {
        launch_elastic_step(P.tshape, P.kind == KIND_VTI, shots, tiles, ntiles, md, P.C, it, flags, P.dtg, st);
        return 1;
    }
    // the x-band tiles and the top / bottom bands on two side streams, beside the core
    CK(cudaEventRecord(ctx->fork, st));
    CK(cudaStreamWaitEvent(ctx->side, ctx->fork, 0));
    CK(cudaStreamWaitEvent(ctx->side2, ctx->fork, 0));
    launch_elastic_xband(P.kind == KIND_VTI, P.band_split, shots, tiles, ntiles, md, P.C, it, flags, P.dtg, ctx->side);
    launch_elastic_zband(P.kind == KIND_VTI, P.band_split, P.d_bands.as<BandRef>() + R.b0, R.b1 - R.b0, shots, md, P.C,
                         it, flags, P.dtg, ctx->side2);
    n += 2;
    CK(cudaEventRecord(ctx->join, ctx->side));
    CK(cudaEventRecord(ctx->join2, ctx->side2));
    if (P.framed)
        launch_elastic_step(P.ishape, P.kind == KIND_VTI, shots, P.d_itiles.as<TileRef>() + R.i0, R.i1 - R.i0, md,
                            P.C, it, flags, P.dtg, st, true);
    else
        launch_elastic_march(P.kind == KIND_VTI, shots, P.d_march.as<MarchRef>() + R.m0, R.m1 - R.m0, P.nth, md, P.C,
                             it, flags, P.dtg, st);
    n++;
    CK(cudaStreamWaitEvent(st, ctx->join, 0));
    CK(cudaStreamWaitEvent(st, ctx->join2, 0));
    return n;
}

// Time `steps` forward steps of the current plan from launch it0 (fields
// zeroed, no output), in milliseconds per step.  Shots whose records end
// before a launch return from it, as in a full pass.
static float time_forward_steps(fwi2d_ctx *ctx, int steps, int it0 = 0)
{
    Plan &P = *ctx->plan;
    for (auto &S : P.shots) {
        CK(cudaMemsetAsync(S->u0.p, 0, S->u0.n, ctx->st));
        CK(cudaMemsetAsync(S->u1.p, 0, S->u1.n, ctx->st));
    }
    const ModelDev md = ctx->M.dev();
    const ShotDev *shots = P.d_shots_f.as<ShotDev>();
    const int nsteps = std::max(0, std::min(steps, P.nt_max - 1 - it0));
    for (int it = it0; it < it0 + std::min(3, nsteps); it++)
        launch_step(ctx, P, shots, md, it, STEP_EXTRACT, ctx->st);
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, ctx->st));
    for (int it = it0; it < it0 + nsteps; it++) launch_step(ctx, P, shots, md, it, STEP_EXTRACT, ctx->st);
    CK(cudaEventRecord(b, ctx->st));
    CK(cudaEventSynchronize(b));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(cudaGetLastError());
    return ms / std::max(nsteps, 1);
}

// Time `steps` adjoint steps with the imaging condition of the current plan
// (built without snapshot storage), in milliseconds per step.  Every shot
// images against a scratch window of 3 snapshot slots (zeroed), addressed like
// the checkpoint windows: the shot tables carry the window shifted to the
// snapshot index of the timed step.
static float time_adjoint_steps(fwi2d_ctx *ctx, int steps)
{
    Plan &P = *ctx->plan;
    const ModelState &M = ctx->M;
    int nt_min = P.nt_max;
    for (auto &S : P.shots) nt_min = std::min(nt_min, S->nt);
    if (nt_min < 4) return 0.f;
    const int it = nt_min - 3;   // every shot active, imaged snapshot index >= 1
    const size_t esz = P.par.snapshot_precision == FWI2D_SNAP_FP32 ? 4 : 2;
    std::vector<ShotDev> sd(P.shots.size());
    CK(cudaMemcpy(sd.data(), P.d_shots_a.p, sd.size() * sizeof(ShotDev), cudaMemcpyDeviceToHost));
    std::vector<std::unique_ptr<DevBuf>> win(P.shots.size()), amx(P.shots.size());
    DevBuf ones;
    ones.upload(std::vector<float>(3, 1.f), ctx->st);
    for (size_t s = 0; s < P.shots.size(); s++) {
        ShotPlan &S = *P.shots[s];
        const long long slot = (long long)S.ncomp * S.nx * M.ldz;
        // snapshot index imaged at launch it: nt-2-it (elastic), nt-1-it (acoustic)
        const long long itf = S.nt - (P.kind == KIND_ACOUSTIC ? 1 : 2) - it;
        win[s] = std::make_unique<DevBuf>();
        win[s]->alloc(3 * (size_t)slot * esz);
        amx[s] = std::make_unique<DevBuf>();
        amx[s]->alloc(3 * sizeof(unsigned));
        CK(cudaMemsetAsync(win[s]->p, 0, win[s]->n, ctx->st));
        CK(cudaMemsetAsync(amx[s]->p, 0, amx[s]->n, ctx->st));
        CK(cudaMemsetAsync(S.u0.p, 0, S.u0.n, ctx->st));
        CK(cudaMemsetAsync(S.u1.p, 0, S.u1.n, ctx->st));
        CK(cudaMemsetAsync(S.src_a.p, 0, S.src_a.n, ctx->st));
        // slots itf-1 .. itf+1 of this shot map onto the window's 0 .. 2
        sd[s].snap = (char *)win[s]->p - (itf - 1) * slot * (long long)esz;
        sd[s].snap_slot = slot;
        sd[s].snap_amax = amx[s]->as<unsigned>() - (itf - 1);
        sd[s].gwt = ones.as<float>() - (itf - 1);
    }
    DevBuf d_sd;
    d_sd.upload(sd, ctx->st);
    const ModelDev md = M.dev();
    const ShotDev *shots = d_sd.as<ShotDev>();
    for (int k = 0; k < std::min(3, steps); k++) launch_step(ctx, P, shots, md, it, STEP_GRAD, ctx->st);
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, ctx->st));
    for (int k = 0; k < steps; k++) launch_step(ctx, P, shots, md, it, STEP_GRAD, ctx->st);
    CK(cudaEventRecord(b, ctx->st));
    CK(cudaEventSynchronize(b));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(cudaGetLastError());
    return ms / std::max(steps, 1);
}

// Autotuner choices also persist across processes in the file named by the
// environment variable FWI2D_TUNE_FILE (lines "<key> <shape>"), keyed by the
// library build and the device, so that a later run -- for instance one under
// a profiler, whose serialised launches would skew the timing -- reuses the
// measured choice.
static std::string tune_build_key(int device)
{
    cudaDeviceProp pr;
    CK(cudaGetDeviceProperties(&pr, device));
    std::string k = std::string(__DATE__ "_" __TIME__) + "/" + pr.name + "/" + std::to_string(pr.multiProcessorCount);
    for (auto &c : k)
        if (c == ' ') c = '_';
    return k;
}

static int tune_file_lookup(const std::string &key)
{
    const char *path = std::getenv("FWI2D_TUNE_FILE");
    if (!path || !*path) return -1;
    FILE *f = std::fopen(path, "r");
    if (!f) return -1;
    char k[1024];
    int v, found = -1;
    while (std::fscanf(f, "%1023s %d", k, &v) == 2)
        if (key == k) found = v;
    std::fclose(f);
    return found;
}

static void tune_file_store(const std::string &key, int shape)
{
    const char *path = std::getenv("FWI2D_TUNE_FILE");
    if (!path || !*path || key.size() >= 1024) return;
    FILE *f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d\n", key.c_str(), shape);
    std::fclose(f);
}

// Tile-shape autotuner: for plans that leave the shape open (tile_shape < 0),
// time forward steps of every shape that tiles the grids -- plus adjoint
// steps with the imaging condition for plans that keep snapshots (gradients)
// -- and keep the fastest.  The forward is sampled in kTuneWindows windows
// centred on equal parts of the whole time loop, so that a batch whose
// shorter records end early is judged on its emptier late steps too (there,
// units fewer than a wave favour narrower shapes); the adjoint, timed with
// every shot active, is scaled by the ratio of the sampled loop to the
// all-active forward steps.  The choice is cached per (kind, nz, snapshots,
// shot grid widths).
constexpr int kTuneWindows = 8, kTuneWindowSteps = 8;
// Gradient plans: the shapes whose sampled score lies within kTuneClose of the
// best are then timed over one whole forward pass with snapshots and one
// adjoint pass, through the plan's own CUDA graphs (the sampled steps run as
// plain stream launches and miss part of the tail's cost).  The environment
// variable FWI2D_TUNE_CLOSE overrides the ratio (e.g. 100 to time every shape).
constexpr float kTuneClose = 1.04f;

static float tune_close()
{
    const char *v = std::getenv("FWI2D_TUNE_CLOSE");
    const float r = v ? (float)std::atof(v) : 0.f;
    return r >= 1.f ? r : kTuneClose;
}

static void run(fwi2d_ctx *ctx, bool adjoint, bool store);
static void run_wave(fwi2d_ctx *ctx, Plan &P, int w, bool adjoint);
static float pass_ms(Plan &P, int e);

// One whole forward pass with snapshots and one adjoint pass of the current
// plan on zero traces, in milliseconds (the plan's graphs, CUDA events).
static float time_full_pass(fwi2d_ctx *ctx)
{
    Plan &P = *ctx->plan;
    for (auto &S : P.shots) {
        CK(cudaMemsetAsync(S->src_f.p, 0, S->src_f.n, ctx->st));
        CK(cudaMemsetAsync(S->src_a.p, 0, S->src_a.n, ctx->st));
    }
    for (int w = 0; w < (int)P.waves.size(); w++) {
        run_wave(ctx, P, w, false);
        run_wave(ctx, P, w, true);
    }
    CK(cudaStreamSynchronize(ctx->st));
    return pass_ms(P, 0) + pass_ms(P, 1);
}
static void set_shots(fwi2d_ctx *ctx, const fwi2d_params *par, int nshots, const fwi2d_shot *shots)
{
    REQ(par != nullptr && shots != nullptr && nshots > 0, "no shots");
    fwi2d_params p = *par;
    if (p.tile_shape < 0 && ctx->M.kind >= 0) {
        static std::vector<std::pair<std::string, int>> cache;
        const bool grad = p.sub > 0;
        std::string key = tune_build_key(ctx->device) + "/" + std::to_string(ctx->M.kind) + "/" +
                          std::to_string(ctx->M.nz) + "/" + (grad ? "g" + std::to_string(p.snapshot_precision) : "f") +
                          "/" + std::to_string(nshots) + (band_split_for(nshots, ctx->M.nz) ? "/bs" : "");
        long long cells = 0;
        for (int i = 0; i < nshots; i++) {
            key += "/" + std::to_string(shots[i].nx);
            cells += (long long)shots[i].nx * ctx->M.nz * shots[i].nt;
        }
        int chosen = -1;
        for (auto &kv : cache)
            if (kv.first == key) chosen = kv.second;
        if (chosen < 0 && cells >= 20000000LL) {
            chosen = tune_file_lookup(key);
            if (chosen >= shape_count()) chosen = -1;
            if (chosen >= 0) cache.emplace_back(key, chosen);
        }
        if (chosen < 0 && cells >= 20000000LL) {
            float best = 1e30f;
            std::vector<std::pair<float, int>> scored;
            for (int s = 0; s < shape_count(); s++) {
                fwi2d_params q = p;
                q.tile_shape = s;
                q.sub = 0;
                q.checkpoint_every = 0;
                try {
                    set_shots_impl(ctx, &q, nshots, shots);
                } catch (const Error &e) {
                    if (e.code == FWI2D_ERR_ARG) continue;   // shape does not tile these grids
                    throw;
                }
                const int ntm = ctx->plan->nt_max;
                float ms;
                if (ntm - 1 >= 2 * kTuneWindows * kTuneWindowSteps) {
                    // all shots active in the first steps: the reference for the adjoint's scaling
                    const float first = time_forward_steps(ctx, kTuneWindowSteps, 0);
                    float all = 0.f;
                    for (int w = 0; w < kTuneWindows; w++) {
                        const int it0 = (int)(((long long)(2 * w + 1) * (ntm - 1)) / (2 * kTuneWindows));
                        all += time_forward_steps(ctx, kTuneWindowSteps, it0) / kTuneWindows;
                    }
                    ms = all;
                    const float adj = grad ? time_adjoint_steps(ctx, 30) : 0.f;
                    if (grad) ms += adj * (first > 0.f ? all / first : 1.f);
                    if (std::getenv("FWI2D_TUNE_VERBOSE"))
                        std::fprintf(stderr, "fwi2d autotune: shape %d forward %.4f ms/step (all active %.4f), "
                                     "adjoint %.4f ms/step, score %.4f\n", s, all, first, adj, ms);
                } else {
                    ms = time_forward_steps(ctx, 30);
                    if (grad) ms += time_adjoint_steps(ctx, 30);
                    if (std::getenv("FWI2D_TUNE_VERBOSE"))
                        std::fprintf(stderr, "fwi2d autotune: shape %d score %.4f ms/step\n", s, ms);
                }
                scored.emplace_back(ms, s);
                if (ms < best) {
                    best = ms;
                    chosen = s;
                }
            }
            ctx->plan.reset();
            const float ratio = tune_close();
            int close = 0;
            for (auto &sc : scored) close += sc.first <= ratio * best;
            if (grad && close > 1) {
                float bestf = 1e30f;
                for (auto &sc : scored) {
                    if (sc.first > ratio * best) continue;
                    fwi2d_params q = p;
                    q.tile_shape = sc.second;
                    set_shots_impl(ctx, &q, nshots, shots);
                    const float t = time_full_pass(ctx);
                    ctx->plan.reset();   // before the next plan allocates its snapshots
                    if (std::getenv("FWI2D_TUNE_VERBOSE"))
                        std::fprintf(stderr, "fwi2d autotune: shape %d whole forward + adjoint %.1f ms\n", sc.second,
                                     t);
                    if (t < bestf) {
                        bestf = t;
                        chosen = sc.second;
                    }
                }
            }
            if (chosen >= 0) {
                cache.emplace_back(key, chosen);
                tune_file_store(key, chosen);
            }
        }
        p.tile_shape = chosen;
    }
    set_shots_impl(ctx, &p, nshots, shots);
}

// Compensated accumulation (params.compensated): after adjoint launch
// `count` (1-based), close a window every kCompWindow launches; `final` adds
// the last window and leaves the sum in the gradient accumulators.  Returns
// the number of launches.
static int grad_flush(const Plan &P, const Plan::Wave &R, int count, bool final, cudaStream_t st)
{
    if (!P.par.compensated || P.shots.empty() || !P.shots[0]->gcomp.p) return 0;
    if (!final && count % kCompWindow != 0) return 0;
    k_grad_flush<<<dim3(148, (unsigned)(R.s1 - R.s0)), 256, 0, st>>>(P.d_shots_a.as<ShotDev>() + R.s0, P.ncompg,
                                                                        final ? 1 : 0);
    CK(cudaGetLastError());
    return 1;
}

// Checkpoint-and-recompute time loops (all shots share nt, sub = 1).
// Forward: receivers and 16-bit snapshot scales as usual, no snapshot store;
// before launch cuts[k] - 1 (k >= 1) both field buffers of every shot are
// saved as checkpoint k - 1.  Adjoint: segments k = last .. 0, each a replay
// of launches cuts[k] - 1 .. cuts[k+1] - 1 from checkpoint k - 1 (segment 0
// from the initial state) on separate fields, storing the snapshots of times
// cuts[k] - 1 .. cuts[k+1] into the replay window, then the adjoint launches
// whose imaging times fall in [cuts[k], cuts[k+1]).  The replay repeats the
// forward launches exactly, so the gradient equals the stored-snapshot one.
static long long capture_checkpointed(fwi2d_ctx *ctx, Plan &P, bool adj, cudaStream_t cst)
{
    const ModelDev md = ctx->M.dev();
    const int nshots = (int)P.shots.size();
    const int ncomp = P.kind == KIND_ACOUSTIC ? 1 : 2;
    const int nt = P.nt_max, nseg = (int)P.cuts.size() - 1;
    long long n = 0;
    if (!adj) {
        const ShotDev *shots = P.d_shots_f.as<ShotDev>();
        int flags = STEP_EXTRACT;
        if (P.par.snapshot_precision != FWI2D_SNAP_FP32) flags |= STEP_AMAX;
        int kn = 1;
        for (int it = 0; it < nt - 1; it++) {
            if (kn < nseg && it == P.cuts[kn] - 1) {
                launch_checkpoint(shots, nshots, ncomp, kn - 1, false, cst);
                n++;
                kn++;
            }
            n += launch_step(ctx, P, shots, md, it, flags, cst);
        }
        launch_finalize(shots, nshots, P.C, ncomp, STEP_EXTRACT, cst);
        return n + 1;
    }
    // acoustic imaging at launch it uses time nt-1-it, the elastic one nt-2-it
    const int a = P.kind == KIND_ACOUSTIC ? 1 : 0;
    const ShotDev *last_adj = nullptr;
    int nadj = 0;   // adjoint launches so far (compensated accumulation windows)
    for (int k = nseg - 1; k >= 0; k--) {
        const ShotDev *rs = P.d_shots_r.as<ShotDev>() + (size_t)k * nshots;
        const ShotDev *as = P.d_shots_c.as<ShotDev>() + (size_t)k * nshots;
        if (k == 0) {
            for (auto &S : P.shots) {
                CK(cudaMemsetAsync(S->r0.p, 0, S->r0.n, cst));
                CK(cudaMemsetAsync(S->r1.p, 0, S->r1.n, cst));
            }
            launch_init_state(rs, nshots, P.d_icells[0].as<InitCell>(), P.d_ioff[0].as<int>(),
                              P.d_iidx[0].as<int>(), cst);
        } else {
            launch_checkpoint(rs, nshots, ncomp, k - 1, true, cst);
        }
        n++;
        const int t0 = k == 0 ? 0 : P.cuts[k] - 1, t1 = P.cuts[k + 1];
        for (int it = t0; it < t1; it++) n += launch_step(ctx, P, rs, md, it, STEP_STORE, cst);
        launch_finalize(rs, nshots, P.C, ncomp, STEP_STORE, cst, t1);
        n++;
        const int lo = k == nseg - 1 ? 0 : nt - 1 - P.cuts[k + 1] + a;
        const int hi = k == 0 ? nt - 2 : nt - 2 - P.cuts[k] + a;
        for (int it = lo; it <= hi; it++) {
            n += launch_step(ctx, P, as, md, it, STEP_GRAD, cst);
            n += grad_flush(P, P.all, ++nadj, false, cst);
        }
        last_adj = as;
    }
    if (P.kind == KIND_ACOUSTIC) {
        launch_acoustic_final_grad(last_adj, nshots, md, P.C, P.dtg, cst);
        n++;
    }
    return n;
}

// Capture one pass as a CUDA graph: mode 0 the forward of every shot without
// snapshots; mode 1 the forward with snapshots and mode 2 the adjoint of the
// shots of wave `w`.
static void capture(fwi2d_ctx *ctx, Plan &P, int mode, int w = 0)
{
    const ModelState &M = ctx->M;
    const bool adj = mode == 2;
    const bool store = mode == 1;
    const Plan::Wave &R = mode == 0 ? P.all : P.waves[w];
    cudaGraph_t g;
    // graphs are captured on the context's own stream and may be launched on any stream
    cudaStream_t cst = ctx->own;
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaStreamBeginCapture(cst, cudaStreamCaptureModeThreadLocal));
    long long n = 0;
    for (int s = R.s0; s < R.s1; s++) {
        ShotPlan *S = P.shots[s].get();
        CK(cudaMemsetAsync(S->u0.p, 0, S->u0.n, cst));
        CK(cudaMemsetAsync(S->u1.p, 0, S->u1.n, cst));
        if (adj) CK(cudaMemsetAsync(S->grad.p, 0, S->grad.n, cst));
        if (adj && S->gcomp.p) CK(cudaMemsetAsync(S->gcomp.p, 0, S->gcomp.n, cst));
        if (store && S->amax.p) CK(cudaMemsetAsync(S->amax.p, 0, S->amax.n, cst));
        if (P.ae) {
            CK(cudaMemsetAsync(S->fluid->u0.p, 0, S->fluid->u0.n, cst));
            CK(cudaMemsetAsync(S->fluid->u1.p, 0, S->fluid->u1.n, cst));
        }
    }
    // per-shot kernels take the wave's run of the shot tables; the step
    // kernels take the whole tables (their units carry the shot numbers)
    const ShotDev *shots = (adj ? P.d_shots_a : P.d_shots_f).as<ShotDev>();
    const ShotDev *wshots = P.ae ? (adj ? P.d_wshots_a : P.d_wshots_f).as<ShotDev>() : nullptr;
    const int nshots = R.s1 - R.s0;
    const int im = adj ? 1 : 0;
    // acoustic-elastic: the initial injection goes to the fluid layer when the
    // source is in the water, else to the elastic grid, in both directions
    // (we_op.cpp:2220-2236)
    if (P.ae && P.ae_src_fluid)
        launch_init_state(wshots + R.s0, nshots, P.d_wicells[im].as<InitCell>(), P.d_wioff[im].as<int>() + R.s0,
                          P.d_wiidx[im].as<int>(), cst);
    else
        launch_init_state(shots + R.s0, nshots, P.d_icells[im].as<InitCell>(), P.d_ioff[im].as<int>() + R.s0,
                          P.d_iidx[im].as<int>(), cst);
    n++;
    int flags = 0;
    if (adj) flags = STEP_GRAD;
    else {
        flags = STEP_EXTRACT;
        if (store) {
            flags |= STEP_STORE;
            if (P.par.snapshot_precision != FWI2D_SNAP_FP32) flags |= STEP_AMAX;
        }
    }
    const ModelDev md = M.dev();
    const int ncomp = P.kind == KIND_ACOUSTIC ? 1 : 2;
    if (P.ckpt > 0 && (store || adj)) {
        n += capture_checkpointed(ctx, P, adj, cst);
    } else {
        for (int it = 0; it < R.nt_max - 1; it++) {
            n += launch_step(ctx, P, shots, md, it, flags, cst, &R);
            if (adj) n += grad_flush(P, R, it + 1, false, cst);
        }
        if (!adj) {
            launch_finalize(shots + R.s0, nshots, P.C, ncomp, STEP_EXTRACT | (store ? STEP_STORE : 0), cst);
            n++;
            if (P.ae) {
                launch_finalize(wshots + R.s0, nshots, P.Cw, 1, STEP_EXTRACT, cst);
                n++;
            }
        } else if (P.kind == KIND_ACOUSTIC) {
            // snapshot 0 with the last adjoint field
            launch_acoustic_final_grad(shots + R.s0, nshots, md, P.C, P.dtg, cst);
            n++;
        }
    }
    if (adj) n += grad_flush(P, R, 0, true, cst);
    CK(cudaGetLastError());
    CK(cudaStreamEndCapture(cst, &g));
    cudaGraphExec_t ge;
    cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    if (mode == 0) {
        P.graph[0] = ge;
        P.launches[0] = n;
    } else {
        P.waves[w].graph[mode - 1] = ge;
        P.waves[w].launches[mode - 1] = n;
    }
}

static Plan &need_plan(fwi2d_ctx *ctx)
{
    if (!ctx->plan) throw Error(FWI2D_ERR_STATE, "fwi2d_set_shots must be called first");
    return *ctx->plan;
}

// traces: concatenated per-shot blocks [rows][nt]
static void upload_traces(fwi2d_ctx *ctx, const float *traces, bool adjoint)
{
    Plan &P = need_plan(ctx);
    REQ(traces != nullptr, "null trace array");
    set_device(ctx);
    size_t maxn = 0;
    for (auto &S : P.shots) maxn = std::max(maxn, (size_t)S->nt * (adjoint ? S->nrcv_rows : S->nsrc_rows));
    if (P.d_stage.n < maxn * sizeof(float)) P.d_stage.alloc(maxn * sizeof(float));
    std::vector<const float *> blocks;
    const float *p = traces;
    for (auto &S : P.shots) {
        const int rows = adjoint ? S->nrcv_rows : S->nsrc_rows;
        const size_t n = (size_t)rows * S->nt;
        for (size_t i = 0; i < n; i++)
            if (!std::isfinite(p[i])) throw Error(FWI2D_ERR_ARG, "trace array holds a non-finite value");
        // the staging buffer is reused by the next shot in stream order
        CK(cudaMemcpyAsync(P.d_stage.p, p, n * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
        launch_to_time_major(P.d_stage.as<float>(), (adjoint ? S->src_a : S->src_f).as<float>(), rows, S->nt, ctx->st);
        CK(cudaGetLastError());
        blocks.push_back(p);
        p += n;
    }
    CK(cudaStreamSynchronize(ctx->st));   // the caller's traces may be reused on return
}

// Sources on the data axis (fwi2d_set_data_axis): concatenated per-shot
// blocks [rows][nd], resampled to the propagation axis as apply_forward does
// (we_op.cpp:953-957: sinc or linear interpolation, no scaling).
static void upload_sources_axis(fwi2d_ctx *ctx, const float *traces)
{
    Plan &P = need_plan(ctx);
    REQ(traces != nullptr, "null trace array");
    set_device(ctx);
    size_t maxd = 1, maxp = 1;
    for (size_t k = 0; k < P.shots.size(); k++) {
        maxd = std::max(maxd, (size_t)P.shots[k]->nsrc_rows * P.nd[k]);
        maxp = std::max(maxp, (size_t)P.shots[k]->nsrc_rows * P.shots[k]->nt);
    }
    if (P.d_stage.n < maxd * sizeof(float)) P.d_stage.alloc(maxd * sizeof(float));
    if (P.d_rs1.n < maxp * sizeof(float)) P.d_rs1.alloc(maxp * sizeof(float));
    const float *p = traces;
    for (size_t k = 0; k < P.shots.size(); k++) {
        ShotPlan &S = *P.shots[k];
        const int rows = S.nsrc_rows, nd = P.nd[k];
        const size_t n = (size_t)rows * nd;
        for (size_t i = 0; i < n; i++)
            if (!std::isfinite(p[i])) throw Error(FWI2D_ERR_ARG, "trace array holds a non-finite value");
        if (rows > 0) {
            CK(cudaMemcpyAsync(P.d_stage.p, p, n * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
            k_resample_fwd<<<dim3((S.nt + 127) / 128, rows), 128, 0, ctx->st>>>(
                P.d_stage.as<float>(), P.d_rs1.as<float>(), nd, P.dd, S.nt, P.par.dt, P.rs_hl, P.rs_linear);
            launch_to_time_major(P.d_rs1.as<float>(), S.src_f.as<float>(), rows, S.nt, ctx->st);
            CK(cudaGetLastError());
        }
        p += n;
    }
    CK(cudaStreamSynchronize(ctx->st));   // the caller's traces may be reused on return
}

// One pass of wave w: the forward with snapshots, or the adjoint, which adds
// the wave's shot gradients onto the model grid (wave 0 clears it first).
static void run_wave(fwi2d_ctx *ctx, Plan &P, int w, bool adjoint)
{
    Plan::Wave &W = P.waves[w];
    const int mode = adjoint ? 2 : 1;
    if (!W.graph[mode - 1]) capture(ctx, P, mode, w);
    const int e = adjoint ? 1 : 0;
    if (!W.ev[e][0]) {
        CK(cudaEventCreate(&W.ev[e][0]));
        CK(cudaEventCreate(&W.ev[e][1]));
    }
    CK(cudaEventRecord(W.ev[e][0], ctx->st));
    CK(cudaGraphLaunch(W.graph[mode - 1], ctx->st));
    CK(cudaEventRecord(W.ev[e][1], ctx->st));
    P.timed[e] = true;
    if (!adjoint) P.fwd_waves = true;
    queue_timeout_check(ctx, P);
    if (adjoint) {
        if (w == 0) CK(cudaMemsetAsync(P.d_grad_full.p, 0, P.d_grad_full.n, ctx->st));
        for (int s = W.s0; s < W.s1; s++) {
            const ShotPlan &S = *P.shots[s];
            launch_add_subgrid(P.d_grad_full.as<float>(), S.grad.as<float>(), P.ncompg, S.x0, S.nx, ctx->M.ldz,
                               (long long)ctx->M.nx * ctx->M.ldz, ctx->st);
        }
        CK(cudaGetLastError());
    }
}

static void run(fwi2d_ctx *ctx, bool adjoint, bool store)
{
    Plan &P = need_plan(ctx);
    set_device(ctx);
    if (adjoint) {
        if (!P.have_snapshots || !P.snapshots_valid)
            throw Error(FWI2D_ERR_STATE, "the adjoint needs a forward pass that stored snapshots (sub > 0)");
    }
    if (store && !P.have_snapshots) throw Error(FWI2D_ERR_ARG, "snapshots requested with sub = 0");
    if (adjoint || store) {
        if (P.waves.size() != 1)
            throw Error(FWI2D_ERR_UNSUPPORTED,
                        "the snapshots of this plan's shots do not fit the device together: the plan runs in " +
                            std::to_string(P.waves.size()) +
                            " waves, which fwi2d_fwi_gradient drives (forward and adjoint of each wave in turn)");
        run_wave(ctx, P, 0, adjoint);
        if (store) P.snapshots_valid = true;
        return;
    }
    if (!P.graph[0]) capture(ctx, P, 0);
    if (!P.ev[0][0]) {
        CK(cudaEventCreate(&P.ev[0][0]));
        CK(cudaEventCreate(&P.ev[0][1]));
    }
    CK(cudaEventRecord(P.ev[0][0], ctx->st));
    CK(cudaGraphLaunch(P.graph[0], ctx->st));
    CK(cudaEventRecord(P.ev[0][1], ctx->st));
    P.timed[0] = true;
    P.fwd_waves = false;
    queue_timeout_check(ctx, P);
}

// Device time of the last forward (e = 0) or adjoint (e = 1) pass, summed
// over the waves; -1 if none ran.
static float pass_ms(Plan &P, int e)
{
    if (!P.timed[e]) return -1.f;
    float total = 0.f;
    if (e == 0 && !P.fwd_waves) {
        CK(cudaEventSynchronize(P.ev[0][1]));
        CK(cudaEventElapsedTime(&total, P.ev[0][0], P.ev[0][1]));
        return total;
    }
    for (auto &W : P.waves) {
        if (!W.ev[e][0]) continue;
        float ms = 0.f;
        CK(cudaEventSynchronize(W.ev[e][1]));
        CK(cudaEventElapsedTime(&ms, W.ev[e][0], W.ev[e][1]));
        total += ms;
    }
    return total;
}

static void download_rcv(fwi2d_ctx *ctx, float *rcv)
{
    Plan &P = need_plan(ctx);
    size_t maxn = 0;
    for (auto &S : P.shots) maxn = std::max(maxn, (size_t)S->nt * S->nrcv_rows);
    if (P.d_stage.n < maxn * sizeof(float)) P.d_stage.alloc(maxn * sizeof(float));
    float *p = rcv;
    for (auto &S : P.shots) {
        const size_t n = (size_t)S->nrcv_rows * S->nt;
        launch_from_time_major(S->rcv_f.as<float>(), P.d_stage.as<float>(), S->nrcv_rows, S->nt, ctx->st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(p, P.d_stage.p, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        p += n;
    }
    check_timeout(ctx);
}

static void download_grad(fwi2d_ctx *ctx, float *grad)
{
    Plan &P = need_plan(ctx);
    const ModelState &M = ctx->M;
    const size_t n = (size_t)P.ncompg * M.nx * M.nz;
    if (P.d_stage.n < n * sizeof(float)) P.d_stage.alloc(n * sizeof(float));
    k_unpitch<<<592, 256, 0, ctx->st>>>(P.d_grad_full.as<float>(), P.d_stage.as<float>(), (long long)P.ncompg * M.nx,
                                        M.nz, M.ldz);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(grad, P.d_stage.p, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    check_timeout(ctx);
}


// ---------------------------------------------------------------------------
// FWI gradient pieces on the device (optimization.hpp:590-951 and the
// adjoint-source preparation of we_op.cpp:1108-1134)
// ---------------------------------------------------------------------------

// Per trace sample (row r, time t; one thread per row and chunk of kResChunk
// samples): synthetic data (Dt of the extracted displacement when
// seismotype = 1, misc.cpp:71-84), residual r = syn - obs, the chunk's part
// of the trace misfit sum(r^2) - (r_0^2 + r_{nt-1}^2)/2 (Neumaier summation),
// and the adjoint source
//   q[t] = -r[nt-1-t]  (Ht^-1 of the caller's Ht r, reversed, scaled by -1),
//   then Dt^T (misc.cpp:85-94) when seismotype = 1.
// Acoustic-elastic data (rows [0, neg_rows) hold the fluid traces): with
// seismotype = 1 the fluid synthetic is -Dt of the extracted potential, and
// its adjoint source -Dt^T (we_op.cpp:1033-1040, :1117-1124).
// k_misfit_rows adds the chunk partials of each trace in double.
constexpr int kResChunk = 64;

__global__ void k_residual(const float *__restrict__ u, const float *__restrict__ obs, float *__restrict__ adj,
                           float *__restrict__ syn_out, float2 *__restrict__ part, int nt, int rows, float dt,
                           int seismotype, int neg_rows)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int t0 = blockIdx.y * kResChunk, t1 = min(nt, t0 + kResChunk);
    const bool neg = seismotype && r < neg_rows;
    auto U = [&](int t) { return u[(long long)t * rows + r]; };
    auto syn = [&](int t) -> float {
        if (!seismotype) return U(t);
        float v;
        if (t == 0) v = (U(1) - U(0)) / dt;
        else if (t == nt - 1) v = (U(nt - 1) - U(nt - 2)) / dt;
        else v = (U(t + 1) - U(t - 1)) / (2 * dt);
        return neg ? -v : v;
    };
    auto res = [&](int t) { return syn(t) - obs[(long long)t * rows + r]; };
    float sum = 0.f, comp = 0.f;
    for (int t = t0; t < t1; t++) {
        const float rv = res(t);
        float term = rv * rv;
        if (t == 0 || t == nt - 1) term = 0.5f * term;
        const float y = sum + term;
        if (fabsf(sum) >= fabsf(term)) comp += (sum - y) + term;
        else comp += (term - y) + sum;
        sum = y;
        if (syn_out) syn_out[(long long)t * rows + r] = syn(t);
    }
    part[(long long)blockIdx.y * rows + r] = make_float2(sum, comp);
    auto q = [&](int t) { return -res(nt - 1 - t); };
    for (int t = t0; t < t1; t++) {
        float a;
        if (!seismotype) a = q(t);
        else if (t == 0) a = (q(1) + q(0)) / dt;
        else if (t == nt - 1) a = (-q(nt - 1) - q(nt - 2)) / dt;
        else a = (q(t + 1) - q(t - 1)) / (2 * dt);
        adj[(long long)t * rows + r] = neg ? -a : a;
    }
}

__global__ void k_misfit_rows(const float2 *__restrict__ part, double *__restrict__ misfit, int rows, int nchunk)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double m = 0.0;
    for (int c = 0; c < nchunk; c++) {
        const float2 p = part[(long long)c * rows + r];
        m += (double)p.x + (double)p.y;
    }
    misfit[r] = m;
}

// H quadrature (spatial_operators.cpp:6-98) and the chain rule from
// (lambda, mu, rho) to (vp, vs, rho), or from (K, 1/rho) to (vp, rho) for the
// acoustic propagator (we_op.cpp:1193-1228), in place on the pitched
// model-grid gradient.  Acoustic: lam = K, mu = 1/rho, rho unused.
__global__ void k_quadrature_chain(float *__restrict__ g, const float *__restrict__ lam, const float *__restrict__ mu,
                                   const float *__restrict__ rho, int nx, int nz, int ldz, float dx, float dz,
                                   float h0, float h1, float h2, float h3, int acoustic)
{
    const long long n = (long long)nx * ldz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i / ldz), iz = (int)(i - (long long)ix * ldz);
        if (iz >= nz) continue;
        const float hc[4] = {h0, h1, h2, h3};
        const float wz = iz < 4 ? hc[iz] : (iz >= nz - 4 ? hc[nz - 1 - iz] : 1.f);
        const float wx = ix < 4 ? hc[ix] : (ix >= nx - 4 ? hc[nx - 1 - ix] : 1.f);
        float g0 = g[i], g1 = g[n + i], g2 = acoustic ? 0.f : g[2 * n + i];
        // applyHz then applyHx on each component
        if (iz < 4 || iz >= nz - 4) { g0 = g0 * wz * dz; g1 = g1 * wz * dz; g2 = g2 * wz * dz; }
        else { g0 = g0 * dz; g1 = g1 * dz; g2 = g2 * dz; }
        if (ix < 4 || ix >= nx - 4) { g0 = g0 * wx * dx; g1 = g1 * wx * dx; g2 = g2 * wx * dx; }
        else { g0 = g0 * dx; g1 = g1 * dx; g2 = g2 * dx; }
        if (acoustic) {
            const float K = lam[i], ir = mu[i];
            g[n + i] = ir * K * g0 - ir * ir * g1;                            // rho
            g[i] = (float)(2 * sqrt((double)(K / ir)) * (double)g0);          // vp
            continue;
        }
        const float l = lam[i], m = mu[i], r = rho[i];
        const float n2 = (l / r) * g0 + (m / r) * g1 + g2;
        const float n1 = (float)(2 * sqrt((double)(m * r)) * (double)(g1 - 2 * g0));
        const float n0 = (float)(2 * sqrt((double)(r * (l + 2 * m))) * (double)g0);
        g[i] = n0;
        g[n + i] = n1;
        g[2 * n + i] = n2;
    }
}

static void update_model(fwi2d_ctx *ctx, const float *model)
{
    ModelState &M = ctx->M;
    if (M.kind < 0) throw Error(FWI2D_ERR_STATE, "fwi2d_set_model must be called first");
    REQ(model != nullptr, "null model");
    set_device(ctx);
    upload_model_values(ctx, model);
    if (!ctx->plan) return;
    Plan &P = *ctx->plan;
    const fwi2d_params &p = P.par;
    for (auto &S : P.shots) {
        std::vector<float> den;
        if (M.kind == KIND_ACOUSTIC) {
            const float *K = M.hp(0) + (size_t)S->x0 * M.nz, *irho = M.hp(1) + (size_t)S->x0 * M.nz;
            acoustic_scale_divisors(S->nx, M.nz, M.dx, M.dz, p.dt, K, irho, M.nz, p.bc_top == 2, p.bc_bottom == 2,
                                    p.bc_left == 2, p.bc_right == 2, den);
        } else {
            const float *lam = M.hp(0) + (size_t)S->x0 * M.nz, *mu = M.hp(1) + (size_t)S->x0 * M.nz,
                        *rho = M.hp(2) + (size_t)S->x0 * M.nz;
            const float *eps = M.kind == KIND_VTI ? M.hp(4) + (size_t)S->x0 * M.nz : nullptr;
            elastic_scale_divisors(S->nx, M.nz, M.dx, M.dz, p.dt, lam, mu, rho, eps, M.nz, !P.ae && p.bc_top == 2,
                                   p.bc_bottom == 2, p.bc_left == 2, p.bc_right == 2, den);
        }
        S->den.upload(den, ctx->st);
    }
    init_factors(M, P);
    upload_init_cells(P, ctx->st);
    CK(cudaStreamSynchronize(ctx->st));
}

// One FWI gradient on the device: forward with snapshots, residual against
// the resident observed data, adjoint sources, adjoint with the imaging
// condition, quadrature and chain rule.  Leaves the model-space gradient in
// d_grad_full and the per-trace misfit terms in d_misfit.
static void fwi_gradient(fwi2d_ctx *ctx, int seismotype, bool chain)
{
    Plan &P = need_plan(ctx);
    REQ(P.d_obs.p != nullptr, "no observed data (fwi2d_set_observed)");
    set_device(ctx);
    REQ(P.have_snapshots, "the FWI gradient needs snapshots (sub > 0)");
    const int nsh = (int)P.shots.size();
    size_t rows_total = 0;
    for (auto &S : P.shots) rows_total += S->nrcv_rows;
    P.d_misfit.ensure(std::max<size_t>(rows_total, 1) * sizeof(double));
    size_t part_max = 1;
    for (auto &S : P.shots)
        part_max = std::max(part_max, (size_t)((S->nt + kResChunk - 1) / kResChunk) * S->nrcv_rows);
    // the shots share one partial buffer: their kernels run in stream order and
    // each shot reduces its partials before the next shot writes them
    P.d_part.ensure(part_max * sizeof(float2));
    // observed-data and misfit-row offsets of every shot
    std::vector<size_t> obs_off(nsh + 1, 0), row_off(nsh + 1, 0);
    for (int k = 0; k < nsh; k++) {
        const ShotPlan &S = *P.shots[k];
        obs_off[k + 1] = obs_off[k] + (size_t)(P.dd > 0.f ? P.nd[k] : S.nt) * S.nrcv_rows;
        row_off[k + 1] = row_off[k] + S.nrcv_rows;
    }
    if (P.dd > 0.f) {
        size_t mx = 1, pm = 1;
        for (size_t k = 0; k < P.shots.size(); k++) {
            mx = std::max(mx, (size_t)P.shots[k]->nrcv_rows * std::max(P.shots[k]->nt, P.nd[k]));
            pm = std::max(pm, (size_t)((P.nd[k] + kRsChunk - 1) / kRsChunk) * P.shots[k]->nrcv_rows);
        }
        P.d_rs0.ensure(std::max(P.d_rs0.n, mx * sizeof(float)));
        P.d_rs1.ensure(std::max(P.d_rs1.n, mx * sizeof(float)));
        P.d_part.ensure(std::max(P.d_part.n, pm * sizeof(float2)));
    }
    // residual, misfit rows and adjoint sources of shot k (after its forward)
    auto residual = [&](int k) {
        ShotPlan &S = *P.shots[k];
        if (P.dd > 0.f) {
            // data on their own axis: receivers -> alpha Dt -> adjoint resampling to
            // the data axis; residual, misfit, Ht weighting there; resampling back,
            // Ht^-1, reversal, -alpha, Dt^T (we_op.cpp:1030-1054, 1100-1124)
            const float alpha = P.par.dt / P.dd;
            const int rows = S.nrcv_rows, nt = S.nt, nd = P.nd[k];
            const int neg = P.ae ? S.nr : 0;
            const int nchunk = (nd + kRsChunk - 1) / kRsChunk;
            float *r0 = P.d_rs0.as<float>(), *r1 = P.d_rs1.as<float>();
            k_rcv_to_rate<<<dim3((rows + 127) / 128, nt), 128, 0, ctx->st>>>(S.rcv_f.as<float>(), r0, rows, nt,
                                                                            P.par.dt, alpha, seismotype, neg);
            k_resample_adj<<<dim3((nd + 127) / 128, rows), 128, 0, ctx->st>>>(r0, r1, nd, P.dd, nt, P.par.dt,
                                                                             P.rs_hl, P.rs_linear);
            k_residual_axis<<<dim3((rows + 127) / 128, nchunk), 128, 0, ctx->st>>>(
                r1, P.d_obs.as<float>() + obs_off[k], r0, P.d_part.as<float2>(), rows, nd, P.dd);
            k_misfit_rows<<<(rows + 127) / 128, 128, 0, ctx->st>>>(P.d_part.as<float2>(),
                                                                  P.d_misfit.as<double>() + row_off[k], rows, nchunk);
            k_resample_fwd<<<dim3((nt + 127) / 128, rows), 128, 0, ctx->st>>>(r0, r1, nd, P.dd, nt, P.par.dt,
                                                                             P.rs_hl, P.rs_linear);
            k_adjoint_source_axis<<<dim3((rows + 127) / 128, nt), 128, 0, ctx->st>>>(
                r1, S.src_a.as<float>(), rows, nt, P.par.dt, alpha, seismotype, neg);
        } else {
            const int nchunk = (S.nt + kResChunk - 1) / kResChunk;
            dim3 grid((S.nrcv_rows + 127) / 128, nchunk);
            k_residual<<<grid, 128, 0, ctx->st>>>(S.rcv_f.as<float>(), P.d_obs.as<float>() + obs_off[k],
                                                  S.src_a.as<float>(), nullptr, P.d_part.as<float2>(), S.nt,
                                                  S.nrcv_rows, P.par.dt, seismotype, P.ae ? S.nr : 0);
            k_misfit_rows<<<(S.nrcv_rows + 127) / 128, 128, 0, ctx->st>>>(
                P.d_part.as<float2>(), P.d_misfit.as<double>() + row_off[k], S.nrcv_rows, nchunk);
        }
        CK(cudaGetLastError());
    };
    // wave by wave: forward with snapshots, residuals, adjoint (the waves
    // share the snapshot store; one wave when every shot fits)
    for (int w = 0; w < (int)P.waves.size(); w++) {
        run_wave(ctx, P, w, false);
        for (int k = P.waves[w].s0; k < P.waves[w].s1; k++) residual(k);
        run_wave(ctx, P, w, true);
    }
    P.snapshots_valid = P.waves.size() == 1;
    if (chain) {
        const ModelState &M = ctx->M;
        const SbpTables &t = sbp_tables();
        k_quadrature_chain<<<592, 256, 0, ctx->st>>>(P.d_grad_full.as<float>(), M.p0.as<float>(), M.p1.as<float>(),
                                                     M.p2.as<float>(), M.nx, M.nz, M.ldz, M.dx, M.dz, t.hc[0], t.hc[1],
                                                     t.hc[2], t.hc[3], P.kind == KIND_ACOUSTIC ? 1 : 0);
        CK(cudaGetLastError());
    }
}

static void set_observed(fwi2d_ctx *ctx, const float *obs)
{
    Plan &P = need_plan(ctx);
    REQ(obs != nullptr, "null observed data");
    set_device(ctx);
    size_t total = 0, maxn = 0;
    for (size_t k = 0; k < P.shots.size(); k++) {
        const size_t n = (size_t)(P.dd > 0.f ? P.nd[k] : P.shots[k]->nt) * P.shots[k]->nrcv_rows;
        total += n;
        maxn = std::max(maxn, n);
    }
    P.d_obs.ensure(std::max<size_t>(total, 1) * sizeof(float));
    if (P.dd > 0.f) {
        // data-axis observed data stay row-major [rows][nd] per shot
        CK(cudaMemcpyAsync(P.d_obs.p, obs, total * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        return;
    }
    if (P.d_stage.n < maxn * sizeof(float)) P.d_stage.alloc(maxn * sizeof(float));
    size_t off = 0;
    for (auto &S : P.shots) {
        const size_t n = (size_t)S->nt * S->nrcv_rows;
        CK(cudaMemcpyAsync(P.d_stage.p, obs + off, n * sizeof(float), cudaMemcpyHostToDevice, ctx->st));
        launch_to_time_major(P.d_stage.as<float>(), P.d_obs.as<float>() + off, S->nrcv_rows, S->nt, ctx->st);
        CK(cudaGetLastError());
        off += n;
    }
    CK(cudaStreamSynchronize(ctx->st));
}

// Data time axis of the FWI gradient (the time axis of the reference's
// source and data cubes, analyzeModel, we_op.cpp:436-472): nd[k] samples at
// dd for shot k, resampled to the plan's dt <= dd with the sinc (half length
// hl) or linear resampler.  Each shot's nt must be the propagation length the
// reference derives, round((nd - 1) dd / dt) + 1.  dd <= 0 returns to data on
// the propagation axis.  The resident observed data are dropped.
static void set_data_axis(fwi2d_ctx *ctx, float dd, int method, int hl, const int *nd)
{
    Plan &P = need_plan(ctx);
    P.d_obs.release();
    if (dd <= 0.f) {
        P.dd = 0.f;
        P.nd.clear();
        return;
    }
    REQ(method == FWI2D_RESAMPLE_SINC || method == FWI2D_RESAMPLE_LINEAR, "unknown resampling method");
    REQ(method == FWI2D_RESAMPLE_LINEAR || hl > 0, "the sinc half length must be positive");
    REQ(nd != nullptr, "null data sample counts");
    REQ(P.par.dt <= dd, "the propagation step must not exceed the data step");
    std::vector<int> v(nd, nd + P.shots.size());
    for (size_t k = 0; k < P.shots.size(); k++) {
        REQ(v[k] >= 2, "a shot needs at least two data samples");
        // the trace kernels put rows or samples on grid.y
        REQ(P.shots[k]->nt <= 65535 && v[k] <= 65535 && P.shots[k]->nrcv_rows <= 65535 &&
                P.shots[k]->nsrc_rows <= 65535,
            "data-axis resampling supports at most 65535 samples and trace rows per shot");
        const float tmax = (v[k] - 1) * dd;
        const int nt = (int)std::round(tmax / P.par.dt) + 1;
        if (nt != P.shots[k]->nt)
            throw Error(FWI2D_ERR_ARG, "shot " + std::to_string(k) + ": nt must be round((nd - 1) dd / dt) + 1 = " +
                                           std::to_string(nt));
    }
    P.dd = dd;
    P.rs_linear = method == FWI2D_RESAMPLE_LINEAR;
    P.rs_hl = hl;
    P.nd = v;
}

static double read_misfit(fwi2d_ctx *ctx)
{
    Plan &P = need_plan(ctx);
    size_t rows_total = 0;
    for (auto &S : P.shots) rows_total += S->nrcv_rows;
    std::vector<double> m(rows_total);
    CK(cudaMemcpyAsync(m.data(), P.d_misfit.p, rows_total * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    check_timeout(ctx);
    double f = 0.0;
    for (double v : m) f += v;
    return 0.5 * (double)(P.dd > 0.f ? P.dd : P.par.dt) * f;
}

// Host snapshots [nslot][ncomp][nx][nz] (fp32) -> the device store of shot 0.
static void load_host_snapshots(fwi2d_ctx *ctx, const float *full)
{
    Plan &P = need_plan(ctx);
    REQ(P.par.snapshot_precision == FWI2D_SNAP_FP32, "host snapshots are fp32");
    ShotPlan &S = *P.shots[0];
    const ModelState &M = ctx->M;
    const size_t rows = (size_t)S.ncomp * S.nx;
    const size_t slot_in = rows * M.nz, slot_out = rows * M.ldz;
    if (P.d_stage.n < slot_in * sizeof(float)) P.d_stage.alloc(slot_in * sizeof(float));
    for (int k = 0; k < S.nslot; k++) {
        CK(cudaMemcpyAsync(P.d_stage.p, full + (size_t)k * slot_in, slot_in * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->st));
        k_pitch<<<592, 256, 0, ctx->st>>>(P.d_stage.as<float>(), (float *)S.snap_base + (size_t)k * slot_out,
                                          (long long)rows, M.nz, M.ldz);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(ctx->st));
    P.snapshots_valid = true;
}

static void store_host_snapshots(fwi2d_ctx *ctx, float *full)
{
    Plan &P = need_plan(ctx);
    ShotPlan &S = *P.shots[0];
    const ModelState &M = ctx->M;
    const size_t rows = (size_t)S.ncomp * S.nx;
    const size_t slot_in = rows * M.ldz, slot_out = rows * M.nz;
    if (P.d_stage.n < slot_out * sizeof(float)) P.d_stage.alloc(slot_out * sizeof(float));
    // the reference writes slots it/sub for it in [0, nt-1]; later slots stay untouched
    const int written = (S.nt - 1) / P.C.sub + 1;
    for (int k = 0; k < std::min(written, S.nslot); k++) {
        k_unpitch<<<592, 256, 0, ctx->st>>>((const float *)S.snap_base + (size_t)k * slot_in, P.d_stage.as<float>(),
                                            (long long)rows, M.nz, M.ldz);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(full + (size_t)k * slot_out, P.d_stage.p, slot_out * sizeof(float), cudaMemcpyDeviceToHost,
                           ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
}

static fwi2d_ctx *thread_ctx(int device)
{
    static thread_local std::vector<std::unique_ptr<fwi2d_ctx, int (*)(fwi2d_ctx *)>> pool;
    for (auto &c : pool)
        if (c->device == device) return c.get();
    fwi2d_ctx *c = nullptr;
    int rc = fwi2d_ctx_create(device, &c);
    if (rc != FWI2D_OK) throw Error(rc, g_err);
    pool.emplace_back(c, fwi2d_ctx_destroy);
    return c;
}

}  // namespace fwi2d

// ===========================================================================
// C ABI
// ===========================================================================
using namespace fwi2d;

#define ABI_TRY try {
#define ABI_END                                   \
    }                                             \
    catch (const Error &e)                        \
    {                                             \
        g_err = e.what();                         \
        return e.code;                            \
    }                                             \
    catch (const std::bad_alloc &)                \
    {                                             \
        g_err = "host memory exhausted";          \
        return FWI2D_ERR_OOM;                     \
    }                                             \
    catch (const std::exception &e)               \
    {                                             \
        g_err = e.what();                         \
        return FWI2D_ERR_ARG;                     \
    }                                             \
    return FWI2D_OK;

extern "C" {

const char *fwi2d_last_error(void) { return g_err.c_str(); }

int fwi2d_version(void) { return 100; }

int fwi2d_injector_weights(int type, int ntr, const float *locx, const float *locz, int nx, int nz, float dx,
                           float dz, float ox, float oz, int *xind, int *zind, float *xw, float *zw)
{
    ABI_TRY
    REQ(type == FWI2D_INJ_DELTA || type == FWI2D_INJ_DDELTA, "unknown injector type");
    REQ(ntr >= 0 && nx >= 3 && nz >= 3 && dx > 0 && dz > 0, "invalid grid");
    REQ(ntr == 0 || (locx && locz && xind && zind && xw && zw), "null array");
    injector_weights(type, ntr, locx, locz, nx, nz, dx, dz, ox, oz, xind, zind, xw, zw);
    ABI_END
}

int fwi2d_dipole_weights(int ntr, const float *locx, const float *locz, const float *dip, float gl, int nx, int nz,
                         float dx, float dz, float ox, float oz, int *xind, int *zind, float *xw, float *zw)
{
    ABI_TRY
    REQ(ntr >= 0 && nx >= 3 && nz >= 3 && dx > 0 && dz > 0 && gl > 0, "invalid grid or gauge length");
    REQ(ntr == 0 || (locx && locz && dip && xind && zind && xw && zw), "null array");
    dipole_weights(ntr, locx, locz, dip, gl, nx, nz, dx, dz, ox, oz, xind, zind, xw, zw);
    ABI_END
}

int fwi2d_analyze_model(int npar, float *model, int nx, int nz, float dx, float dz, int data_nt, float data_dt,
                        fwi2d_model_check *check)
{
    ABI_TRY
    REQ(npar == 2 || npar == 3 || npar == 5, "the model must hold 2 (vp, rho), 3 (vp, vs, rho) or 5 parameters");
    REQ(model && check, "null argument");
    REQ(nx > 0 && nz > 0 && dx > 0 && dz > 0 && data_nt > 0 && data_dt > 0, "invalid grid or data axis");
    analyze_model(npar, model, nx, nz, dx, dz, data_nt, data_dt, *check);
    ABI_END
}

int fwi2d_ctx_create(int device, fwi2d_ctx **out)
{
    ABI_TRY
    REQ(out != nullptr, "null output pointer");
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    REQ(device >= 0 && device < n, "no such CUDA device");
    auto c = std::make_unique<fwi2d_ctx>();
    c->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking));
    // the band kernels' few CTAs are on the critical path of a step: their
    // streams take the highest priority, so that the block scheduler starts
    // them before the core launch fills the SMs
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    CK(cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_hi));
    CK(cudaStreamCreateWithPriority(&c->side2, cudaStreamNonBlocking, prio_hi));
    CK(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->join2, cudaEventDisableTiming));
    c->st = c->own;
    const SbpTables &t = sbp_tables();
    upload_sbp_tables(&t.b1[0][0], &t.b2[0][0][0], t.c2, t.c1, t.sc, t.hc);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    *out = c.release();
    ABI_END
}

int fwi2d_ctx_destroy(fwi2d_ctx *ctx)
{
    ABI_TRY
    if (!ctx) return FWI2D_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->st);
    ctx->plan.reset();
    cudaStreamDestroy(ctx->own);
    cudaStreamDestroy(ctx->side);
    cudaStreamDestroy(ctx->side2);
    cudaEventDestroy(ctx->fork);
    cudaEventDestroy(ctx->join);
    cudaEventDestroy(ctx->join2);
    delete ctx;
    ABI_END
}

int fwi2d_set_model(fwi2d_ctx *ctx, int kind, int nx, int nz, float dx, float dz, const float *model)
{
    ABI_TRY
    REQ(ctx, "null context");
    set_model(ctx, kind, nx, nz, dx, dz, model);
    ABI_END
}

int fwi2d_set_shots(fwi2d_ctx *ctx, const fwi2d_params *par, int nshots, const fwi2d_shot *shots)
{
    ABI_TRY
    REQ(ctx, "null context");
    set_shots(ctx, par, nshots, shots);
    ABI_END
}

int fwi2d_forward(fwi2d_ctx *ctx, const float *src, float *rcv, int store_snapshots)
{
    ABI_TRY
    REQ(ctx && rcv, "null argument");
    upload_traces(ctx, src, false);
    run(ctx, false, store_snapshots != 0);
    download_rcv(ctx, rcv);
    ABI_END
}

int fwi2d_adjoint(fwi2d_ctx *ctx, const float *adj, float *grad)
{
    ABI_TRY
    REQ(ctx && grad, "null argument");
    upload_traces(ctx, adj, true);
    run(ctx, true, false);
    download_grad(ctx, grad);
    ABI_END
}

int fwi2d_upload_traces(fwi2d_ctx *ctx, const float *traces, int adjoint)
{
    ABI_TRY
    REQ(ctx, "null context");
    upload_traces(ctx, traces, adjoint != 0);
    ABI_END
}

int fwi2d_run(fwi2d_ctx *ctx, int adjoint, int store_snapshots)
{
    ABI_TRY
    REQ(ctx, "null context");
    run(ctx, adjoint != 0, store_snapshots != 0);
    ABI_END
}

int fwi2d_sync(fwi2d_ctx *ctx)
{
    ABI_TRY
    REQ(ctx, "null context");
    set_device(ctx);
    CK(cudaStreamSynchronize(ctx->st));
    check_timeout(ctx);
    ABI_END
}

int fwi2d_snapshot(fwi2d_ctx *ctx, int shot, int slot, float *out)
{
    ABI_TRY
    REQ(ctx && out, "null argument");
    Plan &P = need_plan(ctx);
    REQ(shot >= 0 && shot < (int)P.shots.size(), "no such shot");
    ShotPlan &S = *P.shots[shot];
    REQ(P.have_snapshots && slot >= 0 && slot < S.nslot, "no such snapshot");
    REQ(P.ckpt == 0, "snapshots are recomputed segment by segment under checkpointing and are not kept");
    REQ(P.waves.size() == 1, "the plan runs its shots in waves that share one snapshot store");
    set_device(ctx);
    const ModelState &M = ctx->M;
    const size_t field = (size_t)S.ncomp * S.nx * M.ldz;
    const int prec = P.par.snapshot_precision;
    const size_t esz = prec == FWI2D_SNAP_FP32 ? 4 : 2;
    std::vector<unsigned char> raw(field * esz);
    CK(cudaMemcpyAsync(raw.data(), (const char *)S.snap_base + (size_t)slot * field * esz, field * esz,
                       cudaMemcpyDeviceToHost, ctx->st));
    unsigned amax = 0;
    if (prec != FWI2D_SNAP_FP32)
        CK(cudaMemcpyAsync(&amax, S.amax.as<unsigned>() + slot, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    float inv = 1.f;
    if (prec != FWI2D_SNAP_FP32) {
        float m;
        std::memcpy(&m, &amax, 4);
        if (m > 0.f) inv = 1.f / std::ldexp(1.f, 14 - (std::ilogb(m) + 1));
    }
    for (int c = 0; c < S.ncomp; c++)
        for (int ix = 0; ix < S.nx; ix++)
            for (int iz = 0; iz < M.nz; iz++) {
                const size_t i = ((size_t)c * S.nx + ix) * M.ldz + iz;
                float v;
                if (prec == FWI2D_SNAP_FP32) std::memcpy(&v, &raw[i * 4], 4);
                else {
                    unsigned short h;
                    std::memcpy(&h, &raw[i * 2], 2);
                    if (prec == FWI2D_SNAP_BF16) {
                        unsigned b = (unsigned)h << 16;
                        std::memcpy(&v, &b, 4);
                    } else {
                        // IEEE half -> float
                        const unsigned sgn = (h >> 15) & 1, ex = (h >> 10) & 31, man = h & 1023;
                        float f;
                        if (ex == 0) f = std::ldexp((float)man, -24);
                        else if (ex == 31) f = man ? NAN : INFINITY;
                        else f = std::ldexp((float)(man + 1024), (int)ex - 25);
                        v = sgn ? -f : f;
                    }
                    v *= inv;
                }
                out[((size_t)c * S.nx + ix) * M.nz + iz] = v;
            }
    ABI_END
}

int fwi2d_plan_info(fwi2d_ctx *ctx, long long *lf, long long *la, int *shape, long long *snap_bytes)
{
    ABI_TRY
    REQ(ctx, "null context");
    Plan &P = need_plan(ctx);
    const long long per = (P.march || P.framed || P.ae) ? 3 : 1;
    const long long nseg = P.ckpt > 0 ? (long long)P.cuts.size() - 1 : 0;
    const long long acf = P.kind == KIND_ACOUSTIC ? 1 : 0;
    // per wave -- forward: init, steps, last sample (+ checkpoint copies);
    // adjoint: init, steps, acoustic final imaging, per-shot scatter (+ replays:
    // restore, steps, last snapshot) and, with compensated accumulation, one
    // window flush per kCompWindow adjoint launches plus the final one
    long long f = 0, a = 0;
    for (const auto &W : P.waves) {
        const long long steps = W.nt_max - 1;
        f += steps * per + 2 + (P.ae ? 1 : 0) + (nseg > 0 ? nseg - 1 : 0);
        const long long flushes = P.par.compensated && P.par.sub > 0 ? steps / kCompWindow + 1 : 0;
        a += steps * per + 1 + acf + (W.s1 - W.s0) + (nseg > 0 ? (steps + nseg - 1) * per + 2 * nseg : 0) + flushes;
    }
    if (lf) *lf = f;
    if (la) *la = a;
    if (shape) *shape = P.shape;
    if (snap_bytes) *snap_bytes = P.snap_bytes;
    ABI_END
}

int fwi2d_plan_waves(fwi2d_ctx *ctx, int *nwaves, long long *snapshot_bytes_all)
{
    ABI_TRY
    REQ(ctx, "null context");
    Plan &P = need_plan(ctx);
    if (nwaves) *nwaves = (int)P.waves.size();
    if (snapshot_bytes_all) {
        long long b = 0;
        for (auto &S : P.shots) b += (long long)S->snap_need;
        *snapshot_bytes_all = b;
    }
    ABI_END
}

int fwi2d_set_stream(fwi2d_ctx *ctx, void *stream)
{
    ABI_TRY
    REQ(ctx, "null context");
    set_device(ctx);
    CK(cudaStreamSynchronize(ctx->st));
    ctx->st = stream ? (cudaStream_t)stream : ctx->own;
    ABI_END
}

int fwi2d_copy_gradient(fwi2d_ctx *ctx, float *dst_device)
{
    ABI_TRY
    REQ(ctx && dst_device, "null argument");
    Plan &P = need_plan(ctx);
    const ModelState &M = ctx->M;
    set_device(ctx);
    k_unpitch<<<592, 256, 0, ctx->st>>>(P.d_grad_full.as<float>(), dst_device, (long long)P.ncompg * M.nx, M.nz, M.ldz);
    CK(cudaGetLastError());
    ABI_END
}

int fwi2d_last_timing(fwi2d_ctx *ctx, float *forward_ms, float *adjoint_ms)
{
    ABI_TRY
    REQ(ctx, "null context");
    Plan &P = need_plan(ctx);
    set_device(ctx);
    float *out[2] = {forward_ms, adjoint_ms};
    for (int e = 0; e < 2; e++)
        if (out[e]) *out[e] = pass_ms(P, e);
    ABI_END
}

int fwi2d_tile_shape_count(void) { return shape_count(); }

int fwi2d_tile_shape(int index, int *tz, int *tx)
{
    ABI_TRY
    REQ(index >= 0 && index < shape_count() && tz && tx, "no such tile shape");
    if (index < elastic_tile_count()) elastic_tile_shape(index, tz, tx);
    else if (is_framed_shape(index)) elastic_tile_shape(framed_tile_shape(index), tz, tx);
    else {
        *tz = kMarchShapes[index - elastic_tile_count()].nth;
        *tx = kMarchShapes[index - elastic_tile_count()].lx;
    }
    ABI_END
}

int fwi2d_update_model(fwi2d_ctx *ctx, const float *model)
{
    ABI_TRY
    REQ(ctx, "null context");
    update_model(ctx, model);
    ABI_END
}

int fwi2d_set_data_axis(fwi2d_ctx *ctx, float dt_data, int method, int sinc_half_length, const int *nd)
{
    ABI_TRY
    REQ(ctx, "null context");
    set_device(ctx);
    set_data_axis(ctx, dt_data, method, sinc_half_length, nd);
    ABI_END
}

int fwi2d_resample(int method, int adjoint, int sinc_half_length, int ntr, int nm, float dm, int np, float dp,
                   const float *in, float *out)
{
    ABI_TRY
    REQ(in && out, "null argument");
    REQ(method == FWI2D_RESAMPLE_SINC || method == FWI2D_RESAMPLE_LINEAR, "unknown resampling method");
    REQ(method == FWI2D_RESAMPLE_LINEAR || sinc_half_length > 0, "the sinc half length must be positive");
    REQ(ntr >= 0 && ntr <= 65535 && nm > 0 && np > 0 && dm > 0.f && dp > 0.f, "bad resampling axes");
    if (ntr == 0) return FWI2D_OK;
    const size_t nin = (size_t)ntr * (adjoint ? np : nm), nout = (size_t)ntr * (adjoint ? nm : np);
    DevBuf a, b;
    a.alloc(nin * sizeof(float));
    b.alloc(nout * sizeof(float));
    CK(cudaMemcpy(a.p, in, nin * sizeof(float), cudaMemcpyHostToDevice));
    if (!adjoint)
        k_resample_fwd<<<dim3((np + 127) / 128, ntr), 128>>>(a.as<float>(), b.as<float>(), nm, dm, np, dp,
                                                             sinc_half_length, method == FWI2D_RESAMPLE_LINEAR);
    else
        k_resample_adj<<<dim3((nm + 127) / 128, ntr), 128>>>(a.as<float>(), b.as<float>(), nm, dm, np, dp,
                                                             sinc_half_length, method == FWI2D_RESAMPLE_LINEAR);
    CK(cudaGetLastError());
    CK(cudaMemcpy(out, b.p, nout * sizeof(float), cudaMemcpyDeviceToHost));
    ABI_END
}

int fwi2d_set_observed(fwi2d_ctx *ctx, const float *obs)
{
    ABI_TRY
    REQ(ctx, "null context");
    set_observed(ctx, obs);
    ABI_END
}

int fwi2d_fwi_gradient(fwi2d_ctx *ctx, const float *model, const float *src, const float *obs, int seismotype,
                       float *grad, double *misfit)
{
    ABI_TRY
    REQ(ctx, "null context");
    REQ(seismotype == 0 || seismotype == 1, "seismotype must be 0 or 1");
    if (model) update_model(ctx, model);
    if (src) {
        if (need_plan(ctx).dd > 0.f) upload_sources_axis(ctx, src);
        else upload_traces(ctx, src, false);
    }
    if (obs) set_observed(ctx, obs);
    fwi_gradient(ctx, seismotype, true);
    if (grad) download_grad(ctx, grad);
    if (misfit) *misfit = read_misfit(ctx);
    ABI_END
}

}  // extern "C"

// Dipole receivers (dipole_m3) in the drop-in: each dipole becomes two delta
// receivers, one per end, interleaved (trace t's ends are rows 2t and 2t+1),
// with the dipole's own index and weight tables.  The forward's dipole trace is
// end 2 minus end 1 (injector.cpp:359-380, the same per-cell products summed
// per end); the adjoint injects -q at end 1 and +q at end 2 (:328-357).
struct DipoleSplit {
    std::vector<int> xi, zi;
    std::vector<float> xw, zw;
    fwi2d_injector inj;
};

static void split_dipole(const fwi2d_injector &d, DipoleSplit &s)
{
    REQ(d.ntr >= 0 && (d.ntr == 0 || (d.xind && d.zind && d.xw && d.zw)), "dipole injector: null table");
    const int n = d.ntr;
    s.xi.resize((size_t)6 * n);
    s.zi.resize((size_t)6 * n);
    s.xw.resize((size_t)12 * n);
    s.zw.resize((size_t)12 * n);
    for (int t = 0; t < n; t++)
        for (int e = 0; e < 2; e++) {
            const int row = 2 * t + e;
            for (int k = 0; k < 3; k++) {
                s.xi[row * 3 + k] = d.xind[t * 6 + 3 * e + k];
                s.zi[row * 3 + k] = d.zind[t * 6 + 3 * e + k];
                for (int p = 0; p < 2; p++) {
                    s.xw[(row * 2 + p) * 3 + k] = d.xw[(t * 2 + p) * 6 + 3 * e + k];
                    s.zw[(row * 2 + p) * 3 + k] = d.zw[(t * 2 + p) * 6 + 3 * e + k];
                }
            }
        }
    s.inj = {FWI2D_INJ_DELTA, 2 * n, s.xi.data(), s.zi.data(), s.xw.data(), s.zw.data()};
}

extern "C" {

int fwi2d_propagate(int kind, int adj, const float *model, const float *allsrc, float *allrcv,
                    const fwi2d_injector *inj, const fwi2d_injector *ext, const fwi2d_injector *inja,
                    const fwi2d_injector *exta, float *full_wfld, float *grad, const fwi2d_params *par, int ns, int nr,
                    int nx, int nz, float dx, float dz)
{
    ABI_TRY
    REQ(par && model, "null argument");
    REQ(kind >= FWI2D_ELASTIC && kind <= FWI2D_ACOUSTIC_ELASTIC, "unknown propagator kind");
    const bool ae = kind == FWI2D_ACOUSTIC_ELASTIC;
    const bool src_fluid = ae && par->acoustic_source;
    // acoustic-elastic: forward sources in the fluid (inja) or the solid (inj),
    // receivers in both (ext, exta); the adjoint injects at both receiver sets
    // (inj, inja) and needs the source side (ext or exta) only for the plan.
    // Other propagators: inj and ext.
    if (!ae) REQ(inj && ext, "null argument");
    else if (!adj) REQ(ext && exta && (src_fluid ? inja : inj), "null argument");
    else REQ(inj && inja && (src_fluid || ext), "null argument");
    // dipole receivers: ext in the forward, inj in the adjoint (elastic and VTI)
    const fwi2d_injector *rcv_side = adj ? inj : ext;
    const bool dipole = rcv_side && rcv_side->type == FWI2D_INJ_DIPOLE;
    if (dipole && kind != FWI2D_ELASTIC && kind != FWI2D_VTI)
        throw Error(FWI2D_ERR_UNSUPPORTED, "dipole receivers are supported for the elastic and VTI propagators");
    REQ(!((adj ? ext : inj) && (adj ? ext : inj)->type == FWI2D_INJ_DIPOLE), "a dipole cannot be a source");
    DipoleSplit dsplit;
    if (dipole) split_dipole(*rcv_side, dsplit);
    const fwi2d_injector none = {FWI2D_INJ_DELTA, 0, nullptr, nullptr, nullptr, nullptr};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    fwi2d_ctx *ctx = thread_ctx(dev);
    fwi2d_params p = *par;
    p.snapshot_precision = FWI2D_SNAP_FP32;
    p.checkpoint_every = 0;
    const int nt = p.nt;
    if (adj) REQ(p.sub > 0 && full_wfld && grad, "the adjoint needs snapshots (sub > 0) and a gradient buffer");
    set_model(ctx, kind, nx, nz, dx, dz, model);
    // forward: inject the sources, extract the receivers; adjoint: inject the receivers
    fwi2d_shot sh;
    std::memset(&sh, 0, sizeof(sh));
    sh.x0 = 0;
    sh.nx = nx;
    sh.nt = nt;
    if (!ae) {
        sh.src = adj ? *ext : *inj;
        sh.rcv = dipole ? dsplit.inj : (adj ? *inj : *ext);
        if (adj) p.mt = sh.src.type == FWI2D_INJ_DDELTA;
    } else if (!adj) {
        sh.src = src_fluid ? none : *inj;
        sh.src_water = src_fluid ? *inja : none;
        sh.rcv = *ext;
        sh.rcv_water = *exta;
    } else {
        // the plan needs the source side only for its forward tables
        sh.rcv = *inj;
        sh.rcv_water = *inja;
        sh.src = src_fluid ? none : *ext;
        sh.src_water = src_fluid ? (exta ? *exta : *inja) : none;
    }
    const bool store = !adj && p.sub > 0 && full_wfld != nullptr;
    fwi2d_params pp = p;
    if (!store && !adj) pp.sub = 0;
    set_shots(ctx, &pp, 1, &sh);
    Plan &P = *ctx->plan;
    ShotPlan &S = *P.shots[0];
    // gather the component blocks (stride ns*nt / nr*nt in the reference's buffers)
    const int in_ntr = adj ? S.nr : S.ntr_src;
    const int out_comp = S.nrcv_rows / S.nr;   // traces per receiver: 1, 2, or 3 (fluid, x, z)
    const int in_comp = adj ? out_comp : S.ncomp_src;
    const int stride = adj ? nr : ns;
    std::vector<float> in((size_t)in_comp * in_ntr * nt);
    if (dipole && adj) {
        // end 1 takes -q, end 2 +q
        for (int c = 0; c < in_comp; c++)
            for (int t = 0; t < in_ntr / 2; t++) {
                const float *q = allsrc + ((size_t)c * stride + t) * nt;
                float *e1 = &in[((size_t)c * in_ntr + 2 * t) * nt], *e2 = e1 + nt;
                for (int k = 0; k < nt; k++) {
                    e1[k] = -q[k];
                    e2[k] = q[k];
                }
            }
    } else {
        for (int c = 0; c < in_comp; c++)
            for (int t = 0; t < in_ntr; t++)
                std::memcpy(&in[((size_t)c * in_ntr + t) * nt], allsrc + ((size_t)c * stride + t) * nt,
                            nt * sizeof(float));
    }
    if (!adj) {
        std::vector<float> out((size_t)out_comp * S.nr * nt);
        upload_traces(ctx, in.data(), false);
        run(ctx, false, store);
        download_rcv(ctx, out.data());
        if (dipole) {
            for (int c = 0; c < out_comp; c++)
                for (int t = 0; t < S.nr / 2; t++) {
                    float *dst = allrcv + ((size_t)c * nr + t) * nt;
                    const float *e1 = &out[((size_t)c * S.nr + 2 * t) * nt], *e2 = e1 + nt;
                    for (int k = 0; k < nt; k++) dst[k] += e2[k] - e1[k];
                }
        } else {
            for (int c = 0; c < out_comp; c++)
                for (int t = 0; t < S.nr; t++) {
                    float *dst = allrcv + ((size_t)c * nr + t) * nt;
                    const float *src = &out[((size_t)c * S.nr + t) * nt];
                    for (int k = 0; k < nt; k++) dst[k] += src[k];
                }
        }
        if (store) store_host_snapshots(ctx, full_wfld);
    } else {
        load_host_snapshots(ctx, full_wfld);
        std::vector<float> g((size_t)P.ncompg * nx * nz);
        upload_traces(ctx, in.data(), true);
        run(ctx, true, false);
        download_grad(ctx, g.data());
        for (size_t i = 0; i < g.size(); i++) grad[i] += g[i];
    }
    ABI_END
}

}  // extern "C"
