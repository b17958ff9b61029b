/*
 * fwi2d_b200 -- C ABI of the B200 (sm_100a) SBP propagation library.
 *
 * The library replaces the GPU hook of the reference's wave-equation
 * operators: nl_we_op_e::propagate_gpu / nl_we_op_vti::propagate_gpu
 * (src/include/we_op.hpp:82, :174, implemented by src/cuda/cudaWeOp.cpp:10-433,
 * :436-876) and the hooks the acoustic and acoustic-elastic operators declare
 * but leave commented out (we_op.hpp:259-260, :339).  Plain pointers and sizes
 * only; no exception crosses this boundary.  Every function returns
 * FWI2D_OK (0) or a negative status; fwi2d_last_error() gives the message.
 *
 * Array layouts are the reference's (x-major, z fastest, "[ix*nz+iz]"):
 *   converted model  [npar][nx][nz]   elastic (lambda, mu, rho), VTI (lambda, mu,
 *                                     rho, c13, eps), acoustic (K, 1/rho)
 *   traces           [ncomp][ntr][nt] time fastest
 *   snapshots        [nt/sub+1][ncomp][nx][nz]
 *   gradient         [3][nx][nz] (lambda, mu, rho) or [2][nx][nz] (K, 1/rho)
 * Units are the reference's: km, s, km/s, g/cm^3.
 */
#ifndef FWI2D_B200_H
#define FWI2D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define FWI2D_OK 0
#define FWI2D_ERR_ARG (-1)          /* invalid argument, geometry or parameter */
#define FWI2D_ERR_CUDA (-2)         /* CUDA runtime error */
#define FWI2D_ERR_OOM (-3)          /* device memory exhausted */
#define FWI2D_ERR_STATE (-4)        /* call out of order (no model / no shots) */
#define FWI2D_ERR_UNSUPPORTED (-5)  /* option the kernels do not implement */
#define FWI2D_ERR_TIMEOUT (-6)      /* a bounded device wait gave up */

/* propagators: nl_we_op_e, nl_we_op_vti, nl_we_op_a, nl_we_op_ae */
#define FWI2D_ELASTIC 0
#define FWI2D_VTI 1
#define FWI2D_ACOUSTIC 2
#define FWI2D_ACOUSTIC_ELASTIC 3

/* snapshot storage */
#define FWI2D_SNAP_FP32 0
#define FWI2D_SNAP_BF16 1
#define FWI2D_SNAP_FP16 2

/* injector types (src/include/injector.hpp:39, :69) */
#define FWI2D_INJ_DELTA 0   /* delta_m3: 3x3 discrete delta */
#define FWI2D_INJ_DDELTA 1  /* ddelta_m3: moment tensor */
#define FWI2D_INJ_DIPOLE 2  /* dipole_m3 (injector.hpp:99-120): two 3x3 deltas gl apart along the dip, for
                             * distributed acoustic sensing receivers (param.gl > 0); tables xind/zind
                             * [ntr][6], xw/zw [ntr][2][6], end 1 in columns 0-2, end 2 in 3-5.
                             * fwi2d_propagate only (elastic and VTI), as ext (forward) or inj (adjoint). */

/* The fields of the reference's `param` (src/include/param.hpp:8-83) that the
 * propagation reads, plus the storage options of this library. */
typedef struct fwi2d_params {
    int nt, sub;
    float dt;
    int bc_top, bc_bottom, bc_left, bc_right;              /* 1 free/rigid, 2 absorbing, 3 Neumann (acoustic) */
    int taper_top, taper_bottom, taper_left, taper_right;
    float taper_strength, free_surface_stiffness;
    int mt;                                                /* moment-tensor source */
    float gdamp_tmin, gdamp_tmax, gdamp_power;
    int nza;                                               /* acoustic-elastic: water rows */
    float water_velocity, water_density;
    int acoustic_source;                                   /* acoustic-elastic: source in the water */
    /* library options */
    int snapshot_precision;                                /* FWI2D_SNAP_* */
    int checkpoint_every;                                  /* 0: keep snapshots; k>0: recompute from checkpoints every k steps */
    int compensated;                                       /* 1: compensated (two-level) gradient accumulation: the
                                                            * imaging terms of 8 adjoint steps are summed in FP32,
                                                            * each such partial sum joins a running (hi, lo) pair by
                                                            * Neumaier's compensated summation; 0: the reference's
                                                            * plain FP32 accumulation (bitwise) */
    int tile_shape;                                        /* -1: autotuned; else fwi2d_tile_shape index */
} fwi2d_params;

/* Public tables of the reference's injector (src/include/injector.hpp:9-13). */
typedef struct fwi2d_injector {
    int type;           /* FWI2D_INJ_* */
    int ntr;
    const int *xind;    /* [ntr][3] */
    const int *zind;    /* [ntr][3] */
    const float *xw;    /* [ntr][2][3] (delta) or [ntr][2][6] (moment tensor) */
    const float *zw;
} fwi2d_injector;

/* One shot of a batch: its own grid is the model columns [x0, x0+nx). */
typedef struct fwi2d_shot {
    int x0, nx;
    int nt;                     /* time samples of this shot, <= params.nt */
    fwi2d_injector src;         /* sources on the shot grid */
    fwi2d_injector rcv;         /* receivers on the shot grid */
    fwi2d_injector src_water;   /* acoustic-elastic: water-layer source (ntr = 0 if none) */
    fwi2d_injector rcv_water;   /* acoustic-elastic: water-layer receivers */
} fwi2d_shot;

typedef struct fwi2d_ctx fwi2d_ctx;

const char *fwi2d_last_error(void);
int fwi2d_version(void);

/* The fields of the reference's `param` that analyzeModel reads and writes
 * (src/include/param.hpp:11-46; defaults there: courant 0.6, dt -1, sub 0,
 * vp 0.2-8, vs 0.1-5, rho 0.1-8, delta -0.5-1, epsilon 0-1 km/s, g/cc). */
typedef struct fwi2d_model_check {
    float vpmin, vpmax, vsmin, vsmax, rhomin, rhomax, deltamin, deltamax, epsilonmin, epsilonmax;
    int soft_clip;          /* keep values outside the bounds (elastic and VTI only) */
    int acoustic_elastic;   /* the water velocity joins vmax / vmin */
    float water_velocity;
    float courant;          /* in/out */
    float dt;               /* in/out: 0 from the CFL number; > 0 min(dt, data step); < 0 the CFL step rounded down to divide the data step */
    int sub;                /* in/out: < 0 becomes round(data step / dt) */
    int nt;                 /* out: round(tmax / dt) + 1 */
    float tmax, vmax, vmin; /* out */
} fwi2d_model_check;

/* analyzeModel (src/cpp/we_op.cpp:267-474) on a raw host model [npar][nx][nz]
 * (npar 2: vp, rho; 3: vp, vs, rho; 5: + delta, epsilon), in place: the Thomsen
 * delta admissibility clip (VTI), the hard clip to the bounds, Vs <= Vp/sqrt(2),
 * the maximum P velocity (VTI: vp sqrt(1 + 2 eps)), then the propagation step,
 * nt and sub from the data time axis (data_nt samples at data_dt).  Host only:
 * needs no GPU. */
int fwi2d_analyze_model(int npar, float *model, int nx, int nz, float dx, float dz, int data_nt, float data_dt,
                        fwi2d_model_check *check);

/* delta_m3 / ddelta_m3::findIndicesWeights (src/cpp/injector.cpp:3-64, 114-187). */
int fwi2d_injector_weights(int type, int ntr, const float *locx, const float *locz, int nx, int nz,
                           float dx, float dz, float ox, float oz, int *xind, int *zind, float *xw, float *zw);

/* dipole_m3::findIndicesWeights (src/cpp/injector.cpp:241-326): the tables of
 * ntr dipoles centred at (locx, locz) with dip angles dip (radians) and gauge
 * length gl (param.gl; param.rdip gives the angles, param.cpp). */
int fwi2d_dipole_weights(int ntr, const float *locx, const float *locz, const float *dip, float gl, int nx, int nz,
                         float dx, float dz, float ox, float oz, int *xind, int *zind, float *xw, float *zw);

/* Context: one device, one stream, one model, one batch plan.  Calls on one
 * context must be serialised by the caller. */
int fwi2d_ctx_create(int device, fwi2d_ctx **out);
int fwi2d_ctx_destroy(fwi2d_ctx *ctx);

/* Upload a converted model (host [npar][nx][nz]); the model grid is dx x dz. */
int fwi2d_set_model(fwi2d_ctx *ctx, int kind, int nx, int nz, float dx, float dz, const float *model);

/* Build the batch plan: per-shot device buffers, tables and CUDA graphs. */
int fwi2d_set_shots(fwi2d_ctx *ctx, const fwi2d_params *par, int nshots, const fwi2d_shot *shots);

/* Forward propagation of every shot of the plan (nl_we_op_*::propagate with
 * adj=false, we_op.cpp:564).  src: concatenated per-shot blocks [ncomp][ntr][nt];
 * rcv: concatenated per-shot blocks [ncomp][nr][nt], overwritten.  With
 * store_snapshots the forward wavefields stay on the device for fwi2d_adjoint. */
int fwi2d_forward(fwi2d_ctx *ctx, const float *src, float *rcv, int store_snapshots);

/* Adjoint propagation with the zero-lag imaging condition (propagate with
 * adj=true).  adj: concatenated per-shot blocks in the receiver layout;
 * grad: model-grid gradient [3 or 2][nx][nz], the sum over shots, overwritten. */
int fwi2d_adjoint(fwi2d_ctx *ctx, const float *adj, float *grad);

/* Device-resident variants: upload traces once (adjoint=0 sources, 1 adjoint
 * sources), then run the propagation with inputs and outputs left on the
 * device.  fwi2d_run returns when the work is queued; fwi2d_sync waits. */
int fwi2d_upload_traces(fwi2d_ctx *ctx, const float *traces, int adjoint);
int fwi2d_run(fwi2d_ctx *ctx, int adjoint, int store_snapshots);
int fwi2d_sync(fwi2d_ctx *ctx);

/* New values for the current model geometry (converted, host [npar][nx][nz]);
 * the batch plan, its tables and graphs stay valid. */
int fwi2d_update_model(fwi2d_ctx *ctx, const float *model);

/* Observed data of every shot, concatenated per-shot blocks [ncomp][nr][nt]
 * ([ncomp][nr][nd] after fwi2d_set_data_axis), kept on the device for
 * fwi2d_fwi_gradient. */
int fwi2d_set_observed(fwi2d_ctx *ctx, const float *obs);

/* time resamplers (src/cpp/operator.cpp:734-856; param.resampling) */
#define FWI2D_RESAMPLE_SINC 0     /* sinc_resampler: cosine-windowed sinc, param.sinc_half_length */
#define FWI2D_RESAMPLE_LINEAR 1   /* linear_resampler */

/* Sources and data of fwi2d_fwi_gradient on their own time axis, as the
 * reference's operators take them (the time axis of the source and data cubes;
 * nl_we_op_e::apply_forward / apply_jacobianT, we_op.cpp:930-1054, 1086-1124):
 * shot k has nd[k] samples at dt_data, and the plan propagates at its
 * params.dt <= dt_data with nt = round((nd[k] - 1) dt_data / dt) + 1 (analyzeModel,
 * we_op.cpp:446-464; other nt are rejected).  fwi2d_fwi_gradient then takes src
 * as per-shot blocks [rows][nd] and obs as [ncomp][nr][nd], resamples the
 * sources to dt, the synthetics (alpha Dt of the receivers, alpha = dt /
 * dt_data) back to dt_data, forms the residual, the misfit 1/2 dt_data (...)
 * and the applyHt weighting on the data axis, and the adjoint sources through
 * the forward resampler, applyHt^-1, reversal, -alpha and Dt^T.  Call after
 * fwi2d_set_shots (a new plan clears it); dt_data <= 0 clears it.  The
 * resident observed data are dropped. */
int fwi2d_set_data_axis(fwi2d_ctx *ctx, float dt_data, int method, int sinc_half_length, const int *nd);

/* The reference's resampler on ntr host traces (sinc_resampler /
 * linear_resampler::apply_forward and apply_adjoint with add = false,
 * operator.cpp:760-856), computed on the current device.  Domain axis: nm
 * samples at dm; range axis: np samples at dp; both from t = 0.  adjoint = 0:
 * in [ntr][nm] -> out [ntr][np]; adjoint = 1: in [ntr][np] -> out [ntr][nm]. */
int fwi2d_resample(int method, int adjoint, int sinc_half_length, int ntr, int nm, float dm, int np, float dp,
                   const float *in, float *out);

/* One FWI gradient evaluation on the device (nlls_fwi_eco::compute_res_and_grad,
 * optimization.hpp:590-951, with the data-side options off): forward with
 * snapshots, residual against the observed data (seismotype 1: particle
 * velocity, the time derivative of the extracted displacement), L2 misfit
 * 1/2 dt (|r|^2 - (r_0^2 + r_end^2)/2), adjoint sources, adjoint propagation
 * with the imaging condition, H quadrature and the chain rule to (vp, vs, rho),
 * or (vp, rho) for the acoustic propagator.  model / src / obs may be NULL to
 * reuse what is resident; grad (host [3 or 2][nx][nz]) and misfit may be NULL
 * to leave the results on the device. */
int fwi2d_fwi_gradient(fwi2d_ctx *ctx, const float *model, const float *src, const float *obs, int seismotype,
                       float *grad, double *misfit);

/* Read back one stored snapshot [ncomp][nx][nz] of one shot (dequantised). */
int fwi2d_snapshot(fwi2d_ctx *ctx, int shot, int slot, float *out);

/* Per-plan facts: number of kernel launches of one forward / adjoint pass,
 * the tile shape in use, snapshot bytes held. */
int fwi2d_plan_info(fwi2d_ctx *ctx, long long *launches_fwd, long long *launches_adj, int *tile_shape,
                    long long *snapshot_bytes);

/* Waves of the plan.  When the snapshots of all its shots do not fit the
 * device together (less a reserve), an elastic or VTI plan runs its shots in
 * waves: contiguous runs of shots whose snapshots fit, sharing one snapshot
 * store.  fwi2d_fwi_gradient then runs forward, residual and adjoint wave by
 * wave; fwi2d_forward with snapshots, fwi2d_adjoint and fwi2d_snapshot return
 * FWI2D_ERR_UNSUPPORTED.  The environment variable FWI2D_SNAPSHOT_BUDGET
 * (bytes), read by fwi2d_set_shots, replaces the budget.  No counterpart in
 * the reference, which runs one shot at a time (we_op.cpp:970, 1146). */
int fwi2d_plan_waves(fwi2d_ctx *ctx, int *nwaves, long long *snapshot_bytes_all);

/* Order all later work of the context on a caller's CUDA stream (a
 * cudaStream_t; NULL returns to the context's own stream). */
int fwi2d_set_stream(fwi2d_ctx *ctx, void *stream);

/* Copy the model-grid gradient of the last adjoint into caller device memory
 * [3 or 2][nx][nz], ordered on the context stream. */
int fwi2d_copy_gradient(fwi2d_ctx *ctx, float *dst_device);

/* Device time (CUDA events on the context stream) of the last forward and
 * adjoint time loops, in milliseconds (-1 if none ran). */
int fwi2d_last_timing(fwi2d_ctx *ctx, float *forward_ms, float *adjoint_ms);

/* Work shapes offered to the autotuner: tile shapes of the tile kernel over
 * whole shot grids (tz x tx cells), then marching shapes (tz threads, one z
 * cell each, marching runs of tx rows) for the cells clear of the boundary
 * bands, then framed tile shapes (tz x tx tiles of the tile kernel's interior
 * path over those cells); marching and framed plans run the boundary bands on
 * the band kernels. */
int fwi2d_tile_shape_count(void);
int fwi2d_tile_shape(int index, int *tz, int *tx);

/* Drop-in for propagate_gpu: one shot, host buffers, the reference's argument
 * meaning (we_op.hpp:82).  ns / nr are the trace counts that separate the
 * component blocks of allsrc / allrcv (par.ns and par.nr of the reference).
 * Forward accumulates into allrcv and writes full_wfld when sub > 0; adjoint
 * reads full_wfld and accumulates the imaging condition into grad.
 * Acoustic-elastic propagator (FWI2D_ACOUSTIC_ELASTIC, we_op.cpp:2137-2577):
 * inja / exta are the injectors on the fluid layer's grid (nx x par->nza,
 * depths from 0).  Forward: sources through inja (par->acoustic_source) or
 * inj, receivers through ext (solid) and exta (fluid), traces [3][nr][nt] as
 * (fluid, x, z).  Adjoint: the adjoint traces [3][nr][nt] are injected
 * through inja (fluid block) and inj (x, z blocks); ext / exta are the source
 * side.  NULL for the other propagators. */
int fwi2d_propagate(int kind, int adj, const float *model, const float *allsrc, float *allrcv,
                    const fwi2d_injector *inj, const fwi2d_injector *ext,
                    const fwi2d_injector *inja, const fwi2d_injector *exta,
                    float *full_wfld, float *grad, const fwi2d_params *par, int ns, int nr,
                    int nx, int nz, float dx, float dz);

/* Allocation-free forward propagation.  No counterpart in the reference: it
 * serves callers that cannot allocate device memory (plug-ins whose host
 * framework owns the device allocator, real-time loops that forbid the
 * device-synchronising cudaMalloc / cudaFree after start-up).  Same meaning and results as
 * fwi2d_propagate with adj = 0 and no snapshots, for the elastic isotropic
 * propagator with point-force sources: host inputs, receivers accumulated into
 * allrcv.  All device-side buffers live in one static array of
 * FWI2D_NOALLOC_SCRATCH_BYTES; problems that do not fit it (or exceed the
 * FWI2D_NOALLOC_MAX_* table limits) are rejected with FWI2D_ERR_ARG.
 * The CUDA runtime loads that array lazily: the first call on a device
 * reserves it (a GPU then holds it until the process exits), looks up its
 * device address with that device current and may synchronise the device.
 * Make that first call at start-up, before any real-time loop or stream
 * capture; later calls allocate nothing.  The array keeps the last call's
 * contents (each call clears what must start at zero).  Calls that overlapped
 * on the GPU would race on it: a host mutex serialises the calls of a process
 * and each returns only after its GPU work is done, so they never overlap;
 * every process has its own copy.  Each call runs on the legacy default
 * stream (not the stream of fwi2d_set_stream), so it synchronises with every
 * blocking stream on the device.  Errors: fwi2d_noalloc_last_error(). */
#define FWI2D_NOALLOC_SCRATCH_BYTES (64u << 20)
#define FWI2D_NOALLOC_MAX_AXIS 16384
#define FWI2D_NOALLOC_MAX_SOURCES 16
#define FWI2D_NOALLOC_MAX_RECEIVERS 8192
int fwi2d_propagate_noalloc(const float *model, const float *allsrc, float *allrcv, const fwi2d_injector *inj,
                            const fwi2d_injector *ext, const fwi2d_params *par, int ns, int nr, int nx, int nz,
                            float dx, float dz);
const char *fwi2d_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
