// C entry points over the reference's own propagation code, for the oracle
// build only.  Compiled together with the reference sources (src/cpp/we_op.cpp,
// spatial_operators.cpp, injector.cpp, misc.cpp, operator.cpp, dummy.cpp) by
// oracle/build_ref.sh into oracle/_ref/.  Used to generate tests/golden/ and
// to pin the restatement in oracle/fwi2d_oracle.c.
#include <algorithm>
#include <vector>
#include <memory>
#include <cstdio>
#include <cstring>
#include "we_op.hpp"
#include "nlsolver.hpp"
#include "IO.hpp"

struct ref_param {
    int nt, sub;
    double dt;
    int ns, nr;
    int bc_top, bc_bottom, bc_left, bc_right;
    int taper_top, taper_bottom, taper_left, taper_right;
    double taper_strength, free_surface_stiffness;
    int mt;
    double gdamp_tmin, gdamp_tmax, gdamp_power;
    int nza;
    double water_velocity, water_density;
    int acoustic_source;
};

static param to_param(const ref_param *p)
{
    param par;
    par.nt = p->nt; par.sub = p->sub; par.dt = (data_t)p->dt;
    par.ns = p->ns; par.nr = p->nr;
    par.bc_top = p->bc_top; par.bc_bottom = p->bc_bottom; par.bc_left = p->bc_left; par.bc_right = p->bc_right;
    par.taper_top = p->taper_top; par.taper_bottom = p->taper_bottom;
    par.taper_left = p->taper_left; par.taper_right = p->taper_right;
    par.taper_strength = (data_t)p->taper_strength;
    par.free_surface_stiffness = (data_t)p->free_surface_stiffness;
    par.mt = p->mt != 0;
    par.gdamp_tmin = (data_t)p->gdamp_tmin; par.gdamp_tmax = (data_t)p->gdamp_tmax; par.gdamp_power = (data_t)p->gdamp_power;
    par.nza = p->nza;
    par.water_velocity = (data_t)p->water_velocity; par.water_density = (data_t)p->water_density;
    par.acoustic_source = p->acoustic_source != 0;
    par.acoustic_elastic = p->nza > 0;
    par.version = 2;
    par.pml = false; par.pml_T = par.pml_B = par.pml_L = par.pml_R = false;
    par.verbose = 0;
    return par;
}

static std::vector<std::vector<data_t> > locs(int n, const data_t *x, const data_t *z)
{
    std::vector<std::vector<data_t> > v(n);
    for (int i = 0; i < n; i++) v[i] = {x[i], z[i], 0};
    return v;
}

static hypercube<data_t> grid(int nx, int nz, double dx, double dz, double ox, double oz)
{
    return hypercube<data_t>(axis<data_t>(nz, (data_t)oz, (data_t)dz), axis<data_t>(nx, (data_t)ox, (data_t)dx));
}

extern "C" {

int ref_real_size(void) { return (int)sizeof(data_t); }

// nl_we_op_*::convert_model, in place on [npar][n].
int ref_convert_model(int kind, data_t *m, int n, int forward)
{
    if (kind == 0 || kind == 3) { nl_we_op_e op; op.convert_model(m, n, forward != 0); }
    else if (kind == 1) { nl_we_op_vti op; op.convert_model(m, n, forward != 0); }
    else if (kind == 2) { nl_we_op_a op; op.convert_model(m, n, forward != 0); }
    else return -1;
    return 0;
}

// injector tables built by the reference's delta_m3 / ddelta_m3.
int ref_injector_weights(int type, int ntr, const data_t *lx, const data_t *lz, int nx, int nz,
                         double dx, double dz, double ox, double oz, int *xind, int *zind, data_t *xw, data_t *zw)
{
    hypercube<data_t> g = grid(nx, nz, dx, dz, ox, oz);
    injector *J;
    if (type == 0) J = new delta_m3(g, locs(ntr, lx, lz));
    else J = new ddelta_m3(g, locs(ntr, lx, lz));
    std::memcpy(xind, J->_xind.data(), J->_xind.size() * sizeof(int));
    std::memcpy(zind, J->_zind.data(), J->_zind.size() * sizeof(int));
    std::memcpy(xw, J->_xw.data(), J->_xw.size() * sizeof(data_t));
    std::memcpy(zw, J->_zw.data(), J->_zw.size() * sizeof(data_t));
    delete J;
    return 0;
}

// One shot through the reference's operator interface: nl_we_op_e (kind 0)
// or nl_we_op_vti (kind 1) forward modelling of the raw model (vp, vs, rho
// [, delta, eps]) with seismotype 1 (particle velocity), linear resampling at
// the propagation rate (the identity), and, when obs is given, the gradient
// the solver forms (optimization.hpp:760-890): residual r = f(m) - obs
// weighted by applyHt, then apply_jacobianT (we_op.cpp:1057-1239).  src is
// [2][nt] (x, z force), syn and obs [2][nr][nt], grad [npar][nx][nz].
static int misfit_grad(int kind, const ref_param *rp, int nx, int nz, double dx, double dz, int nt, double dt,
                       double prop_dt, const char *resampling, int hl,
                       data_t sx, data_t sz, int nr, const data_t *rx, const data_t *rz, const data_t *model,
                       const data_t *src, const data_t *obs, data_t *syn, data_t *grad)
{
    try {
        param par = to_param(rp);
        par.nt = nt;
        par.dt = (data_t)prop_dt;
        par.sub = obs ? 1 : 0;
        par.ns = 1;
        par.nr = nr;
        par.nmodels = kind == 1 ? 5 : (kind == 2 ? 2 : 3);
        const int nc = kind == 2 ? 1 : 2;   // trace components (sources and receivers)
        par.seismotype = 1;
        par.resampling = resampling;
        par.sinc_half_length = hl;
        data_t sl[2] = {sx, sz};
        par.sxz = locs(1, sl, sl + 1);
        par.rxz = {locs(nr, rx, rz)};
        hypercube<data_t> dom(axis<data_t>(nz, 0, (data_t)dz), axis<data_t>(nx, 0, (data_t)dx),
                              axis<data_t>(par.nmodels, 0, 1));
        auto allsrc = std::make_shared<vecReg<data_t> >(hypercube<data_t>(axis<data_t>(nt, 0, (data_t)dt), axis<data_t>(nc, 0, 1)));
        std::memcpy(allsrc->getVals(), src, nc * (size_t)nt * sizeof(data_t));
        std::shared_ptr<nl_we_op> op;
        if (kind == 0) op = std::make_shared<nl_we_op_e>(dom, allsrc, par);
        else if (kind == 1) op = std::make_shared<nl_we_op_vti>(dom, allsrc, par);
        else op = std::make_shared<nl_we_op_a>(dom, allsrc, par);
        auto m = std::make_shared<vecReg<data_t> >(dom);
        std::memcpy(m->getVals(), model, m->getN123() * sizeof(data_t));
        auto d = std::make_shared<vecReg<data_t> >(*op->getRange());
        op->forward(false, m, d);
        std::memcpy(syn, d->getCVals(), d->getN123() * sizeof(data_t));
        if (obs) {
            auto r = std::make_shared<vecReg<data_t> >(*op->getRange());
            data_t *pr = r->getVals();
            const long n = (long)r->getN123();
            for (long i = 0; i < n; i++) pr[i] = syn[i] - obs[i];
            applyHt(false, false, pr, pr, nc * nr, nt, (data_t)dt, 0, nc * nr);
            auto g = std::make_shared<vecReg<data_t> >(dom);
            op->jacobianT(false, g, m, r);
            std::memcpy(grad, g->getCVals(), g->getN123() * sizeof(data_t));
        }
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_misfit_grad: %s\n", e.what());
        return -1;
    }
    return 0;
}

int ref_misfit_grad(int kind, const ref_param *rp, int nx, int nz, double dx, double dz, int nt, double dt,
                    data_t sx, data_t sz, int nr, const data_t *rx, const data_t *rz, const data_t *model,
                    const data_t *src, const data_t *obs, data_t *syn, data_t *grad)
{
    return misfit_grad(kind, rp, nx, nz, dx, dz, nt, dt, dt, "linear", 11, sx, sz, nr, rx, rz, model, src, obs, syn,
                       grad);
}

// As ref_misfit_grad with sources and data on their own time axis (nd samples
// at dd) and the propagation at prop_dt: apply_forward / apply_jacobianT
// resample with the reference's sinc (linear = 0, half length hl) or linear
// resampler (we_op.cpp:930-955, 1086-1103); analyzeModel sets the propagation
// nt = round((nd-1) dd / dt) + 1 with dt = min(prop_dt, dd) (we_op.cpp:446-464).
// syn and obs are [nc][nr][nd]; the residual weighting applyHt uses dd, as
// compute_res_and_grad does (optimization.hpp:606-607, 780).
int ref_misfit_grad_rs(int kind, const ref_param *rp, int nx, int nz, double dx, double dz, int nd, double dd,
                       double prop_dt, int linear, int hl, data_t sx, data_t sz, int nr, const data_t *rx,
                       const data_t *rz, const data_t *model, const data_t *src, const data_t *obs, data_t *syn,
                       data_t *grad)
{
    return misfit_grad(kind, rp, nx, nz, dx, dz, nd, dd, prop_dt, linear ? "linear" : "sinc", hl, sx, sz, nr, rx, rz,
                       model, src, obs, syn, grad);
}

// analyzeModel (we_op.cpp:267-474) on a raw model [npar][nx][nz] in place,
// with the data time axis (data_nt samples at data_dt).  c holds, in order:
// vpmin, vpmax, vsmin, vsmax, rhomin, rhomax, deltamin, deltamax, epsilonmin,
// epsilonmax, soft_clip, acoustic_elastic, water_velocity, courant, dt, sub
// (inputs) and receives courant, dt, sub, nt, tmax, vmax, vmin in c[13..19].
int ref_analyze_model(int npar, data_t *model, int nx, int nz, double dx, double dz, int data_nt, double data_dt,
                      double *c)
{
    try {
        param par;
        par.verbose = 0;
        par.nmodels = npar;
        par.vpmin = (data_t)c[0]; par.vpmax = (data_t)c[1]; par.vsmin = (data_t)c[2]; par.vsmax = (data_t)c[3];
        par.rhomin = (data_t)c[4]; par.rhomax = (data_t)c[5]; par.deltamin = (data_t)c[6]; par.deltamax = (data_t)c[7];
        par.epsilonmin = (data_t)c[8]; par.epsilonmax = (data_t)c[9];
        par.soft_clip = c[10] != 0;
        par.acoustic_elastic = c[11] != 0;
        par.water_velocity = (data_t)c[12];
        par.courant = (data_t)c[13];
        par.dt = (data_t)c[14];
        par.sub = (int)c[15];
        hypercube<data_t> dom(axis<data_t>(nz, 0, (data_t)dz), axis<data_t>(nx, 0, (data_t)dx), axis<data_t>(npar, 0, 1));
        auto m = std::make_shared<vecReg<data_t> >(dom);
        std::memcpy(m->getVals(), model, (size_t)npar * nx * nz * sizeof(data_t));
        hypercube<data_t> T(axis<data_t>(data_nt, 0, (data_t)data_dt), axis<data_t>(1, 0, 1));
        analyzeModel(T, m, par);
        std::memcpy(model, m->getCVals(), (size_t)npar * nx * nz * sizeof(data_t));
        c[13] = par.courant; c[14] = par.dt; c[15] = par.sub; c[16] = par.nt; c[17] = par.tmax;
        c[18] = par.vmax; c[19] = par.vmin;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_analyze_model: %s\n", e.what());
        return -1;
    }
    return 0;
}

// dipole_m3 tables (injector.cpp:241-326) for ntr dipoles at (x, z) with dip
// angles dip and gauge length gl.
int ref_dipole_weights(int ntr, const data_t *x, const data_t *z, const data_t *dip, double gl, int nx, int nz,
                       double dx, double dz, double ox, double oz, int *xind, int *zind, data_t *xw, data_t *zw)
{
    hypercube<data_t> g = grid(nx, nz, dx, dz, ox, oz);
    std::vector<std::vector<data_t> > l(ntr);
    for (int i = 0; i < ntr; i++) l[i] = {x[i], z[i], dip[i]};
    dipole_m3 J(g, l, (data_t)gl);
    std::memcpy(xind, J._xind.data(), J._xind.size() * sizeof(int));
    std::memcpy(zind, J._zind.data(), J._zind.size() * sizeof(int));
    std::memcpy(xw, J._xw.data(), J._xw.size() * sizeof(data_t));
    std::memcpy(zw, J._zw.data(), J._zw.size() * sizeof(data_t));
    return 0;
}

// nl_we_op_e / nl_we_op_vti::propagate (kind 0 / 1) with one delta source at
// (sx, sz) and nr dipole receivers (dipole_m3, gauge gl, dip angles rdip) at
// (rx, rz): the forward extracts into allrcv [2][nr][nt]; the adjoint (adj = 1)
// injects allsrc [2][nr][nt] through the dipoles (allrcv then is the source's
// [2][1][nt]) and images into grad.
int ref_propagate_dipole(int kind, int adj, const data_t *model, const data_t *allsrc, data_t *allrcv,
                         data_t sx, data_t sz, int nr, const data_t *rx, const data_t *rz, const data_t *rdip,
                         double gl, data_t *full, data_t *grad, const ref_param *rp, int nx, int nz, double dx,
                         double dz)
{
    try {
        param par = to_param(rp);
        par.gl = (data_t)gl;
        hypercube<data_t> g = grid(nx, nz, dx, dz, 0, 0);
        data_t sl[2] = {sx, sz};
        injector *src = new delta_m3(g, locs(1, sl, sl + 1));
        std::vector<std::vector<data_t> > l(nr);
        for (int i = 0; i < nr; i++) l[i] = {rx[i], rz[i], rdip[i]};
        injector *rcv = new dipole_m3(g, l, (data_t)gl);
        injector *inj = adj ? rcv : src, *ext = adj ? src : rcv;
        if (kind == 0) { nl_we_op_e op; op.propagate(adj != 0, model, allsrc, allrcv, inj, ext, full, grad, par, nx, nz, (data_t)dx, (data_t)dz, 0, 0, 0); }
        else { nl_we_op_vti op; op.propagate(adj != 0, model, allsrc, allrcv, inj, ext, full, grad, par, nx, nz, (data_t)dx, (data_t)dz, 0, 0, 0); }
        delete src;
        delete rcv;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_propagate_dipole: %s\n", e.what());
        return -1;
    }
    return 0;
}

// binWrite (IO.hpp:179-222): vals on ndim axes (axis 1 first: n, o, d) to
// the header file `header` and its binary <datapath>/<header>@.
int ref_bin_write(const char *header, const data_t *vals, int ndim, const int *n, const double *o, const double *d,
                  const char *datapath)
{
    try {
        std::vector<axis<data_t> > ax;
        for (int i = 0; i < ndim; i++) ax.push_back(axis<data_t>(n[i], (data_t)o[i], (data_t)d[i]));
        auto v = std::make_shared<vecReg<data_t> >(hypercube<data_t>(ax));
        std::memcpy(v->getVals(), vals, v->getN123() * sizeof(data_t));
        binWrite<data_t>(v, header, datapath);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_bin_write: %s\n", e.what());
        return -1;
    }
    return 0;
}

// binRead (IO.hpp:226-429): the samples into out (at most cap), the kept
// axes into ndim, n, o, d (6 entries each).
int ref_bin_read(const char *header, int ndim0, data_t *out, long cap, int *ndim, int *n, double *o, double *d)
{
    try {
        auto v = binRead<data_t>(header, ndim0);
        const std::vector<axis<data_t> > ax = v->getHyper()->getAxes();
        *ndim = (int)ax.size();
        for (int i = 0; i < *ndim; i++) { n[i] = ax[i].n; o[i] = ax[i].o; d[i] = ax[i].d; }
        if (v->getN123() > cap) return -2;
        std::memcpy(out, v->getCVals(), v->getN123() * sizeof(data_t));
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_bin_read: %s\n", e.what());
        return -1;
    }
    return 0;
}

#ifdef CUDA
// nl_we_op_e / nl_we_op_vti::propagate_gpu with ref_propagate's arguments
// (kind 0 or 1), in the builds with -DCUDA: the reference's own GPU path
// (src/cuda/cudaWeOp.cpp; timed beside this library) or the hook on
// fwi2d_b200 (fwi2d_b200/integration/we_op_b200.cpp; tested against the CPU
// build).
int ref_propagate_gpu(int kind, int adj, const data_t *model, const data_t *allsrc, data_t *allrcv,
                      int inj_type, int ninj, const data_t *ix, const data_t *iz,
                      int next, const data_t *ex, const data_t *ez,
                      data_t *full, data_t *grad, const ref_param *rp, int nx, int nz,
                      double dx, double dz, double ox, double oz)
{
    try {
        param par = to_param(rp);
        par.device = 0;
        hypercube<data_t> g = grid(nx, nz, dx, dz, ox, oz);
        injector *inj = inj_type == 0 ? (injector *)new delta_m3(g, locs(ninj, ix, iz))
                                      : (injector *)new ddelta_m3(g, locs(ninj, ix, iz));
        injector *ext = new delta_m3(g, locs(next, ex, ez));
        if (kind == 0) { nl_we_op_e op; op.propagate_gpu(adj != 0, model, allsrc, allrcv, inj, ext, full, grad, par, nx, nz, (data_t)dx, (data_t)dz, (data_t)ox, (data_t)oz, 0); }
        else if (kind == 1) { nl_we_op_vti op; op.propagate_gpu(adj != 0, model, allsrc, allrcv, inj, ext, full, grad, par, nx, nz, (data_t)dx, (data_t)dz, (data_t)ox, (data_t)oz, 0); }
        else return -1;
        delete inj;
        delete ext;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_propagate_gpu: %s\n", e.what());
        return -1;
    }
    return 0;
}
#endif

// The reference's time resamplers (operator.cpp:760-856) on ntr traces:
// domain axis (nm samples at dm), range axis (np samples at dp), both from
// t = 0.  adjoint = 0: in [ntr][nm] -> out [ntr][np] (apply_forward);
// adjoint = 1: in [ntr][np] -> out [ntr][nm] (apply_adjoint).  add = false.
int ref_resample(int linear, int adjoint, int hl, int ntr, int nm, double dm, int np_, double dp, const data_t *in,
                 data_t *out)
{
    try {
        hypercube<data_t> dom(axis<data_t>(nm, 0, (data_t)dm), axis<data_t>(ntr, 0, 1));
        hypercube<data_t> rng(axis<data_t>(np_, 0, (data_t)dp), axis<data_t>(ntr, 0, 1));
        resampler *r;
        if (linear) r = new linear_resampler(dom, rng);
        else r = new sinc_resampler(dom, rng, hl);
        if (!adjoint) r->apply_forward(false, in, out);
        else r->apply_adjoint(false, out, in);
        delete r;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_resample: %s\n", e.what());
        return -1;
    }
    return 0;
}

// The acoustic-elastic solver gradient (nl_we_op_ae through nl_we_op_e's
// apply_forward / apply_jacobianT): model [3][nx][nz] (vp, vs, rho) on a grid
// whose first row is at depth oz, the fluid layer above it; one source at
// (sx, sz) (in the fluid when acoustic_source, its traces [1][nt], else on the
// elastic grid, [2][nt]); nr receivers at (rx, rz) on the elastic grid and
// (rx, rzw) in the fluid.  Data [3][nr][nt] (fluid, x, z), seismotype 1.
static int misfit_grad_ae(const ref_param *rp, int nx, int nz, double dx, double dz, double oz, int nt, double dt,
                          double prop_dt, const char *resampling, data_t sx, data_t sz, int nr, const data_t *rx,
                          const data_t *rz, const data_t *rzw, const data_t *model, const data_t *src,
                          const data_t *obs, data_t *syn, data_t *grad)
{
    try {
        param par = to_param(rp);
        par.nt = nt;
        par.dt = (data_t)prop_dt;
        par.sub = obs ? 1 : 0;
        par.ns = 1;
        par.nr = nr;
        par.nmodels = 3;
        par.acoustic_elastic = true;
        par.seismotype = 1;
        par.resampling = resampling;
        data_t sl[2] = {sx, sz};
        par.sxz = locs(1, sl, sl + 1);
        par.rxz = {locs(nr, rx, rz)};
        std::vector<data_t> rxw(rx, rx + nr);
        par.rxza = {locs(nr, rxw.data(), rzw)};
        hypercube<data_t> dom(axis<data_t>(nz, (data_t)oz, (data_t)dz), axis<data_t>(nx, 0, (data_t)dx),
                              axis<data_t>(3, 0, 1));
        const int ncs = par.acoustic_source ? 1 : 2;
        auto allsrc = std::make_shared<vecReg<data_t> >(hypercube<data_t>(axis<data_t>(nt, 0, (data_t)dt), axis<data_t>(ncs, 0, 1)));
        std::memcpy(allsrc->getVals(), src, ncs * (size_t)nt * sizeof(data_t));
        auto op = std::make_shared<nl_we_op_ae>(dom, allsrc, par);
        auto m = std::make_shared<vecReg<data_t> >(dom);
        std::memcpy(m->getVals(), model, m->getN123() * sizeof(data_t));
        auto d = std::make_shared<vecReg<data_t> >(*op->getRange());
        op->forward(false, m, d);
        std::memcpy(syn, d->getCVals(), d->getN123() * sizeof(data_t));
        if (obs) {
            auto r = std::make_shared<vecReg<data_t> >(*op->getRange());
            data_t *pr = r->getVals();
            const long n = (long)r->getN123();
            for (long i = 0; i < n; i++) pr[i] = syn[i] - obs[i];
            applyHt(false, false, pr, pr, 3 * nr, nt, (data_t)dt, 0, 3 * nr);
            auto g = std::make_shared<vecReg<data_t> >(dom);
            op->jacobianT(false, g, m, r);
            std::memcpy(grad, g->getCVals(), g->getN123() * sizeof(data_t));
        }
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_misfit_grad_ae: %s\n", e.what());
        return -1;
    }
    return 0;
}

int ref_misfit_grad_ae(const ref_param *rp, int nx, int nz, double dx, double dz, double oz, int nt, double dt,
                       data_t sx, data_t sz, int nr, const data_t *rx, const data_t *rz, const data_t *rzw,
                       const data_t *model, const data_t *src, const data_t *obs, data_t *syn, data_t *grad)
{
    return misfit_grad_ae(rp, nx, nz, dx, dz, oz, nt, dt, dt, "linear", sx, sz, nr, rx, rz, rzw, model, src, obs, syn,
                          grad);
}

// ref_misfit_grad_ae with sources and data on their own axis (nd samples at
// dd), the propagation at prop_dt, and the sinc (linear = 0, half length 11)
// or linear resampler, as ref_misfit_grad_rs.
int ref_misfit_grad_ae_rs(const ref_param *rp, int nx, int nz, double dx, double dz, double oz, int nd, double dd,
                          double prop_dt, int linear, data_t sx, data_t sz, int nr, const data_t *rx,
                          const data_t *rz, const data_t *rzw, const data_t *model, const data_t *src,
                          const data_t *obs, data_t *syn, data_t *grad)
{
    return misfit_grad_ae(rp, nx, nz, dx, dz, oz, nd, dd, prop_dt, linear ? "linear" : "sinc", sx, sz, nr, rx, rz, rzw,
                          model, src, obs, syn, grad);
}

// kind: 0 elastic, 1 VTI, 2 acoustic, 3 acoustic-elastic.
// inj/ext locations are on the (elastic) grid; for kind 3 the water-layer
// source (sa) and receiver (ra) locations are passed too.
int ref_propagate(int kind, int adj, const data_t *model, const data_t *allsrc, data_t *allrcv,
                  int inj_type, int ninj, const data_t *ix, const data_t *iz,
                  int next, const data_t *ex, const data_t *ez,
                  int nsa, const data_t *sax, const data_t *saz, int nra, const data_t *rax, const data_t *raz,
                  data_t *full, data_t *grad, const ref_param *rp, int nx, int nz,
                  double dx, double dz, double ox, double oz)
{
    try {
        param par = to_param(rp);
        hypercube<data_t> g = grid(nx, nz, dx, dz, ox, oz);
        injector *inj = nullptr, *ext = nullptr;
        if (ninj > 0) inj = inj_type == 0 ? (injector *)new delta_m3(g, locs(ninj, ix, iz)) : (injector *)new ddelta_m3(g, locs(ninj, ix, iz));
        if (next > 0) ext = new delta_m3(g, locs(next, ex, ez));
        if (kind == 3) {
            par.sxz = locs(nsa, sax, saz);
            par.rxza = {locs(nra, rax, raz)};
            par.rxz = {locs(next, ex, ez)};
        }
        if (kind == 0) { nl_we_op_e op; op.propagate(adj != 0, model, allsrc, allrcv, inj, ext, full, grad, par, nx, nz, (data_t)dx, (data_t)dz, (data_t)ox, (data_t)oz, 0); }
        else if (kind == 1) { nl_we_op_vti op; op.propagate(adj != 0, model, allsrc, allrcv, inj, ext, full, grad, par, nx, nz, (data_t)dx, (data_t)dz, (data_t)ox, (data_t)oz, 0); }
        else if (kind == 2) { nl_we_op_a op; op.propagate(adj != 0, model, allsrc, allrcv, inj, ext, full, grad, par, nx, nz, (data_t)dx, (data_t)dz, (data_t)ox, (data_t)oz, 0); }
        else if (kind == 3) { nl_we_op_ae op; op.propagate(adj != 0, model, allsrc, allrcv, inj, ext, full, grad, par, nx, nz, (data_t)dx, (data_t)dz, (data_t)ox, (data_t)oz, 0); }
        delete inj;
        delete ext;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_propagate: %s\n", e.what());
        return -1;
    }
    return 0;
}


// A full-waveform inversion run of the reference's own solver stack, as
// main/fwi2d.cpp:234-356 assembles it with no model preconditioner,
// regularization, mask, weights or filter: nlls_fwi_eco
// (optimization.hpp:462-915) over the wave-equation operator of `kind`
// (0 elastic, 1 VTI, 2 acoustic, 3 acoustic-elastic) and the lbfgs solver
// (nlsolver.hpp:308-335, nlsolver.cpp:1207-1345) with the regular_wolfe line
// search, the parameter defaults of param.hpp:58-73 (c1 = 1e-4, c2 = 0.9,
// a0 = 1, max step 1e6, 10 trials, 5 pairs) and the initial step fraction
// ls_a1 of the model norm, for niter iterations.  ns shots at (sx[s], sz[s]);
// every shot records the same nr receivers at (rx, rz) -- for kind 3 also at
// (rx, rzw) in the fluid layer above the grid, whose first row lies at depth
// oz.  src is the reference's allsrc [ncs][ns][nt]; obs [nc][ns * nr][nt] (the
// operator's range: component, then shot-major traces); model
// [npar][nx][nz] holds the starting model (vp, vs, rho ...) on input and the
// final model on output; func receives the objective function of every
// iteration (at most niter + 1 values).  Returns the number of values, or -1.
int ref_fwi_lbfgs(int kind, const ref_param *rp, int nx, int nz, double dx, double dz, double oz, int nt, double dt,
                  int ns, const data_t *sx, const data_t *sz, int nr, const data_t *rx, const data_t *rz,
                  const data_t *rzw, const data_t *src, const data_t *obs, data_t *model, int niter, double ls_a1,
                  data_t *func)
{
    try {
        param par = to_param(rp);
        par.nt = nt;
        par.dt = (data_t)dt;
        par.sub = rp->sub > 0 ? rp->sub : 1;
        par.ns = ns;
        par.nr = ns * nr;
        par.nmodels = kind == 1 ? 5 : (kind == 2 ? 2 : 3);
        par.acoustic_elastic = kind == 3;
        par.seismotype = 1;
        par.resampling = "linear";
        par.niter = niter;
        par.verbose = 0;
        par.sxz.clear();
        par.rxz.clear();
        par.rxza.clear();
        for (int s = 0; s < ns; s++) {
            par.sxz.push_back({sx[s], sz[s], 0});
            par.rxz.push_back(locs(nr, rx, rz));
            if (kind == 3) par.rxza.push_back(locs(nr, rx, rzw));
        }
        const int ncs = (kind == 2 || (kind == 3 && par.acoustic_source)) ? 1 : 2;
        hypercube<data_t> dom(axis<data_t>(nz, (data_t)oz, (data_t)dz), axis<data_t>(nx, 0, (data_t)dx),
                              axis<data_t>(par.nmodels, 0, 1));
        auto allsrc = std::make_shared<vecReg<data_t> >(
            hypercube<data_t>(axis<data_t>(nt, 0, (data_t)dt), axis<data_t>(ns, 0, 1), axis<data_t>(ncs, 0, 1)));
        std::memcpy(allsrc->getVals(), src, (size_t)ncs * ns * nt * sizeof(data_t));
        std::unique_ptr<nl_we_op> L;
        if (kind == 0) L.reset(new nl_we_op_e(dom, allsrc, par));
        else if (kind == 1) L.reset(new nl_we_op_vti(dom, allsrc, par));
        else if (kind == 2) L.reset(new nl_we_op_a(dom, allsrc, par));
        else L.reset(new nl_we_op_ae(dom, allsrc, par));
        auto m = std::make_shared<vecReg<data_t> >(dom);
        std::memcpy(m->getVals(), model, m->getN123() * sizeof(data_t));
        auto d = std::make_shared<vecReg<data_t> >(*L->getRange());
        std::memcpy(d->getVals(), obs, d->getN123() * sizeof(data_t));
        nlls_fwi_eco prob(L.get(), m, d);
        regular_wolfe ls(par.ls_c1, par.ls_c2, par.ls_a0, (data_t)ls_a1, par.ls_max_step, par.ls_version);
        lbfgs solver(niter, par.max_trial, par.threshold, &ls, nullptr, par.lbfgs_m);
        solver.run(&prob, false, "none", par.isave, par.format, "none");
        std::memcpy(model, m->getCVals(), m->getN123() * sizeof(data_t));
        const int nf = (int)std::min<size_t>(solver._func.size(), (size_t)niter + 1);
        for (int i = 0; i < nf; i++) func[i] = solver._func[i];
        return nf;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_fwi_lbfgs: %s\n", e.what());
        return -1;
    }
}

}
