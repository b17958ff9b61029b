// we_op_b200.cpp -- the reference's GPU hook routed to fwi2d_b200.
//
// A maintainer of the reference adds this file to its source tree and builds
// the reference with CUDA defined: apply_forward and
// apply_jacobianT of the wave-equation operators then call the virtual
// propagate_gpu (src/cpp/we_op.cpp:994-998, 1170-1174, 1301-1302, 1419-1420)
// instead of propagate, and this file implements that hook -- declared in
// src/include/we_op.hpp:82 (nl_we_op_e, inherited by nl_we_op_a and
// nl_we_op_ae) and :174 (nl_we_op_vti) -- on fwi2d_propagate.  It replaces
// src/cuda/cudaWeOp.cpp and cudaKernels.cu (or src/cpp/dummy.cpp in a CPU
// build); the solver, I/O, bounds and B-spline code stay as they are.
//
// Compiled against the reference's headers (we_op.hpp, injector.hpp,
// param.hpp, vecReg.hpp) and include/fwi2d_b200.h; linked with
// libfwi2d_b200.so.  oracle/build_ref.sh builds it that way for the tests.
#include <memory>
#include <stdexcept>
#include <vector>

#include "we_op.hpp"
#include "fwi2d_b200.h"

namespace {

// The injector's public tables (src/include/injector.hpp:9-13), viewed in place.
fwi2d_injector view(const injector *J)
{
    fwi2d_injector v = {};
    if (!J) return v;
    v.type = FWI2D_INJ_DELTA;
    if (dynamic_cast<const ddelta_m3 *>(J)) v.type = FWI2D_INJ_DDELTA;
    if (dynamic_cast<const dipole_m3 *>(J)) v.type = FWI2D_INJ_DIPOLE;   // DAS receivers (elastic, VTI)
    v.ntr = J->_ntr;
    v.xind = J->_xind.data();
    v.zind = J->_zind.data();
    v.xw = J->_xw.data();
    v.zw = J->_zw.data();
    return v;
}

// The fields of the reference's param (src/include/param.hpp) the propagation reads.
fwi2d_params params(const param &par)
{
    fwi2d_params p = {};
    p.nt = par.nt;
    p.sub = par.sub;
    p.dt = par.dt;
    p.bc_top = par.bc_top;
    p.bc_bottom = par.bc_bottom;
    p.bc_left = par.bc_left;
    p.bc_right = par.bc_right;
    p.taper_top = par.taper_top;
    p.taper_bottom = par.taper_bottom;
    p.taper_left = par.taper_left;
    p.taper_right = par.taper_right;
    p.taper_strength = par.taper_strength;
    p.free_surface_stiffness = par.free_surface_stiffness;
    p.mt = par.mt;
    p.gdamp_tmin = par.gdamp_tmin;
    p.gdamp_tmax = par.gdamp_tmax;
    p.gdamp_power = par.gdamp_power;
    p.snapshot_precision = FWI2D_SNAP_FP32;   // the host owns FP32 snapshots in full_wfld
    p.tile_shape = -1;                        // autotuned
    return p;
}

void run(int kind, bool adj, const data_t *model, const data_t *allsrc, data_t *allrcv, const injector *inj,
         const injector *ext, data_t *full, data_t *grad, const param &par, int nx, int nz, data_t dx, data_t dz,
         data_t ox, int s)
{
    if (par.version != 2 && kind != FWI2D_ACOUSTIC_ELASTIC)
        throw std::logic_error("fwi2d_b200: version-2 operators only (the acoustic-elastic operator's own split)");
    if (par.pml) throw std::logic_error("fwi2d_b200: SAT and taper boundaries only (pml = 0)");
    fwi2d_params p = params(par);
    const fwi2d_injector vi = view(inj), ve = view(ext);
    fwi2d_injector va = {}, vb = {};
    const fwi2d_injector *pa = nullptr, *pb = nullptr;
    std::unique_ptr<delta_m3> ia, ea;
    if (kind == FWI2D_ACOUSTIC_ELASTIC) {
        // the fluid layer's injectors, built as nl_we_op_ae::propagate builds them (we_op.cpp:2244-2254)
        p.nza = par.nza;
        p.water_velocity = par.water_velocity;
        p.water_density = par.water_density;
        p.acoustic_source = par.acoustic_source;
        hypercube<data_t> domaina(axis<data_t>(par.nza, 0, dz), axis<data_t>(nx, ox, dx));
        const std::vector<std::vector<data_t>> src = {par.sxz[s]};
        if (!adj) {
            if (par.acoustic_source) ia.reset(new delta_m3(domaina, src));
            ea.reset(new delta_m3(domaina, par.rxza[s]));
        } else {
            if (par.acoustic_source) ea.reset(new delta_m3(domaina, src));
            ia.reset(new delta_m3(domaina, par.rxza[s]));
        }
        if (ia) {
            va = view(ia.get());
            pa = &va;
        }
        if (ea) {
            vb = view(ea.get());
            pb = &vb;
        }
    }
    const int rc = fwi2d_propagate(kind, adj ? 1 : 0, model, allsrc, allrcv, inj ? &vi : nullptr, ext ? &ve : nullptr,
                                   pa, pb, full, grad, &p, par.ns, par.nr, nx, nz, dx, dz);
    if (rc != FWI2D_OK) throw std::logic_error(fwi2d_last_error());   // successCheck's exception type
}

}  // namespace

// nl_we_op_a and nl_we_op_ae inherit apply_forward / apply_jacobianT and this
// hook from nl_we_op_e (we_op.hpp:233, :318): dispatch on the dynamic type.
void nl_we_op_e::propagate_gpu(bool adj, const data_t *model, const data_t *allsrc, data_t *allrcv,
                               const injector *inj, const injector *ext, data_t *full_wfld, data_t *grad,
                               const param &par, int nx, int nz, data_t dx, data_t dz, data_t ox, data_t, int s) const
{
    int kind = FWI2D_ELASTIC;
    if (dynamic_cast<const nl_we_op_ae *>(this)) kind = FWI2D_ACOUSTIC_ELASTIC;
    else if (dynamic_cast<const nl_we_op_a *>(this)) kind = FWI2D_ACOUSTIC;
    run(kind, adj, model, allsrc, allrcv, inj, ext, full_wfld, grad, par, nx, nz, dx, dz, ox, s);
}

void nl_we_op_vti::propagate_gpu(bool adj, const data_t *model, const data_t *allsrc, data_t *allrcv,
                                 const injector *inj, const injector *ext, data_t *full_wfld, data_t *grad,
                                 const param &par, int nx, int nz, data_t dx, data_t dz, data_t ox, data_t, int s) const
{
    run(FWI2D_VTI, adj, model, allsrc, allrcv, inj, ext, full_wfld, grad, par, nx, nz, dx, dz, ox, s);
}

// The imaging condition is fused into the adjoint propagation.
void nl_we_op_e::compute_gradients_gpu(const data_t *, const data_t *, const data_t *, const data_t *, const data_t *,
                                       data_t *, data_t *, const param &, int, int, int, data_t, data_t, data_t) const
{
}
void nl_we_op_vti::compute_gradients_gpu(const data_t *, const data_t *, const data_t *, const data_t *,
                                         const data_t *, data_t *, data_t *, const param &, int, int, int, data_t,
                                         data_t, data_t) const
{
}

// The injectors' per-sample GPU hooks are not used: injection and extraction
// run inside the step kernels.
void delta_m3::inject_gpu(bool, const data_t **, data_t *, int, int, int, int, int, int, int, const int *, const int *,
                          const data_t *, const data_t *) const
{
}
void delta_m3::extract_gpu(bool, const data_t *, data_t **, int, int, int, int, int, int, int, const int *,
                           const int *, const data_t *, const data_t *) const
{
}
void ddelta_m3::inject_gpu(bool, const data_t **, data_t *, int, int, int, int, int, int, int, const int *,
                           const int *, const data_t *, const data_t *) const
{
}
void ddelta_m3::extract_gpu(bool, const data_t *, data_t **, int, int, int, int, int, int, int, const int *,
                            const int *, const data_t *, const data_t *) const
{
}
void dipole_m3::inject_gpu(bool, const data_t **, data_t *, int, int, int, int, int, int, int, const int *,
                           const int *, const data_t *, const data_t *) const
{
}
void dipole_m3::extract_gpu(bool, const data_t *, data_t **, int, int, int, int, int, int, int, const int *,
                            const int *, const data_t *, const data_t *) const
{
}
