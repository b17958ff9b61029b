// Acoustic (variable density) step kernel: pressure p, model (K, 1/rho).
//
// One launch advances every shot of a batch by one time step, one CTA per
// 32 x TX tile (windows and ownership as in the elastic tile kernel), and
// performs the reference's step (src/cpp/we_op.cpp:1937-2134):
//   next = Dxx_var(1/rho) curr + Dzz_var(1/rho) curr + sources,
//   the acoustic SAT of each side in order (spatial_operators.cpp:551-860:
//   pressure release with stiffness alpha for bc 1, absorbing for bc 2,
//   rigid for bc 3), next = dt^2 K next + 2 curr - prev, the implicit
//   absorbing scaling and the cos^2 taper,
// plus receiver extraction and snapshot storage (forward) or the zero-lag
// imaging condition of nl_we_op_a::compute_gradients (we_op.cpp:1883-1935),
// which uses the adjoint field at the start of the step (adjoint).
#pragma once

namespace fwi2d {

// One SAT side of the acoustic step at one cell (x, z); `side` 0 top,
// 1 bottom, 2 left, 3 right.  U / IR point at the cell inside the tile
// arrays, su / sw are the strides across the side (into the domain), k the
// cell's distance from the side.
__device__ __forceinline__ float asat_cell(float n, int side, int bc, int k, const float *U, int su, const float *IR,
                                           int sw, float p, float K, const StepConst &C)
{
    const bool zside = side < 2;
    const float d = zside ? C.dz : C.dx;
    const float d2 = zside ? C.d2z : C.d2x;
    if (bc == 1) {
        if (k < 4) {
            // the side's boundary sample of this line feeds the first four cells (asat_dirichlet_*)
            const float in = U[-k * su], ir = IR[-k * sw];
            n = (float)((double)n + 1.0 / (double)(kHC[k] * d2) * (double)kSC[k] * (double)ir * (double)in);
        }
        if (k == 0) n = n - IR[0] * U[0] / (C.alpha * kHC[0] * d2);
    } else if (k == 0) {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j < 4; j++) s += kSC[j] * U[j * su];
        const double a = 1.0 / (double)(kHC[0] * d);
        if (bc == 2)
            n = (float)((double)n - a * ((double)(IR[0] * s / d) - (double)p / ((double)(2 * C.dt) * sqrt((double)(K / IR[0])))));
        else
            n = (float)((double)n - a * (double)IR[0] * (double)s / (double)d);
    }
    return n;
}

// AE: the fluid layer of the acoustic-elastic propagator (we_op.cpp:2137-2577):
// the bottom edge is the interface (Neumann SAT, C.bc[1] = 3) applied after
// the left and right sides, and the interface row is left untapered, with its
// prev saved in halo_save, for ae_couple.
template <int TX, bool GRAD, bool AE>
__global__ void __launch_bounds__(32 * TX)
acoustic_step(const ShotDev *__restrict__ shots, const TileRef *__restrict__ tiles, ModelDev M, StepConst C, int it,
              int flags, float dtg)
{
    constexpr int TZ = 32, UZ = TZ + 8, UX = TX + 8, WZ = TZ + 4, WX = TX + 4, NT = 32 * TX;
    __shared__ float U[UX * UZ];                  // curr, 4-cell halo
    __shared__ float IR[WX * WZ];                 // 1/rho, 2-cell halo
    __shared__ float F[GRAD ? WX * WZ : 1];       // forward snapshot of the imaging condition
    __shared__ float red[NT / 32];

    const TileRef tr = tiles[blockIdx.x];
    const ShotDev *__restrict__ Sp = shots + tr.shot;
    const int nt = Sp->nt;
    if (it >= nt - 1) return;
    const int nx = Sp->nx, nz = Sp->nz, ldz = Sp->ldz, mld = M.ldz;
    const int wx0 = tr.wx0, wz0 = tr.wz0;
    const float *__restrict__ curr = Sp->u[(it + 1) & 1];
    float *__restrict__ pn = Sp->u[it & 1];
    const long long mofs = (long long)Sp->x0 * mld;
    const float *__restrict__ Km = M.p0 + mofs;
    const float *__restrict__ Im = M.p1 + mofs;
    const int prec = C.snap_prec;
    // imaging condition of this step: snapshot (nt-1-it)/sub, skipped at it == 0 (we_op.cpp:2044-2046)
    const int itf = GRAD ? (nt - 1 - it) / C.sub : 0;
    const bool do_grad = GRAD && (flags & F_GRAD) && it != 0 && ((nt - 1 - it) % C.sub == 0);
    float finv = 1.f;
    if (GRAD && do_grad && prec != SNAP_FP32) finv = 1.f / snap_scale(Sp->snap_amax, itf);

    for (int i = threadIdx.x; i < UX * UZ; i += NT) {
        const int sx = i / UZ, sz = i - sx * UZ;
        const int gx = wx0 - 4 + sx, gz = wz0 - 4 + sz;
        U[i] = (gx >= 0 && gx < nx && gz >= 0 && gz < nz) ? curr[(long long)gx * ldz + gz] : 0.f;
    }
    for (int i = threadIdx.x; i < WX * WZ; i += NT) {
        const int sx = i / WZ, sz = i - sx * WZ;
        const int gx = wx0 - 2 + sx, gz = wz0 - 2 + sz;
        const bool in = gx >= 0 && gx < nx && gz >= 0 && gz < nz;
        IR[i] = in ? Im[(long long)gx * mld + gz] : 0.f;
        if (GRAD) F[i] = (in && do_grad) ? snap_load(Sp->snap, (long long)itf * Sp->snap_slot + (long long)gx * ldz + gz,
                                                      prec, finv)
                                         : 0.f;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile_id = tr.unit;
    if (flags & F_EXTRACT) {
        const int e0 = Sp->ext_off[tile_id], e1 = Sp->ext_off[tile_id + 1];
        for (int e = e0 + threadIdx.x; e < e1; e += NT) {
            const ExtEntry &E = Sp->ext[e];
            const int base = (E.gx0 - wx0 + 4) * UZ + (E.gz0 - wz0 + 4);
            float o = 0.f;
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++) o += E.w[a * 3 + b] * U[base + a * UZ + b];
            Sp->rcv[(long long)it * Sp->nrcv + E.row] = o;
        }
    }
    const int e0 = Sp->inj_off[tile_id], e1 = Sp->inj_off[tile_id + 1];
    const float *srcrow = Sp->src + (long long)it * Sp->nsrc;
    const bool store = (flags & F_STORE) && (it % C.sub == 0);
    float amax = 0.f;

    const int tz = lane, tx = warp;
    const int gx = wx0 + tx, gz = wz0 + tz;
    if (gx >= tr.ox0 && gx < tr.ox1 && gz >= tr.oz0 && gz < tr.oz1) {
        const int ui = (tx + 4) * UZ + (tz + 4);
        const int wi = (tx + 2) * WZ + (tz + 2);
        const long long cell = (long long)gx * ldz + gz;
        const long long mcell = (long long)gx * mld + gz;
        if (store) {
            const int slot = it / C.sub;
            const float sc = prec == SNAP_FP32 ? 1.f : snap_scale(Sp->snap_amax, slot);
            snap_store(Sp->snap, (long long)slot * Sp->snap_slot + cell, prec, U[ui], sc);
        }
        if (GRAD && do_grad) {
            const float t0 = d1(F + wi, WZ, gx, nx, C.dx, C.sdx);
            const float t1 = d1(F + wi, 1, gz, nz, C.dz, C.sdz);
            const float t2 = d1(U + ui, UZ, gx, nx, C.dx, C.sdx);
            const float t3 = d1(U + ui, 1, gz, nz, C.dz, C.sdz);
            const float f = F[wi], adj = U[ui], K = Km[mcell];
            const int last = nt / C.sub;
            float fp = 0.f, fm = 0.f;
            if (itf + 1 <= last) {
                const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf + 1);
                fp = snap_load(Sp->snap, (long long)(itf + 1) * Sp->snap_slot + cell, prec, inv);
            }
            if (itf > 0) {
                const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(Sp->snap_amax, itf - 1);
                fm = snap_load(Sp->snap, (long long)(itf - 1) * Sp->snap_slot + cell, prec, inv);
            }
            const float w = Sp->gwt[itf];
            const double c = (double)w * 1.0 / (double)(dtg * K * K) * (double)adj;
            float *g0 = Sp->grad + cell, *g1 = g0 + (long long)nx * ldz;
            if (itf > 0 && itf < last) {
                *g0 = (float)((double)*g0 - c * (double)(fp - 2 * f + fm));
                *g1 += w * dtg * (t2 * t0 + t3 * t1);
            } else if (itf == 0) {
                *g0 = (float)((double)*g0 - c * (double)(fp - f));
                *g1 = (float)((double)*g1 + (double)w * 0.5 * (double)dtg * (double)(t2 * t0 + t3 * t1));
            } else {
                *g0 = (float)((double)*g0 - c * (double)(-f + fm));
                *g1 += w * dtg * (t2 * t0 + t3 * t1);
            }
        }

        float n = 0.f;
        d2acc(n, U + ui, UZ, IR + wi, WZ, 1.f, gx, nx, C.inv_d2x, C.d2x);
        d2acc(n, U + ui, 1, IR + wi, 1, 1.f, gz, nz, C.inv_d2z, C.d2z);
        for (int e = e0; e < e1; e++) {
            const InjEntry &E = Sp->inj[e];
            if (E.gx == gx && E.gz == gz) n += E.wa * srcrow[E.ia];
        }
        const float tzv = Sp->tz[gz], txv = Sp->tx[gx];
        float p = pn[cell];
        if (it > 0) p = p * tzv * txv;
        const float K = Km[mcell];
        if (C.bc[0] >= 1 && C.bc[0] <= 3 && gz < 4) n = asat_cell(n, 0, C.bc[0], gz, U + ui, 1, IR + wi, 1, p, K, C);
        if (!AE && C.bc[1] >= 1 && C.bc[1] <= 3 && gz >= nz - 4)
            n = asat_cell(n, 1, C.bc[1], nz - 1 - gz, U + ui, -1, IR + wi, -1, p, K, C);
        if (C.bc[2] >= 1 && C.bc[2] <= 3 && gx < 4) n = asat_cell(n, 2, C.bc[2], gx, U + ui, UZ, IR + wi, WZ, p, K, C);
        if (C.bc[3] >= 1 && C.bc[3] <= 3 && gx >= nx - 4)
            n = asat_cell(n, 3, C.bc[3], nx - 1 - gx, U + ui, -UZ, IR + wi, -WZ, p, K, C);
        if (AE && C.bc[1] >= 1 && C.bc[1] <= 3 && gz >= nz - 4)
            n = asat_cell(n, 1, C.bc[1], nz - 1 - gz, U + ui, -1, IR + wi, -1, p, K, C);
        n = C.dt2 * n * K + 2 * U[ui] - p;
        if (gz == 0 || gz == nz - 1 || gx == 0 || gx == nx - 1) {
            int k;
            if (gz == 0) k = gx;
            else if (gz == nz - 1) k = nx + gx;
            else if (gx == 0) k = 2 * nx + gz;
            else k = 2 * nx + nz + gz;
            n = n / Sp->den[k];
        }
        if (AE && gz == nz - 1) Sp->halo_save[gx] = p;   // interface row: coupled and tapered by ae_couple
        else n = n * tzv * txv;
        pn[cell] = n;
        amax = fabsf(n);
    }

    if ((flags & F_AMAX) && ((it + 1) % C.sub == 0)) {
        float m = amax;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) red[warp] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < NT / 32; w++) m = fmaxf(m, red[w]);
            m = fmaxf(m, red[0]);
            if (m > 0.f) atomicMax(Sp->snap_amax + (it + 1) / C.sub, __float_as_uint(m));
        }
    }
}

// Imaging condition with the adjoint field after the last step (snapshot 0;
// we_op.cpp:2132).  One thread per cell.
__global__ void acoustic_final_grad(const ShotDev *__restrict__ shots, int nshots, ModelDev M, StepConst C, float dtg)
{
    const ShotDev &S = shots[blockIdx.y];
    if (blockIdx.y >= nshots) return;
    const int nx = S.nx, nz = S.nz, ldz = S.ldz;
    const float *adj = S.u[S.nt & 1];   // the field after launch nt-2 is curr at time nt-1
    const int prec = C.snap_prec;
    const int last = S.nt / C.sub;
    const float finv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(S.snap_amax, 0);
    const float finvp = prec == SNAP_FP32 || last < 1 ? 1.f : 1.f / snap_scale(S.snap_amax, 1);
    const long long n = (long long)nx * nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int gx = (int)(i / nz), gz = (int)(i - (long long)gx * nz);
        const long long cell = (long long)gx * ldz + gz;
        // snapshot 0 through a small gather: the first derivatives need their closures
        float fx[6], fz[6], ax[6], az[6];
        const int bx = gx < 4 ? 0 : (gx >= nx - 4 ? nx - 6 : gx - 2);
        const int bz = gz < 4 ? 0 : (gz >= nz - 4 ? nz - 6 : gz - 2);
        for (int k = 0; k < 6; k++) {
            const int xx = min(bx + k, nx - 1), zz = min(bz + k, nz - 1);
            fx[k] = snap_load(S.snap, (long long)xx * ldz + gz, prec, finv);
            fz[k] = snap_load(S.snap, (long long)gx * ldz + zz, prec, finv);
            ax[k] = adj[(long long)xx * ldz + gz];
            az[k] = adj[(long long)gx * ldz + zz];
        }
        const float t0 = d1(fx + (gx - bx), 1, gx, nx, C.dx, C.sdx);
        const float t1 = d1(fz + (gz - bz), 1, gz, nz, C.dz, C.sdz);
        const float t2 = d1(ax + (gx - bx), 1, gx, nx, C.dx, C.sdx);
        const float t3 = d1(az + (gz - bz), 1, gz, nz, C.dz, C.sdz);
        const float f = fx[gx - bx], a = adj[cell];
        const float K = M.p0[(long long)S.x0 * M.ldz + (long long)gx * M.ldz + gz];
        float fp = 0.f;
        if (1 <= last) fp = snap_load(S.snap, S.snap_slot + cell, prec, finvp);
        const float w = S.gwt[0];
        const double c = (double)w * 1.0 / (double)(dtg * K * K) * (double)a;
        float *g0 = S.grad + cell, *g1 = g0 + (long long)nx * ldz;
        *g0 = (float)((double)*g0 - c * (double)(fp - f));
        *g1 = (float)((double)*g1 + (double)w * 0.5 * (double)dtg * (double)(t2 * t0 + t3 * t1));
    }
}

}  // namespace fwi2d

namespace fwi2d {

// Implicit coupling of the fluid potential and the elastic uz at the
// interface (we_op.cpp:2486-2512, the it >= 0 branch), after both launches of
// the step, then the taper of the two interface rows.  One thread per column.
// E, W: the elastic and fluid tables of each shot; prev of both interface rows
// (already tapered) is in halo_save.  sign = +1 forward, -1 adjoint.  With
// F_GRAD, the density term of the imaging condition on the interface row,
// which needs the coupled uz (the elastic kernel leaves it out there).
__global__ void ae_couple(const ShotDev *__restrict__ E, const ShotDev *__restrict__ W, int nshots, ModelDev M,
                          StepConst C, int it, int flags, float dtg, float Kw, float val0, int sign)
{
    const int s = blockIdx.y;
    if (s >= nshots) return;
    const ShotDev &e = E[s], &w = W[s];
    if (it >= e.nt - 1) return;
    const long long nxz = (long long)e.nx * e.ldz;
    float *n1 = e.u[it & 1] + nxz;              // next uz, row 0
    float *na = w.u[it & 1] + (w.nz - 1);       // next potential, last fluid row
    for (int ix = blockIdx.x * blockDim.x + threadIdx.x; ix < e.nx; ix += gridDim.x * blockDim.x) {
        const long long ie = (long long)ix * e.ldz, ia = (long long)ix * w.ldz;
        const float p1 = e.halo_save[ix], pa = w.halo_save[ix];
        const float rho = M.p2[(long long)(e.x0 + ix) * M.ldz];
        const float v1 = Kw * val0 * (n1[ie] - p1 + sign * val0 / rho * pa);
        const float v2 = 1 + val0 * val0 * Kw / rho;
        const float a = (na[ia] + sign * v1) / v2;
        const float b = n1[ie] - sign * val0 / rho * (a - pa);
        na[ia] = a * w.tz[w.nz - 1] * w.tx[ix];
        const float a1 = b * e.tz[0] * e.tx[ix];
        n1[ie] = a1;
        const int tt = e.nt - 1 - (it + 1);
        if ((flags & F_GRAD) && tt % C.sub == 0 && tt / C.sub != 0) {
            // density term at snapshot itf with the coupled next field, as the
            // elastic kernel's (nl_we_op_e::compute_gradients, we_op.cpp:505-562)
            const int itf = tt / C.sub, last = e.nt / C.sub, prec = C.snap_prec;
            const float inv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(e.snap_amax, itf);
            const long long o = (long long)itf * e.snap_slot + ie;
            const float f0 = snap_load(e.snap, o, prec, inv), f1 = snap_load(e.snap, o + nxz, prec, inv);
            float fp0 = 0.f, fp1 = 0.f, fm0 = 0.f, fm1 = 0.f;
            if (itf + 1 <= last) {
                const float iv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(e.snap_amax, itf + 1);
                const long long op = (long long)(itf + 1) * e.snap_slot + ie;
                fp0 = snap_load(e.snap, op, prec, iv);
                fp1 = snap_load(e.snap, op + nxz, prec, iv);
            }
            {
                const float iv = prec == SNAP_FP32 ? 1.f : 1.f / snap_scale(e.snap_amax, itf - 1);
                const long long om = (long long)(itf - 1) * e.snap_slot + ie;
                fm0 = snap_load(e.snap, om, prec, iv);
                fm1 = snap_load(e.snap, om + nxz, prec, iv);
            }
            const float a0 = e.u[it & 1][ie];
            const float gw = e.gwt[itf];
            const double wdt = (double)gw * 1.0 / (double)dtg;
            float *g2 = e.grad + 2 * nxz + ie;
            if (itf < last)
                *g2 = (float)((double)*g2 + wdt * (double)(a0 * (fp0 - 2 * f0 + fm0) + a1 * (fp1 - 2 * f1 + fm1)));
            else
                *g2 = (float)((double)*g2 + wdt * (double)(a0 * (-f0 + fm0) + a1 * (-f1 + fm1)));
        }
    }
}

}  // namespace fwi2d
