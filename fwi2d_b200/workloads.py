"""Seeded synthetic stand-ins for the benchmark configurations.

No dataset ships with the reference; these generate the shapes, sizes and
value distributions the configurations describe, in the reference's units
(km, s, km/s, g/cm^3):

* elastic_single  -- 401 x 801 grid at 5 m, vp = 2 + 0.75 z km/s with a
  +-5 % smoothed random perturbation (sigma 50 m), vs = vp/1.73,
  rho = 0.31 (1000 vp)^0.25; Ricker 10 Hz delayed 0.1 s, dt 0.4 ms, 5001
  samples; one vertical force at (2.0, 0.01) km; 400 two-component receivers
  at z = 10 m every 10 m; free surface on top, absorbing elsewhere with
  60-cell tapers.  Starting model for the gradient: the true model smoothed
  with sigma 250 m.
* vti_batch       -- the same grid, VTI with eps in [0.05, 0.20] and delta in
  [0, 0.10] as smooth seeded fields; 64 shots 60 m apart, each with a 1.0-3.5
  km receiver aperture on its own cropped grid and a 1.2-2.0 s record.
* elastic_batch   -- the batch geometry of vti_batch on the isotropic model
  of elastic_single (batched elastic gradients).
* ae_fwi          -- acoustic-elastic FWI: a 200 m water layer (vp 1.5,
  vs 0, rho 1.0) over a flat seabed on four elastic layers with seeded
  velocities in [2.2, 4.0] km/s and a Gaussian low-velocity lens; 601 x 1601
  cells at 5 m in all (the water rows are the fluid layer above the elastic
  grid), Ricker 8 Hz, dt 0.4 ms, 6001 samples, 96 shots in the water; or the
  same model on a coarser, smaller grid (scale) for solver runs that the
  reference's CPU build finishes in minutes.
"""
import math

import numpy as np

from . import _capi as C


def ricker(nt, dt, f0, t0):
    t = np.arange(nt, dtype=np.float64) * dt - t0
    a = (math.pi * f0 * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(np.float32)


def _smooth(rng_field, sigma):
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(rng_field, sigma, mode="nearest")


def elastic_model(nx=801, nz=401, d=0.005, seed=0, sigma_cells=10):
    """Raw (vp, vs, rho) of the true model: the perturbation is smoothed with a
    Gaussian of sigma_cells cells (50 m on the 5 m grid)."""
    rng = np.random.default_rng(seed)
    z = np.arange(nz) * d
    p = _smooth(rng.uniform(-1, 1, (nx, nz)), sigma_cells)
    p *= 0.05 / np.abs(p).max()
    vp = (2.0 + 0.75 * z)[None, :] * (1 + p)
    vs = vp / 1.73
    rho = 0.31 * (1000 * vp) ** 0.25
    return np.stack([vp, vs, rho]).astype(np.float32)


def smoothed(model, sigma_cells):
    return np.stack([_smooth(m.astype(np.float64), sigma_cells) for m in model]).astype(np.float32)


def vti_model(nx=801, nz=401, d=0.005, seed=2):
    """Raw (vp, vs, rho, delta, eps)."""
    base = elastic_model(nx, nz, d, seed=0)
    rng = np.random.default_rng(seed)

    def field(lo, hi):
        f = _smooth(rng.uniform(-1, 1, (nx, nz)), 20)
        f = (f - f.min()) / max(f.max() - f.min(), 1e-12)
        return lo + (hi - lo) * f

    eps = field(0.05, 0.20)
    dl = field(0.0, 0.10)
    return np.concatenate([base, dl[None], eps[None]]).astype(np.float32)


def convert(kind, raw):
    """nl_we_op_*::convert_model (we_op.cpp:476-494, 1441-1462, 1863-1881) in float32."""
    m = raw.astype(np.float32).copy()
    if kind == C.ACOUSTIC:
        m[0] = m[1] * m[0] * m[0]
        m[1] = np.float32(1.0) / m[1]
        return m
    vp, vs, rho = m[0].copy(), m[1].copy(), m[2].copy()
    lam = rho * (vp * vp - np.float32(2) * vs * vs)
    mu = rho * vs * vs
    m[0], m[1] = lam, mu
    if kind == C.VTI:
        dl = m[3]
        m[3] = (np.sqrt((np.float32(2) * (lam + np.float32(2) * mu) * (lam + mu) * dl + (lam + mu) * (lam + mu)).astype(np.float64))
                - mu).astype(np.float32)
    return m


def elastic_single(nt=5001):
    """Elastic single-shot gradient workload; returns a dict."""
    nx, nz, d, dt = 801, 401, 0.005, 4e-4
    true = elastic_model(nx, nz, d)
    start = smoothed(true, 50)
    w = ricker(nt, dt, 10.0, 0.1)
    ang = np.float32(1.5708)
    src = np.stack([w * np.float32(np.cos(ang)), w * np.float32(np.sin(ang))])[:, None, :].astype(np.float32)
    rx = (0.005 + 0.01 * np.arange(400)).astype(np.float32)
    rz = np.full(400, 0.01, np.float32)
    params = dict(nt=nt, sub=1, dt=dt, bc_top=1, bc_bottom=2, bc_left=2, bc_right=2, taper_top=0, taper_bottom=60,
                  taper_left=60, taper_right=60, taper_strength=0.05)
    return dict(kind=C.ELASTIC, nx=nx, nz=nz, d=d, dt=dt, nt=nt, true=true, start=start, src=src,
                shots=[dict(x0=0, nx=nx, sx=[2.0], sz=[0.01], rx=rx, rz=rz, nt=nt)], params=params, seismotype=1)


def elastic_large(nt=16001, checkpoint_every=200, snapshot_precision=C.SNAP_FP16, nshots=1):
    """Large-grid elastic gradient workload: 1201 x 4001 cells at 2.5 m, Ricker
    15 Hz, dt = 0.2 ms, nt = 16001, shots at x = 5 km (one shot) or spread
    over 1-9 km (nshots > 1), each with 798 two-component receivers every
    12.5 m at 10 m depth on the whole grid.  The perturbation of the true
    model is smoothed over 50 m (20 cells), the starting model over 125 m
    (50 cells).  Snapshots are 16-bit, rebuilt by checkpoint-and-recompute
    every 200 steps (the FP32 snapshots of one shot would take 615 GB)."""
    nx, nz, d, dt = 4001, 1201, 0.0025, 2e-4
    true = elastic_model(nx, nz, d, sigma_cells=20)
    start = smoothed(true, 50)
    w = ricker(nt, dt, 15.0, 0.1)
    ang = np.float32(1.5708)
    src = np.stack([w * np.float32(np.cos(ang)), w * np.float32(np.sin(ang))])[:, None, :].astype(np.float32)
    rx = (0.0125 * (1 + np.arange(798))).astype(np.float32)
    rz = np.full(798, 0.01, np.float32)
    params = dict(nt=nt, sub=1, dt=dt, bc_top=1, bc_bottom=2, bc_left=2, bc_right=2, taper_top=0, taper_bottom=60,
                  taper_left=60, taper_right=60, taper_strength=0.05, checkpoint_every=checkpoint_every,
                  snapshot_precision=snapshot_precision)
    sxs = [5.0] if nshots == 1 else [1.0 + 8.0 * k / (nshots - 1) for k in range(nshots)]
    return dict(kind=C.ELASTIC, nx=nx, nz=nz, d=d, dt=dt, nt=nt, true=true, start=start, src=src,
                shots=[dict(x0=0, nx=nx, sx=[sx], sz=[0.01], rx=rx, rz=rz, nt=nt) for sx in sxs], params=params,
                seismotype=1)


def batch_geometry(nshots=64, nt_max=5001, seed=2, nx=801, d=0.005, dt=4e-4):
    """Shots 60 m apart, each with a receiver aperture drawn from [1.0, 3.5] km
    on its own cropped grid (aperture and source with a 60-cell margin) and a
    record length drawn from [1.2, 2.0] s."""
    rng = np.random.default_rng(seed)
    shots = []
    margin = 60
    for k in range(nshots):
        sx = 0.03 + 0.06 * k
        aperture = rng.uniform(1.0, 3.5)
        rec = rng.uniform(1.2, 2.0)
        nts = min(nt_max, int(round(rec / dt)) + 1)
        # the aperture slides inside the 4 km line near its ends rather than being clipped
        lo = min(max(0.0, sx - aperture / 2), (nx - 1) * d - aperture)
        hi = lo + aperture
        rx = np.arange(lo + 0.005, hi, 0.01, dtype=np.float32)
        x0 = max(0, int(math.floor(min(lo, sx) / d)) - margin)
        x1 = min(nx, int(math.ceil(max(hi, sx) / d)) + margin + 1)
        shots.append(dict(x0=x0, nx=x1 - x0, sx=[sx], sz=[0.01], rx=rx, rz=np.full(len(rx), 0.01, np.float32), nt=nts))
    return shots


def vti_batch(nshots=64, nt_max=5001, seed=2):
    """Batched VTI workload: 64 shots on cropped grids with uneven apertures
    and record lengths."""
    nx, nz, d, dt = 801, 401, 0.005, 4e-4
    true = vti_model(nx, nz, d, seed=seed)
    start = np.concatenate([smoothed(true[:3], 50), true[3:]])
    w = ricker(nt_max, dt, 10.0, 0.1)
    shots = batch_geometry(nshots, nt_max, seed, nx, d, dt)
    ang = np.float32(1.5708)
    src = np.stack([w * np.float32(np.cos(ang)), w * np.float32(np.sin(ang))])[:, None, :].astype(np.float32)
    params = dict(nt=nt_max, sub=1, dt=dt, bc_top=1, bc_bottom=2, bc_left=2, bc_right=2, taper_top=0,
                  taper_bottom=60, taper_left=60, taper_right=60, taper_strength=0.05)
    return dict(kind=C.VTI, nx=nx, nz=nz, d=d, dt=dt, nt=nt_max, true=true, start=start, src=src, shots=shots,
                params=params, seismotype=1)


def elastic_batch(nshots=64, nt_max=5001, seed=2, every=1, snapshot_precision=C.SNAP_FP16):
    """Batched elastic workload: the vti_batch geometry (every `every`-th of its
    shots) on the elastic_single model, with reduced-precision snapshots."""
    wl = elastic_single(nt=nt_max)
    shots = batch_geometry(nshots, nt_max, seed, wl["nx"], wl["d"], wl["dt"])[::every]
    wl["shots"] = shots
    wl["params"] = dict(wl["params"], snapshot_precision=snapshot_precision)
    return wl


def ae_model(nx=1601, nz=561, d=0.005, seed=4):
    """Raw (vp, vs, rho) of the elastic part of the acoustic-elastic model (the
    grid below the seabed): four flat layers whose velocities are drawn from
    [2.2, 4.0] km/s and sorted to increase with depth, at seeded depths, and a
    Gaussian lens 15 % slower than its layer (width a tenth of the line, height
    a quarter of the grid) in the second layer; vs = vp/1.73,
    rho = 0.31 (1000 vp)^0.25."""
    rng = np.random.default_rng(seed)
    vel = np.sort(rng.uniform(2.2, 4.0, 4))
    cuts = np.sort(rng.uniform(0.15, 0.85, 3)) * nz
    z = np.arange(nz)[None, :] * np.ones((nx, 1))
    layer = (z >= cuts[0]).astype(int) + (z >= cuts[1]) + (z >= cuts[2])
    vp = vel[layer]
    x = np.arange(nx)[:, None] * np.ones((1, nz))
    xc, zc = rng.uniform(0.35, 0.65) * nx, 0.5 * (cuts[0] + cuts[1])
    sx, sz = 0.1 * nx / 2.355, 0.25 * nz / 2.355
    vp = vp * (1 - 0.15 * np.exp(-0.5 * (((x - xc) / sx) ** 2 + ((z - zc) / sz) ** 2)))
    vs = vp / 1.73
    rho = 0.31 * (1000 * vp) ** 0.25
    return np.stack([vp, vs, rho]).astype(np.float32)


def ae_fwi(nx=1601, nz=561, nza=41, d=0.005, dt=4e-4, nt=6001, nshots=96, seed=4):
    """Acoustic-elastic FWI workload: a fluid layer of nza rows (200 m at the
    defaults) over an elastic grid of nz x nx cells (ae_model), dt, nt
    samples of a Ricker 8 Hz source delayed 0.15 s, nshots sources 10 m below
    the sea surface spread over the line, receivers every 10 m from 10 m,
    10 m below the seabed on the elastic grid and 10 m below the sea surface
    in the fluid.  Free sea surface, absorbing elsewhere with 20-cell tapers.
    The starting model is the true model smoothed over 150 m."""
    oz = (nza - 1) * d
    true = ae_model(nx, nz, d, seed)
    start = smoothed(true, max(1.0, 0.15 / d))
    w = ricker(nt, dt, 8.0, 0.15)
    width = (nx - 1) * d
    sxs = [width * (0.05 + 0.9 * k / max(1, nshots - 1)) for k in range(nshots)]
    rx = np.arange(0.01, width - 0.005, 0.01, dtype=np.float32)
    params = dict(nt=nt, sub=1, dt=dt, bc_top=1, bc_bottom=2, bc_left=2, bc_right=2, taper_top=0,
                  taper_bottom=20, taper_left=20, taper_right=20, taper_strength=0.05, nza=nza, acoustic_source=1)
    return dict(kind=C.ACOUSTIC_ELASTIC, nx=nx, nz=nz, nza=nza, oz=oz, d=d, dt=dt, nt=nt, true=true, start=start,
                src=w[None, :], sx=np.array(sxs, np.float32), sz=np.full(nshots, 0.01, np.float32), rx=rx,
                rz=np.full(len(rx), oz + 0.01, np.float32), rzw=np.full(len(rx), 0.01, np.float32), params=params,
                seismotype=1)


def ae_fwi_small(nshots=6, nt=1201):
    """The acoustic-elastic FWI model on a grid the reference's CPU build
    inverts in minutes: 10 m cells, a 2 km line (201 cells), the 200 m water
    layer (21 fluid rows) over 600 m of elastic grid (61 rows), dt 1 ms."""
    return ae_fwi(nx=201, nz=61, nza=21, d=0.01, dt=1e-3, nt=nt, nshots=nshots)
