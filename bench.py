#!/usr/bin/env python
"""Benchmark: elastic FWI gradient on B200 (fwi2d_b200) vs the reference CPU path.

One step = one full FWI gradient evaluation of the elastic single-shot
workload (401 x 801 grid at 5 m, nt = 5001, 400 two-component receivers,
FP32 snapshots of every time step kept in HBM): forward propagation with
snapshot storage, residual against observed data, adjoint sources, adjoint
propagation with the zero-lag imaging condition, H quadrature and chain rule.
Cell-updates per step: (nt-1) * nx * nz forward + the same adjoint.

At N = 1 the line also carries:
* "batched": the batched VTI configuration as written -- 64 shots 60 m apart
  on cropped grids (1.0-3.5 km apertures, 1.2-2.0 s records), VTI model,
  FP32 snapshots -- in one plan on one GPU.  Its snapshots (about 430 GB) do
  not fit the device, so the plan runs its shots in HBM-sized waves, each
  wave a CUDA graph, the gradient summed over all shots;
* "large": 4 shots of the large-grid configuration (1201 x 4001 at 2.5 m,
  nt = 16001), FP16 snapshots rebuilt by checkpoint-and-recompute every 200
  steps, with the 32-shot time projected from it;
* "fp64_error" on each of them: trace and gradient error against the
  reference's FP64 build (oracle/_ref) on a bounded sample of the same
  geometry (FP32, and for the large grid also BF16 and FP16 snapshots);
* "reference_gpu": the reference's own GPU implementation (src/cuda, built
  for sm_100a into oracle/_ref by oracle/build_ref.sh) timed on a bounded
  sample of the same shot, with "e2e_speedup" = this library's end-to-end
  value over it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config single|batch|large]

--config large: one shot of the large-grid workload (1201 x 4001 at 2.5 m,
nt = 16001), FP16 snapshots rebuilt by checkpoint-and-recompute every 200
steps; its adjoint loop time includes the replay of the forward segments.

N > 1 runs one process per GPU (torchrun); each rank computes its own shot
(weak scaling) and the model gradient is summed over ranks with NCCL.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "elastic FWI gradient shots/s + Gcell-updates/s, batched vs plain, 1 B200"
BYTES_FWD = 36 + 8      # algorithmic bytes per forward cell-update (fields, model, fp32 snapshot store)
BYTES_ADJ = 68          # adjoint + imaging: fields, model, snapshot read, gradient read-modify-write
VTI_EXTRA = 8           # VTI reads c13 and eps as well


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="single", choices=["single", "batch", "large"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-ae", action="store_true")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# Per framed plan of the single-shot grid: DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum) of the core, x-band and z-band launches of one
# adjoint step, and the core launch's L1-to-L2 bytes, cold duration and L2
# throughput, from the captures summarised in
# profiles/elastic_step_framed_single_shot_401x801.md and, for the split band
# kernels that one shot takes, profiles/elastic_band_split_single_shot_401x801.md
# (cold caches: ncu flushes L2 before each pass).
FRAMED_CAPTURES = {
    16: dict(core="elastic_step<RZ=2, CORE> (64 x 8 z-pair windows)",
             traffic={"core": 21.133312e6, "x_bands": 0.554496e6, "z_bands": 3.61984e6},
             l2_bytes=1447280 * 32, core_cold_us=28.576, lts_pct=7.0),
    14: dict(core="elastic_step<RZ=1, CORE> (32 x 8 windows)",
             traffic={"core": 21.152256e6, "x_bands": 0.499712e6, "z_bands": 3.606528e6},
             l2_bytes=1651721 * 32, core_cold_us=21.312, lts_pct=10.4),
    15: dict(core="elastic_step<RZ=1, CORE> (32 x 16 windows)",
             traffic={"core": 21.128704e6, "x_bands": 0.498688e6, "z_bands": 3.606784e6},
             l2_bytes=1548000 * 32, core_cold_us=25.95, lts_pct=8.1),
}


def roof_kernel(shape, config):
    if config == "single" and shape in FRAMED_CAPTURES:
        return ("adjoint + imaging step of the framed plan: interior %s with the band kernels elastic_xband and "
                "elastic_zband<SPLIT> (a cell's two components in two warps) overlapped on two side streams "
                "(one step = one launch of each)" % FRAMED_CAPTURES[shape]["core"])
    if config == "single":
        return "adjoint + imaging step (tile shape %d)" % shape
    return "adjoint loop: interior, band and imaging kernels"


def step_traffic(shape, config):
    """DRAM bytes of one adjoint step from the committed ncu summaries, or
    None when the plan's launches are not captured."""
    cap = FRAMED_CAPTURES.get(shape) if config == "single" else None
    if not cap or not cap["traffic"]:
        return None
    return sum(cap["traffic"].values())


def l2_note(shape, config):
    """L2 figures of the L2-resident single-shot case, from the committed ncu
    capture of the core launch (cold caches)."""
    cap = FRAMED_CAPTURES.get(shape) if config == "single" else None
    if not cap or not cap["l2_bytes"]:
        return None
    return {"kernel": cap["core"] + " adjoint", "l1_to_l2_bytes_per_launch": cap["l2_bytes"],
            "achieved_gbs": cap["l2_bytes"] / (cap["core_cold_us"] * 1e-6) / 1e9, "lts_throughput_pct": cap["lts_pct"],
            "source": "ncu capture, cold caches (profiles/elastic_step_framed_single_shot_401x801.md, "
                      "profiles/elastic_band_split_single_shot_401x801.md)"}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx = float(c[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for n, v in zip(names, c[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def build_workload(name, rank, world):
    from fwi2d_b200 import workloads as W
    if name == "single":
        wl = W.elastic_single()
        if world > 1:   # one shot per rank, sources 60 m apart
            sh = dict(wl["shots"][0])
            sh["sx"] = [2.0 + 0.06 * rank]
            wl["shots"] = [sh]
    elif name == "large":
        wl = W.elastic_large()
        if world > 1:   # one shot per rank, sources 100 m apart
            sh = dict(wl["shots"][0])
            sh["sx"] = [5.0 + 0.1 * rank]
            wl["shots"] = [sh]
    else:
        wl = W.vti_batch()
        if world > 1:   # cost-balanced shot lists (longest processing time first)
            from fwi2d_b200.distributed import shard_shots
            wl["shots"] = [wl["shots"][i] for i in shard_shots(wl["shots"], rank, world, wl["nz"])]
    return wl


def make_prop(wl, device):
    import fwi2d_b200 as F
    from fwi2d_b200 import workloads as W
    P = F.Propagator(device)
    kind = wl["kind"]
    start = W.convert(kind, wl["start"])
    P.set_model(kind, start, wl["d"], wl["d"])
    shots = [F.ShotSpec(s["x0"], s["nx"], s["nt"], s["sx"], s["sz"], s["rx"], s["rz"]) for s in wl["shots"]]
    P.set_shots(F.make_params(**wl["params"]), shots)
    srcs = [np.ascontiguousarray(wl["src"][:, :, :s["nt"]]) for s in wl["shots"]]
    return P, start, srcs


def observed(wl, device, srcs):
    """Observed data: the forward of the true model through the same library
    (seismotype 1: particle velocity)."""
    import fwi2d_b200 as F
    from fwi2d_b200 import workloads as W
    P = F.Propagator(device)
    kind = wl["kind"]
    P.set_model(kind, W.convert(kind, wl["true"]), wl["d"], wl["d"])
    shots = [F.ShotSpec(s["x0"], s["nx"], s["nt"], s["sx"], s["sz"], s["rx"], s["rz"]) for s in wl["shots"]]
    prm = dict(wl["params"])
    prm["sub"] = 0
    prm["checkpoint_every"] = 0
    P.set_shots(F.make_params(**prm), shots)
    out = P.forward(srcs, store=False)
    P.close()
    obs = []
    dt = wl["dt"]
    for u in out:
        v = np.empty_like(u)
        v[..., 0] = (u[..., 1] - u[..., 0]) / np.float32(dt)
        v[..., -1] = (u[..., -1] - u[..., -2]) / np.float32(dt)
        v[..., 1:-1] = (u[..., 2:] - u[..., :-2]) / np.float32(2 * dt)
        obs.append(v.astype(np.float32))
    return obs


def cells_per_step(wl):
    nz = wl["nz"]
    return sum(2 * (s["nt"] - 1) * s["nx"] * nz for s in wl["shots"])


def fp64_error(kind, mc, nz, d, shot, params, src, nt, device, precs=(0,), checkpoint_every=0, tile_shape=3):
    """Error of this library against the reference's FP64 build (oracle/_ref,
    the reference's sources with DOUBLE_PRECISION) on a bounded sample of one
    shot: its cropped grid, nt time samples.  Forward traces, then the adjoint
    imaging condition with the FP64 traces reversed in time as adjoint
    sources, for each snapshot precision in precs.  Returns a dict of relative
    L2 errors."""
    import oracle as O
    import fwi2d_b200 as F
    if not O.have_reference(64):
        return {"unavailable": "the reference FP64 build (oracle/_ref) is absent"}
    ref = O.Reference(64)
    x0, nx = shot["x0"], shot["nx"]
    mcs = np.ascontiguousarray(mc[:, x0:x0 + nx])
    ox = np.float32(x0 * d)
    sx, sz = np.array(shot["sx"], np.float32) - ox, np.array(shot["sz"], np.float32)
    rx, rz = np.asarray(shot["rx"], np.float32) - ox, np.asarray(shot["rz"], np.float32)
    nr = len(rx)
    src_s = np.ascontiguousarray(src[:, :, :nt])
    keys = ("sub", "dt", "bc_top", "bc_bottom", "bc_left", "bc_right", "taper_top", "taper_bottom", "taper_left",
            "taper_right", "taper_strength")
    par = O.make_par(**{k: params[k] for k in keys}, nt=nt, ns=1, nr=nr)
    m64 = mcs.astype(np.float64)
    rcv64 = np.zeros((2, nr, nt), np.float64)
    full64 = np.zeros((nt + 1, 2, nx, nz), np.float64)
    ref.propagate(kind, 0, m64, src_s.astype(np.float64), rcv64, par, nx, nz, d, d, 0.0, 0.0, (sx, sz), (rx, rz),
                  full=full64)
    adj = np.ascontiguousarray(rcv64[:, :, ::-1] / max(np.abs(rcv64).max(), 1e-30)).astype(np.float32)
    g64 = np.zeros((5 if kind == 1 else 3, nx, nz), np.float64)
    ref.propagate(kind, 1, m64, adj.astype(np.float64), np.zeros((2, 1, nt)), par, nx, nz, d, d, 0.0, 0.0,
                  (rx, rz), (sx, sz), full=full64, grad=g64)
    del full64

    def rel(a, b):
        b = np.asarray(b, np.float64)
        return float(np.linalg.norm((np.asarray(a, np.float64) - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))

    out = {"sample": "shot grid %d x %d, %d time samples; adjoint sources: the FP64 traces reversed in time"
                     % (nz, nx, nt)}
    names = {0: "fp32", 1: "bf16", 2: "fp16"}
    for prec in precs:
        P = F.Propagator(device)
        P.set_model(kind, mcs, d, d)
        prm = {k: params[k] for k in keys}
        prm.update(nt=nt, snapshot_precision=prec, checkpoint_every=checkpoint_every if nt > checkpoint_every else 0,
                   tile_shape=tile_shape)
        P.set_shots(F.make_params(**prm), [F.ShotSpec(0, nx, nt, sx, sz, rx, rz)])
        rcv = P.forward([src_s], store=True)[0]
        g = P.adjoint([adj])
        P.close()
        e = {"gradient": [rel(g[c], g64[c]) for c in range(3)]}
        if prec == precs[0]:
            out["traces"] = rel(rcv, rcv64)
        out[names[prec]] = e
    return out


# ---------------------------------------------------------------------------
# CPU reference timing (reference sources built in oracle/_ref, else the port)
# ---------------------------------------------------------------------------
def cpu_sample(wl, nt_sample, lib=None):
    """Forward with snapshots + adjoint with imaging on the full grid of the
    first shot, nt_sample time samples.  Returns (seconds, cell-updates, kind).
    lib: the reference build (default: oracle/_ref, else the port)."""
    import oracle as O
    from fwi2d_b200 import workloads as W
    if lib is None:
        kind = "reference" if O.have_reference(32) else "port"
        lib = O.Reference(32) if kind == "reference" else O.Port(32)
    else:
        kind = lib.kind
    s = wl["shots"][0]
    nx, nz, d = s["nx"], wl["nz"], wl["d"]
    k = wl["kind"]
    model = W.convert(k, wl["start"])[:, s["x0"]:s["x0"] + nx].copy()
    p = dict(wl["params"])
    p.update(nt=nt_sample, ns=1, nr=len(s["rx"]))
    par = O.make_par(**{kk: v for kk, v in p.items() if kk in dict(O.Par._fields_)})
    src = np.ascontiguousarray(wl["src"][:, :, :nt_sample])
    ox = s["x0"] * d
    sl = (np.array(s["sx"], np.float32) - ox, np.array(s["sz"], np.float32))
    rl = (np.asarray(s["rx"], np.float32) - ox, np.asarray(s["rz"], np.float32))
    rcv = np.zeros((2, len(s["rx"]), nt_sample), np.float32)
    full = np.zeros((1 + nt_sample, 2, nx, nz), np.float32)
    full[...] = 0.0   # first touch outside the timed region
    g = np.zeros((5 if k == 1 else 3, nx, nz), np.float32)
    t0 = time.perf_counter()
    lib.propagate(k, 0, model, src, rcv, par, nx, nz, d, d, 0.0, 0.0, sl, rl, full=full)
    adj = np.ascontiguousarray(-rcv[:, :, ::-1])
    srcb = np.zeros((2, 1, nt_sample), np.float32)
    lib.propagate(k, 1, model, adj, srcb, par, nx, nz, d, d, 0.0, 0.0, rl, sl, full=full, grad=g)
    dtime = time.perf_counter() - t0
    return dtime, 2 * (nt_sample - 1) * nx * nz, kind


def reference_gpu_sample(wl, nt_sample=1001, reps=2):
    """The reference's own GPU path (src/cuda, propagate_gpu, built into
    oracle/_ref/libfwi2d_ref32_cuda.so) on the same shot: forward with
    snapshots copied to host memory, then the adjoint with imaging, nt_sample
    time samples, wall clock (the path is synchronous with the host).  Best of
    reps after one warm-up.  None when that build is absent."""
    import oracle as O
    if not O.have_reference_gpu():
        return None
    lib = O.ReferenceGPU()
    cpu_sample(wl, 21, lib)
    best, cells = None, 0
    for _ in range(reps):
        t, cells, _ = cpu_sample(wl, nt_sample, lib)
        best = t if best is None else min(best, t)
    g = cells / best / 1e9
    return {"value": g, "unit": "Gcell-updates/s", "kind": "reference GPU path (src/cuda, propagate_gpu, sm_100a)",
            "sample": "forward+adjoint gradient of shot 0, %d of %d time samples, host snapshots as the reference"
                      % (nt_sample, wl["nt"]),
            "shots_per_s": g * 1e9 / cells_per_step(wl) * len(wl["shots"])}


def cpu_cores():
    n = os.environ.get("OMP_NUM_THREADS")
    return int(n) if n else (os.cpu_count() or 1)


# ---------------------------------------------------------------------------
def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    os.environ.setdefault("OMP_PROC_BIND", "close")
    wl = build_workload(args.config, 0, 1)
    nt_sample = 301
    for _ in range(args.warmup):
        cpu_sample(wl, nt_sample)
    times, kind, cells = [], None, 0
    for _ in range(args.steps):
        dtime, cells, kind = cpu_sample(wl, nt_sample)
        times.append(dtime)
    tot = sum(times)
    gcell = cells * args.steps / tot / 1e9
    shots = gcell * 1e9 / cells_per_step(wl) * len(wl["shots"])
    sample = "forward+adjoint gradient of shot 0 on its full grid, %d of %d time samples" % (nt_sample, wl["nt"])
    line = {"metric": METRIC, "value": gcell, "unit": "Gcell-updates/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "shots_per_s": shots,
            "config": {"workload": workload_name(args.config), "sample_nt": nt_sample},
            "cpu_baseline": {"value": gcell, "unit": "Gcell-updates/s", "cores": cpu_cores(), "kind": kind,
                             "sample": sample},
            "e2e": {"value": gcell, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.config == "single":
        try:   # the reference's GPU path beside its CPU path, for context (not this line's value)
            rg = reference_gpu_sample(wl)
            if rg is not None:
                line["reference_gpu"] = rg
        except Exception as e:
            line["reference_gpu"] = {"value": None, "sample": "failed: %s" % e}
    print(json.dumps(line), flush=True)


def workload_name(cfg):
    if cfg == "single":
        return "elastic isotropic FWI gradient, 1 shot, 401x801 grid at 5 m, nt=5001, 400 2-C receivers, FP32 snapshots"
    if cfg == "large":
        return ("elastic isotropic FWI gradient, 1 shot, 1201x4001 grid at 2.5 m, nt=16001, 798 2-C receivers, "
                "FP16 snapshots rebuilt by checkpoint-and-recompute every 200 steps")
    return "VTI FWI gradient, 64 shots on cropped grids (1.0-3.5 km apertures, 1.2-2.0 s records), 401x801 at 5 m"


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    import fwi2d_b200 as F
    F.load()
    wl = build_workload(args.config, rank, world)
    P, start, srcs = make_prop(wl, local)
    obs = observed(wl, local, srcs)
    stream = torch.cuda.Stream()
    P.set_stream(stream.cuda_stream)
    P.set_observed(obs)
    P.upload(srcs, adjoint=False)
    L = F.load()
    from fwi2d_b200 import _capi as C
    ng = 3
    gdev = torch.zeros((ng, wl["nx"], wl["nz"]), dtype=torch.float32, device="cuda")

    def grad_step():
        C.check(L.fwi2d_fwi_gradient(P.h, None, None, None, wl["seismotype"], None, None))
        if world > 1:
            P.copy_gradient(gdev.data_ptr())
            with torch.cuda.stream(stream):
                torch.distributed.all_reduce(gdev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # warm-up (graph capture happens on the first call)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            grad_step()
    torch.cuda.synchronize()
    barrier()
    clk = Clocks(local)
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.nvtx.range_push("timed")
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for _ in range(args.steps):
            grad_step()
        ev1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier()
    ms = ev0.elapsed_time(ev1)
    fwd_ms, adj_ms = P.last_timing()
    clocks = clk.stop()

    # end to end through the public call with host buffers (pinned)
    kind = wl["kind"]
    model_h = torch.from_numpy(start).pin_memory().numpy()
    src_h = torch.from_numpy(np.concatenate([s.ravel() for s in srcs])).pin_memory().numpy()
    obs_h = torch.from_numpy(np.concatenate([o.ravel() for o in obs])).pin_memory().numpy()
    grad_pin = torch.empty((ng, wl["nx"], wl["nz"]), dtype=torch.float32).pin_memory()
    import ctypes
    mis = ctypes.c_double(0.0)

    def e2e_step():
        # host inputs in, gradient (summed over ranks) and misfit out to host
        C.check(L.fwi2d_fwi_gradient(P.h, C.ptr(model_h), C.ptr(src_h), C.ptr(obs_h), wl["seismotype"], None,
                                     ctypes.byref(mis)))
        P.copy_gradient(gdev.data_ptr())
        if world > 1:
            torch.distributed.all_reduce(gdev)
        grad_pin.copy_(gdev, non_blocking=True)

    with torch.cuda.stream(stream):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    n_e2e = max(1, args.steps // 2)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(n_e2e):
            e2e_step()
        e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1) / n_e2e

    # max over ranks
    t = torch.tensor([ms, e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms, e2e_ms = float(t[0]), float(t[1])
    info = P.plan_info()
    cells_rank = cells_per_step(wl)
    nshots_rank = len(wl["shots"])
    total_cells = cells_rank * world
    total_shots = nshots_rank * world
    ms_step = ms / args.steps
    value = total_cells / (ms_step / 1e3) / 1e9
    shots_s = total_shots / (ms_step / 1e3)

    # dominant kernel: the adjoint step (imaging condition fused)
    steps_adj = max(s["nt"] for s in wl["shots"]) - 1
    cells_launch = sum(s["nx"] * wl["nz"] for s in wl["shots"])
    adj_launch_s = adj_ms / 1e3 / steps_adj
    fwd_launch_s = fwd_ms / 1e3 / steps_adj
    bytes_adj = BYTES_ADJ - (4 if wl["params"].get("snapshot_precision", 0) else 0)   # 16-bit snapshot read
    achieved = bytes_adj * cells_launch / adj_launch_s / 1e9
    peak, peak_kind = peaks()
    launches = (info["launches_forward"] + info["launches_adjoint"] + 2 * nshots_rank + 1) * args.steps
    if rank == 0:
        h2d = model_h.nbytes + src_h.nbytes + obs_h.nbytes
        d2h = grad_pin.numel() * 4 + 8
        line = {
            "metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "shots_per_s": shots_s,
            "config": {"workload": workload_name(args.config), "nx": wl["nx"], "nz": wl["nz"], "nt": wl["nt"],
                       "shots_per_gpu": nshots_rank,
                       "snapshots": ("fp16, checkpoint-and-recompute every 200 steps (the adjoint loop includes the "
                                     "replay)" if args.config == "large" else "fp32 every step, in HBM"),
                       "cell_updates_per_step": total_cells, "tile_shape": info["tile_shape"],
                       "l2": "inputs larger than L2: %.1f GB of snapshots written and read per step"
                             % (info["snapshot_bytes"] / 1e9),
                       "parallelism": "shots over %d GPU(s), NCCL all-reduce of the gradient" % world},
            "e2e": {"value": total_cells / (e2e_ms / 1e3) / 1e9, "unit": "Gcell-updates/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "shots_per_s": total_shots / (e2e_ms / 1e3)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": roof_kernel(info["tile_shape"], args.config),
                         "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": step_traffic(info["tile_shape"], args.config),
                         "algorithmic_bytes_per_launch": bytes_adj * cells_launch,
                         "launch_ms": adj_launch_s * 1e3,
                         "forward_launch_ms": fwd_launch_s * 1e3,
                         "forward_achieved": BYTES_FWD * cells_launch / fwd_launch_s / 1e9},
            "l2": l2_note(info["tile_shape"], args.config),
            "clocks": clocks,
        }
        if world == 1 and args.config == "single":
            try:
                line["fp64_error"] = fp64_error(wl["kind"], start, wl["nz"], wl["d"], wl["shots"][0], wl["params"],
                                                wl["src"], 500, local, tile_shape=info["tile_shape"])
            except Exception as e:   # never blocks the main line
                line["fp64_error"] = {"unavailable": "failed: %s" % e}
        if world == 1 and args.config == "single" and not args.no_batched:
            try:
                b = run_batched(local, 2, 1)
                b["shots_per_s_vs_plain"] = b["shots_per_s"] / shots_s
                b["gcell_vs_plain"] = b["value"] / value
                line["batched"] = b
            except Exception as e:   # the batched leg never blocks the main line
                line["batched"] = {"error": str(e)}
        if world == 1 and args.config == "single" and not args.no_large:
            try:
                line["large"] = run_large(local)
            except Exception as e:   # the large-grid leg never blocks the main line
                line["large"] = {"error": str(e)}
        if world == 1 and args.config == "single" and not args.no_ae:
            try:
                line["acoustic_elastic"] = run_ae(local)
            except Exception as e:   # the acoustic-elastic leg never blocks the main line
                line["acoustic_elastic"] = {"error": str(e)}
        if world == 1 and args.config == "single":
            try:
                rg = reference_gpu_sample(wl)
                if rg is not None:
                    rg["e2e_speedup"] = line["e2e"]["value"] / rg["value"]
                    line["reference_gpu"] = rg
            except Exception as e:   # the comparison never blocks the GPU line
                line["reference_gpu"] = {"value": None, "sample": "failed: %s" % e}
        if world == 1 and not args.no_cpu_baseline:
            try:
                nt_s = 301
                dtime, cells, kind = cpu_sample(wl, nt_s)
                g = cells / dtime / 1e9
                line["cpu_baseline"] = {"value": g, "unit": "Gcell-updates/s", "cores": cpu_cores(), "kind": kind,
                                        "sample": "forward+adjoint gradient of shot 0, %d of %d time samples"
                                                  % (nt_s, wl["nt"]),
                                        "shots_per_s": g * 1e9 / cells_per_step(wl) * nshots_rank}
            except Exception as e:   # the baseline never blocks the GPU line
                line["cpu_baseline"] = {"value": None, "unit": "Gcell-updates/s", "cores": cpu_cores(),
                                        "kind": "port", "sample": "failed: %s" % e}
        print(json.dumps(line), flush=True)
    P.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def timed_gradients(wl, local, steps, warmup, tile_shape=None):
    """FWI gradients of a workload on one GPU, device-resident inputs; returns
    (ms per gradient, forward ms, adjoint ms, plan info, waves, snapshot bytes
    of all shots)."""
    import torch
    import fwi2d_b200 as F
    from fwi2d_b200 import _capi as C
    if tile_shape is not None:
        wl = dict(wl, params=dict(wl["params"], tile_shape=tile_shape))
    P, start, srcs = make_prop(wl, local)
    obs = observed(wl, local, srcs)
    stream = torch.cuda.Stream()
    P.set_stream(stream.cuda_stream)
    P.set_observed(obs)
    P.upload(srcs, adjoint=False)
    L = F.load()

    def step():
        C.check(L.fwi2d_fwi_gradient(P.h, None, None, None, wl["seismotype"], None, None))

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for _ in range(steps):
            step()
        ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    fwd_ms, adj_ms = P.last_timing()
    info = P.plan_info()
    nwaves, snap_all = P.plan_waves()
    P.close()
    return ms, fwd_ms, adj_ms, info, nwaves, snap_all


def run_batched(local, steps, warmup):
    """The batched VTI configuration (64 shots, cropped grids, uneven records,
    FP32 snapshots) on one GPU; returns a dict."""
    from fwi2d_b200 import workloads as W
    wl = W.vti_batch()
    ms, fwd_ms, adj_ms, info, nwaves, snap_all = timed_gradients(wl, local, steps, warmup)
    cells = cells_per_step(wl)
    # average algorithmic HBM bandwidth of each time loop (VTI, FP32 snapshots)
    peak, peak_kind = peaks()
    half = cells / 2
    fwd_gbs = (BYTES_FWD + VTI_EXTRA) * half / (fwd_ms / 1e3) / 1e9
    adj_gbs = (BYTES_ADJ + VTI_EXTRA) * half / (adj_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": "elastic_march<VTI> + band kernels (adjoint + imaging)", "achieved": adj_gbs,
            "peak": peak, "unit": "GB/s", "frac": adj_gbs / peak, "peak_source": peak_kind,
            "bytes_per_cell_update": {"forward": BYTES_FWD + VTI_EXTRA, "adjoint": BYTES_ADJ + VTI_EXTRA},
            "forward_achieved": fwd_gbs, "forward_frac": fwd_gbs / peak}
    out = {"workload": "VTI FWI gradient, %d shots of the batch geometry on cropped grids (mean %d x %d cells, "
                       "mean nt %d), FP32 snapshots" % (len(wl["shots"]), np.mean([s["nx"] for s in wl["shots"]]),
                                                         wl["nz"], np.mean([s["nt"] for s in wl["shots"]])),
           "shots": len(wl["shots"]), "ms_per_step": ms, "shots_per_s": len(wl["shots"]) / (ms / 1e3),
           "value": cells / (ms / 1e3) / 1e9, "unit": "Gcell-updates/s", "cell_updates_per_step": cells,
           "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "tile_shape": info["tile_shape"], "roofline": roof,
           "waves": nwaves, "snapshot_bytes_all_shots": snap_all, "snapshot_bytes_held": info["snapshot_bytes"],
           "steps": steps, "warmup": warmup}
    try:
        from fwi2d_b200 import workloads as W2
        sh = wl["shots"][0]
        out["fp64_error"] = fp64_error(wl["kind"], W2.convert(wl["kind"], wl["start"]), wl["nz"], wl["d"], sh,
                                       wl["params"], wl["src"], 500, local)
    except Exception as e:
        out["fp64_error"] = {"unavailable": "failed: %s" % e}
    return out


# plan of the large-grid workload, pinned so that the bench does not run the
# tuner's whole-pass stage, whose passes take tens of seconds on this grid:
# the framed plan with 32 x 8 interior windows (on 2 shots it measured 18.9
# Gcell/s against 17.7 for the best marching shape, 224 x 32)
LARGE_TILE_SHAPE = 14


def run_ae(local, nshots=8):
    """FWI gradients of the acoustic-elastic configuration at full size (601 x
    1601 cells at 5 m: 41 fluid rows over 561 elastic rows, nt = 6001, FP32
    snapshots), nshots of its 96 shots in one plan on one GPU (in waves: one
    shot's snapshots take 44 GB); returns a dict with the time of one gradient
    of 96 shots and of 20 L-BFGS iterations projected from it (lower bound)."""
    import ctypes
    import torch
    import fwi2d_b200 as F
    from fwi2d_b200 import _capi as C
    from fwi2d_b200 import workloads as W
    wl = W.ae_fwi(nshots=96)
    pick = np.linspace(0, 95, nshots).round().astype(int)
    nt, d, oz = wl["nt"], wl["d"], wl["oz"]
    prm = dict(wl["params"])

    def shots():
        return [F.ShotSpec(0, wl["nx"], nt, [0.0], [oz], wl["rx"], wl["rz"], water_src_x=[float(wl["sx"][k])],
                           water_src_z=[float(wl["sz"][k])], water_rcv_x=wl["rx"], water_rcv_z=wl["rzw"])
                for k in pick]
    src = np.ascontiguousarray(wl["src"].reshape(1, 1, nt))
    srcs = [src] * nshots
    # observed data: the true model's forward, as particle velocity / -d(potential)/dt (seismotype 1)
    Q = F.Propagator(local)
    Q.set_model(C.ACOUSTIC_ELASTIC, W.convert(C.ELASTIC, wl["true"]), d, d, 0.0, oz)
    Q.set_shots(F.make_params(**dict(prm, sub=0)), shots())
    raw = Q.forward(srcs, store=False)
    Q.close()
    obs = []
    for u in raw:
        v = np.empty_like(u)
        v[..., 0] = (u[..., 1] - u[..., 0]) / np.float32(wl["dt"])
        v[..., -1] = (u[..., -1] - u[..., -2]) / np.float32(wl["dt"])
        v[..., 1:-1] = (u[..., 2:] - u[..., :-2]) / np.float32(2 * wl["dt"])
        v[0] = -v[0]
        obs.append(v.astype(np.float32))
    P = F.Propagator(local)
    P.set_model(C.ACOUSTIC_ELASTIC, W.convert(C.ELASTIC, wl["start"]), d, d, 0.0, oz)
    P.set_shots(F.make_params(**prm), shots())
    stream = torch.cuda.Stream()
    P.set_stream(stream.cuda_stream)
    P.set_observed(obs)
    P.upload(srcs, adjoint=False)
    L = F.load()
    mis = ctypes.c_double(0.0)

    def step():
        C.check(L.fwi2d_fwi_gradient(P.h, None, None, None, 1, None, ctypes.byref(mis)))
    with torch.cuda.stream(stream):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        step()
        ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    fwd_ms, adj_ms = P.last_timing()
    info = P.plan_info()
    nwaves, snap_all = P.plan_waves()
    P.close()
    cells = nshots * 2 * (nt - 1) * wl["nx"] * (wl["nz"] + wl["nza"])
    per96 = ms * 96 / nshots / 1e3
    return {"workload": "acoustic-elastic FWI gradient, %d of the 96 shots of the 601 x 1601 model at 5 m (41 fluid "
                        "rows over 561 elastic rows), nt = %d, FP32 snapshots" % (nshots, nt),
            "shots": nshots, "ms_per_step": ms, "shots_per_s": nshots / (ms / 1e3),
            "value": cells / (ms / 1e3) / 1e9, "unit": "Gcell-updates/s (fluid and elastic cells)",
            "cell_updates_per_step": cells, "forward_ms": fwd_ms, "adjoint_ms": adj_ms,
            "tile_shape": info["tile_shape"], "waves": nwaves, "snapshot_bytes_all_shots": snap_all,
            "misfit": mis.value, "projected_96_shot_gradient_s": per96,
            "projected_20_lbfgs_iterations_s": per96 * 21,
            "projection": "20 L-BFGS iterations at one gradient evaluation each plus the initial one (a lower "
                          "bound: every further line-search trial adds one evaluation)"}


def run_large(local, nshots=4):
    """4 shots of the large-grid configuration (FP16 snapshots rebuilt by
    checkpoint-and-recompute every 200 steps) on one GPU; returns a dict."""
    from fwi2d_b200 import workloads as W
    wl = W.elastic_large(nshots=nshots)
    ms, fwd_ms, adj_ms, info, nwaves, _ = timed_gradients(wl, local, 1, 1, tile_shape=LARGE_TILE_SHAPE)
    cells = cells_per_step(wl)
    out = {"workload": "elastic FWI gradient, %d shots of the 1201 x 4001 grid at 2.5 m, nt = 16001, FP16 "
                       "snapshots rebuilt by checkpoint-and-recompute every 200 steps" % nshots,
           "shots": nshots, "ms_per_step": ms, "shots_per_s": nshots / (ms / 1e3),
           "value": cells / (ms / 1e3) / 1e9, "unit": "Gcell-updates/s", "cell_updates_per_step": cells,
           "recompute": "the adjoint loop replays each 200-step segment; replayed steps are not counted",
           "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "tile_shape": info["tile_shape"],
           "projected_32_shots_s": 32 * ms / nshots / 1e3, "steps": 1, "warmup": 1}
    try:
        # a crop of the large grid: 201 x 601 cells at 2.5 m, Ricker 15 Hz, dt 0.2 ms, 1201 samples
        crop = dict(wl["shots"][0], x0=0, nx=601, sx=[0.75], rx=(0.0125 * (1 + np.arange(46))).astype(np.float32),
                    rz=np.full(46, 0.01, np.float32))
        mc = W.convert(wl["kind"], wl["start"])[:, :601, :201]
        out["fp64_error"] = fp64_error(wl["kind"], mc, 201, wl["d"], crop, wl["params"], wl["src"], 1201, local,
                                       precs=(0, 1, 2), checkpoint_every=200)
    except Exception as e:
        out["fp64_error"] = {"unavailable": "failed: %s" % e}
    return out


def main():
    args = parse()
    # autotuner choices persist across the runs of one machine (a run under a
    # profiler then reuses the shape measured without it)
    os.environ.setdefault("FWI2D_TUNE_FILE", os.path.join(tempfile.gettempdir(), "fwi2d_b200_tune.txt"))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
