"""Run one small propagation case for kernel profiling (ncu) and timing.

    python -m fwi2d_b200.profile_case [--kind elastic|vti|acoustic] [--shots N]
        [--nt NT] [--shape S] [--mode forward|gradient] [--precision fp32|bf16|fp16]

Shots are copies of the single-shot elastic workload's geometry (401 x 801
grid at 5 m) on its true model; --mode gradient runs a forward with snapshots
then an adjoint with a seeded random adjoint source.  Prints the device times
of the last forward and adjoint (ms).
"""
import argparse

import numpy as np

from . import _capi as C
from . import workloads as W
from .propagator import Propagator, ShotSpec, make_params


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--kind", default="elastic", choices=["elastic", "vti", "acoustic"])
    ap.add_argument("--shots", type=int, default=4)
    ap.add_argument("--nt", type=int, default=8)
    ap.add_argument("--shape", type=int, default=-1)
    ap.add_argument("--mode", default="forward", choices=["forward", "gradient"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "bf16", "fp16"])
    a = ap.parse_args(argv)
    kind = {"elastic": C.ELASTIC, "vti": C.VTI, "acoustic": C.ACOUSTIC}[a.kind]
    prec = {"fp32": C.SNAP_FP32, "bf16": C.SNAP_BF16, "fp16": C.SNAP_FP16}[a.precision]
    wl = W.elastic_single(nt=a.nt)
    raw = W.vti_model() if kind == C.VTI else wl["true"]
    if kind == C.ACOUSTIC:
        raw = np.stack([raw[0], raw[2]])
    model = W.convert(kind, raw)
    nx, nz, d = model.shape[1], model.shape[2], wl["d"]
    sh = wl["shots"][0]
    shots = [ShotSpec(0, nx, a.nt, sh["sx"], sh["sz"], sh["rx"], sh["rz"]) for _ in range(a.shots)]
    pd = dict(wl["params"])
    pd.update(nt=a.nt, sub=1 if a.mode == "gradient" else 0)
    P = Propagator(0)
    P.set_model(kind, model, d, d)
    P.set_shots(make_params(**pd, tile_shape=a.shape, snapshot_precision=prec), shots)
    nc = P.ncomp()
    src = wl["src"].reshape(2, a.nt)[:nc]
    P.upload([src] * a.shots, False)
    P.run(False, store=a.mode == "gradient")
    P.sync()
    if a.mode == "gradient":
        rng = np.random.default_rng(0)
        P.upload([rng.standard_normal((nc * len(sh["rx"]), a.nt)).astype(np.float32)] * a.shots, True)
        P.run(True)
        P.sync()
    f, g = P.last_timing()
    print("forward %.3f ms  adjoint %.3f ms  plan %s" % (f, g, P.plan_info()))
    P.close()


if __name__ == "__main__":
    main()
