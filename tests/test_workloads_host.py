"""Host-side pieces of the product: model conversion, synthetic workloads and
shot sharding."""
import numpy as np

import oracle as O
from fwi2d_b200 import workloads as W
from fwi2d_b200 import distributed as D


def test_convert_matches_reference_conversion():
    import glob, os
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    for name in ("elastic_fs_abs_f32.npz", "vti_fs_abs_f32.npz", "acoustic_neumann_f32.npz"):
        g = dict(np.load(os.path.join(gold, name)))
        kind = int(g["kind"])
        m = W.convert(kind, g["raw"])
        assert np.array_equal(m, g["model"]), name


def test_elastic_single_shapes():
    wl = W.elastic_single(nt=11)
    assert wl["true"].shape == (3, 801, 401)
    vp = wl["true"][0]
    z = np.arange(401) * 0.005
    base = (2.0 + 0.75 * z)[None, :]
    assert np.abs(vp / base - 1).max() <= 0.0500001
    assert len(wl["shots"][0]["rx"]) == 400
    assert wl["src"].shape == (2, 1, 11)


def test_vti_batch_geometry():
    wl = W.vti_batch(nshots=64, nt_max=5001)
    assert len(wl["shots"]) == 64
    eps, dl = wl["true"][4], wl["true"][3]
    assert 0.05 - 1e-6 <= eps.min() and eps.max() <= 0.20 + 1e-6
    assert -1e-6 <= dl.min() and dl.max() <= 0.10 + 1e-6
    for s in wl["shots"]:
        assert 0 <= s["x0"] and s["x0"] + s["nx"] <= 801
        assert 0.0 <= s["rx"].min() and s["rx"].max() <= 4.0
        assert 0.9 < (s["rx"].max() - s["rx"].min()) < 3.6
        assert int(1.2 / 4e-4) <= s["nt"] <= 5001


def test_shard_shots_partitions_and_balances():
    shots = [dict(nx=100 + 37 * (i % 5), nt=1000 + 100 * (i % 3)) for i in range(17)]
    for world in (1, 2, 3, 8):
        parts = [D.shard_shots(shots, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(17))
        loads = [sum(D.shot_cost(shots[i], 1) for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(D.shot_cost(s, 1) for s in shots)


def test_analyze_model_matches_reference():
    """The library's host analyzeModel (fwi2d_analyze_model) reproduces the
    reference's (we_op.cpp:267-474, fixtures written by its own build): the
    clipped model bit for bit and the derived dt, nt, sub, courant, tmax, vmax
    and vmin, over the dt / sub branches and the VTI, acoustic and
    acoustic-elastic cases."""
    import os
    import fwi2d_b200 as F
    g = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "analyze_model_f32.npz")))
    nx, nz, d = int(g["grid"][0]), int(g["grid"][1]), float(g["grid"][2])
    keys = ("vpmin", "vpmax", "vsmin", "vsmax", "rhomin", "rhomax", "deltamin", "deltamax", "epsilonmin",
            "epsilonmax", "soft_clip", "acoustic_elastic", "water_velocity", "courant", "dt", "sub")
    k = 0
    while "in%d" % k in g:
        chk = dict(zip(keys, g["check%d" % k]))
        for key in ("soft_clip", "acoustic_elastic", "sub"):
            chk[key] = int(chk[key])
        dnt, ddt = int(g["axis%d" % k][0]), float(g["axis%d" % k][1])
        m, r = F.analyze_model(g["in%d" % k], d, d, dnt, ddt, **chk)
        name = str(g["name%d" % k])
        assert np.array_equal(m, g["out%d" % k]), name
        ref = dict(zip(("courant", "dt", "sub", "nt", "tmax", "vmax", "vmin"), g["res%d" % k]))
        for key in ("courant", "dt", "tmax", "vmax", "vmin"):
            assert np.float32(r[key]) == np.float32(ref[key]), (name, key, r[key], ref[key])
        assert r["nt"] == int(ref["nt"]) and r["sub"] == int(ref["sub"]), name
        k += 1
    assert k == 8


def test_dipole_tables_match_reference():
    """fwi2d_dipole_weights reproduces dipole_m3::findIndicesWeights
    (injector.cpp:241-326, tables written by the reference build), including
    dipoles at the free-surface row and at horizontal and vertical dips."""
    import os
    from fwi2d_b200.propagator import dipole_tables
    g = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dipole_f32.npz")))
    d = float(g["d"])
    xi, zi, xw, zw = dipole_tables(g["rx"], g["rz"], g["rdip"], float(g["gl"]), int(g["nx"]), int(g["nz"]), d, d)
    assert np.array_equal(xi, g["xind"]) and np.array_equal(zi, g["zind"])
    assert np.array_equal(xw, g["xw"]) and np.array_equal(zw, g["zw"])
