"""Shot sharding across processes on CPU (gloo, world size 2).

Each rank propagates its share of the shots through the oracle (standing in
for the device kernels, which the GPU tests cover) and the per-rank gradients
and misfits are summed with fwi2d_b200.distributed.allreduce_sum.  The sum
must equal the single-process sum over all shots, which is what the
reference's MPI_Allreduce of per-rank gradients produces
(src/include/optimization.hpp:609-618)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _shots():
    return [dict(nx=48, nt=60, sx=0.12 + 0.08 * k) for k in range(5)]


def _shot_grad(shot, seed=3):
    import oracle as O
    from tests import cases as K
    nx, nz, d, nt = shot["nx"], 36, 0.01, shot["nt"]
    lib = O.Port(32)
    mc = K.converted(0, K.model_case(0, nx, nz, d, seed=seed))
    rl = (np.linspace(0.05, 0.42, 8).astype(np.float32), np.full(8, 0.02, np.float32))
    sl = (np.array([shot["sx"]], np.float32), np.array([0.03], np.float32))
    src = K.sources(2, nt, 1e-3)
    par = O.make_par(**K.par_dict(nt=nt, dt=1e-3), ns=1, nr=8)
    rcv, full = K.oracle_forward(lib, 0, mc, src, par, nx, nz, d, sl, rl)
    g = K.oracle_adjoint(lib, 0, mc, np.ascontiguousarray(rcv[:, :, ::-1]), par, nx, nz, d, sl, rl, full)
    return g.astype(np.float64), float(np.sum(rcv.astype(np.float64) ** 2))


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from fwi2d_b200 import distributed as D
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shots = _shots()
        mine = D.shard_shots(shots, rank, world, nz=36)
        g = torch.zeros((3, 48, 36), dtype=torch.float64)
        f = torch.zeros(1, dtype=torch.float64)
        for i in mine:
            gi, fi = _shot_grad(shots[i])
            g += torch.from_numpy(gi)
            f += fi
        D.allreduce_sum(g)
        D.allreduce_sum(f)
        out.put((rank, mine, g.numpy(), float(f[0])))
    finally:
        dist.destroy_process_group()


def test_two_rank_gradient_sum_matches_serial():
    import oracle as O
    if not os.path.exists(O.port_path(32)):
        pytest.skip("oracle not built")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda r: r[0])
    assert sorted(res[0][1] + res[1][1]) == list(range(5))
    assert not set(res[0][1]) & set(res[1][1])
    g_ser = sum(_shot_grad(s)[0] for s in _shots())
    f_ser = sum(_shot_grad(s)[1] for s in _shots())
    for _, _, g, f in res:
        assert np.allclose(g, g_ser, rtol=1e-12, atol=1e-12 * np.abs(g_ser).max())
        assert abs(f - f_ser) <= 1e-12 * f_ser
