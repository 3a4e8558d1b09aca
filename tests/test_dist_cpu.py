"""Shot sharding and the gradient all-reduce with world size 2 on gloo (CPU):
the summed per-rank gradients equal the single-process gradient over all shots.
The per-shot gradients come from the FP64 oracle here (no GPU needed); on GPUs
the same rank logic runs with NCCL in bench.py."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from owl_b200.dist import shard_shots


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _case():
    from cases import desc, prepare, random_model, small_shots
    nx, nz, dx, dt, nt = 36, 30, 10.0, 1e-3, 120
    d = desc(nx, nz, dx, dt, nt, pml=8)
    vp, rho = random_model(nx, nz, seed=3)
    shots = small_shots(nx, nz, dx)
    return d, vp, rho, shots, (nx, nz, dx, dt)


def _worker(rank, world, port, out, fail_rank):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import datetime
    import torch.distributed as dist
    import oracle
    from cases import prepare
    from owl_b200.dist import allreduce_sum, shard_shots
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        if rank == fail_rank:
            raise RuntimeError("injected rank failure")
        d, vp, rho, shots, (nx, nz, dx, dt) = _case()
        mine = shard_shots(shots, rank, world)
        ps = prepare([shots[i] for i in mine], nx, nz, dx, dt)
        obs = oracle.ac2d_forward(d, vp * 1.03, rho, ps, "f64")
        _, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=30)
        t = torch.from_numpy(g.copy())
        allreduce_sum(t)
        out[rank] = t.numpy().tolist()
    except Exception as e:  # the failing rank leaves between steps; the peer's collective errors out
        out[rank] = repr(e)
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank=-1):
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        if p.is_alive():
            p.kill()
    return dict(out)


def test_shard_balances_and_partitions():
    from owl_b200.geometry import Receiver, Shot, Source
    shots = [Shot(i, [Source(x=0, z=0)], [Receiver(x=0, z=0)] * (10 + 7 * i)) for i in range(9)]
    parts = [shard_shots(shots, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == list(range(9))
    loads = [sum(len(shots[i].receivers) for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(len(s.receivers) for s in shots)


def test_allreduce_gradient_world2():
    import oracle
    from cases import prepare
    res = _run(2)
    assert set(res) == {0, 1}
    g0, g1 = np.array(res[0]), np.array(res[1])
    d, vp, rho, shots, (nx, nz, dx, dt) = _case()
    ps = prepare(shots, nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vp * 1.03, rho, ps, "f64")
    _, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=30)
    assert np.allclose(g0, g1, rtol=0, atol=0)
    assert np.linalg.norm(g0 - g) <= 1e-12 * np.linalg.norm(g)


def test_rank_failure_surfaces_as_error():
    res = _run(2, fail_rank=1)
    assert "injected rank failure" in res[1]
    assert isinstance(res[0], str)  # the surviving rank's all-reduce ended with an error, not a hang
