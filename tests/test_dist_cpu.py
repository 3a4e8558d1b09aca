"""Shot sharding and the FP64 gradient / misfit all-reduce with world size 2 on
gloo (CPU), through owl_b200.dist.ShotSharding -- the rank logic bench.py runs
with NCCL: the summed per-rank gradients equal the single-process gradient over
all shots, and every shot's misfit lands at its index. The shards are uneven
(3 shots: 2 on one rank, 1 on the other). The per-shot gradients come from the
FP64 oracle here (no GPU needed)."""
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
    from owl_b200.dist import ShotSharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        if rank == fail_rank:
            raise RuntimeError("injected rank failure")
        d, vp, rho, shots, (nx, nz, dx, dt) = _case()
        sh = ShotSharding(shots, rank, world)
        ps = prepare(sh.local(shots), nx, nz, dx, dt)
        obs = oracle.ac2d_forward(d, vp * 1.03, rho, ps, "f64")
        mf, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=30)
        # the rank's FP32 gradient, as the library returns it, summed in FP64
        g64, m64 = sh.reduce(torch.from_numpy(g.astype(np.float32)), torch.from_numpy(mf))
        oom_anywhere = sh.any_rank(rank == 1)
        out[rank] = {"mine": sh.mine, "g": g64.numpy().tolist(), "m": m64.numpy().tolist(),
                     "dtype": str(g64.dtype), "any": oom_anywhere}
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
    r0, r1 = res[0], res[1]
    assert isinstance(r0, dict) and isinstance(r1, dict), (r0, r1)
    assert sorted(r0["mine"] + r1["mine"]) == [0, 1, 2] and len(r0["mine"]) != len(r1["mine"])
    assert r0["dtype"] == "torch.float64" and r0["any"] and r1["any"]
    g0, g1 = np.array(r0["g"]), np.array(r1["g"])
    assert np.array_equal(g0, g1) and np.array_equal(np.array(r0["m"]), np.array(r1["m"]))
    d, vp, rho, shots, (nx, nz, dx, dt) = _case()
    ps = prepare(shots, nx, nz, dx, dt)
    obs = oracle.ac2d_forward(d, vp * 1.03, rho, ps, "f64")
    mf, g, _ = oracle.ac2d_gradient(d, vp, rho, ps, obs, adj_kind=0, k=30)
    # per-rank FP32 gradients summed in FP64: within FP32 rounding of the FP64 total
    assert np.linalg.norm(g0 - g) <= 1e-6 * np.linalg.norm(g)
    # misfits are per shot, each computed by one rank: exact at their global index
    assert np.allclose(np.array(r0["m"]), mf, rtol=1e-12, atol=0)


def test_rank_failure_surfaces_as_error():
    res = _run(2, fail_rank=1)
    assert "injected rank failure" in res[1]
    assert isinstance(res[0], str)  # the surviving rank's all-reduce ended with an error, not a hang
