"""The N > 1 path of bench.py on CPU: two gloo ranks shard independent RVE solves
round-robin (no collective on the data path), solve their shares with the CPU oracle,
and reduce the timing with max and the launch counts with sum over ranks.  Every RVE
is solved exactly once and gives the same result as a one-process run."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# four small elastic RVEs (32x32, one pore, different porosity)
CASES = [0.004, 0.006, 0.008, 0.010]


def _solve(porosity):
    import oracle

    pa = oracle.make_pa(20.0, 20.0, 32, 32, g0=0.5, yield_stress=1.0, porosity=porosity, n_pores=1)
    with oracle.Oracle(32, 32, pa, nl=1, niter=2000, eiter=1e-9, check_every=1000) as o:
        r = o.compute_eff_moduli(-4e-5, [1.0, 1.0, 0.0], 1)
    return r["num"]["kd"], r["num"]["kphi"]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    import oracle

    oracle.set_threads(1)
    mine = bench.shard(len(CASES), rank, world)
    res = {i: _solve(CASES[i]) for i in mine}
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    t_max = bench.reduce_over_ranks([float(rank + 1)], "max")[0]
    n_sum = bench.reduce_over_ranks([float(len(mine))], "sum")[0]
    if rank == 0:
        out.put((gathered, t_max, n_sum))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_sharding_and_reductions():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.shard(10, 0, 3) == [0, 3, 6, 9] and bench.shard(10, 2, 3) == [2, 5, 8]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, t_max, n_sum = q.get(timeout=240)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    merged = {}
    for part in gathered:
        for k, v in part.items():
            assert k not in merged  # no RVE solved twice
            merged[k] = v
    assert sorted(merged) == list(range(len(CASES)))
    assert t_max == 2.0 and n_sum == len(CASES)
    for i, phi in enumerate(CASES):
        assert merged[i] == pytest.approx(_solve(phi), rel=0, abs=0)
