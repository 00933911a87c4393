"""Multi-rank sharding of one evaluation on CPU (gloo, world size 2): disjoint point blocks,
partial sums from the oracle standing in for each rank's GPU pass, one all-reduce, compared
with the single-process sum."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from phf_pcc_b200.distributed import point_range


@pytest.mark.parametrize("n,w", [(10, 3), (112, 2), (7, 8), (3200, 4)])
def test_point_ranges_partition_the_grid(n, w):
    ranges = [point_range(n, r, w) for r in range(w)]
    assert ranges[0][0] == 0 and ranges[-1][1] == n
    for (a, b), (c, d) in zip(ranges, ranges[1:]):
        assert b == c
    sizes = [b - a for a, b in ranges]
    assert max(sizes) - min(sizes) <= 1


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import phf_oracle_c as corc
        from phf_pcc_b200.distributed import allreduce_accumulators
        from tests._golden import grid_kwargs, htwo_mo, load

        c = load("j1_c2v_b1")
        kw = grid_kwargs(c)
        npts = kw["ngrid"][0] * kw["ngrid"][1] * kw["npg"]
        b, e = point_range(npts, rank, world)
        Hm, Sm, Gm, Rm = corc.buildhsg(c["HOne"], htwo_mo(c), c["Ref"], c["Z"], omega_list=np.arange(b, e),
                                       nthreads=1, **kw)
        ts = [torch.from_numpy(np.ascontiguousarray(x)) for x in (Hm, Sm, Gm, Rm)]
        allreduce_accumulators(ts)
        if rank == 0:
            out.put([t.numpy() for t in ts])
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sum_equals_single_process():
    from oracle import phf_oracle_c as corc
    from tests._golden import grid_kwargs, htwo_mo, load

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    c = load("j1_c2v_b1")
    ref = corc.buildhsg(c["HOne"], htwo_mo(c), c["Ref"], c["Z"], nthreads=1, **grid_kwargs(c))
    for x, y in zip(got, ref):
        assert np.abs(x - y).max() <= 1e-12 * max(1.0, np.abs(y).max())
