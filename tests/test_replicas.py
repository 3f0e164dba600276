"""Host logic of the replica multi-GPU mode (glac_b200/replicas.py) with gloo
ranks on CPU: partition of an uneven ensemble, gather of per-lattice
observables to rank 0, max-over-ranks timing."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from glac_b200.replicas import partition, replica_statistics


def test_partition_balances_sites_and_covers_every_lattice():
    from glac_b200.ensemble import draw_ensemble
    dims, _ = draw_ensemble(20261203, 64)
    sites = [int(np.prod(d)) for d in dims]
    for world in (1, 2, 4, 8):
        parts = partition(sites, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(sites[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sites)  # greedy bound
        assert partition(sites, world) == parts  # deterministic
    with pytest.raises(ValueError):
        partition(sites, 0)


def test_replica_statistics():
    m, e = replica_statistics({0: [1.0, 2.0], 1: [3.0, 2.0]})
    assert np.allclose(m, [2.0, 2.0]) and np.allclose(e, [1.0, 0.0])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, sites, q):
    import datetime

    import torch.distributed as dist

    from glac_b200.replicas import gather_observables, max_over_ranks, partition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = partition(sites, world)[rank]
        # stand-in for per-lattice observables: a row that identifies the lattice
        local = {i: np.array([i, sites[i], rank], np.float64) for i in mine}
        merged = gather_observables(local, world, rank)
        t = max_over_ranks(0.5 + rank, world)
        q.put((rank, None if merged is None else {k: v.tolist() for k, v in merged.items()}, t))
    finally:
        dist.destroy_process_group()


def test_gather_and_max_over_two_gloo_ranks():
    sites = [8192, 41472, 131072, 663552, 8192, 131072, 41472]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, sites, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, merged, t = q.get(timeout=120)
        res[r] = (merged, t)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    merged0, t0 = res[0]
    assert res[1][0] is None
    assert sorted(merged0) == list(range(len(sites)))
    owner = {i: r for r, part in enumerate(partition(sites, 2)) for i in part}
    for i, row in merged0.items():
        assert row == [i, sites[i], owner[i]]
    assert t0 == res[1][1] == 1.5
