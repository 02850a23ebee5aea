"""Multi-rank host logic on CPU: two gloo ranks split a solve's irreducible
q-points, each computes its modes' rates with the oracle, and the all-gather
reproduces the single-process rates exactly."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fourphonon_b200 import shard


def test_partition_balanced_and_complete():
    w = np.arange(1, 17, dtype=float)
    parts = shard.partition_qpoints(16, 3, w)
    assert parts[0][0] == 0 and parts[-1][1] == 16
    for a, b in zip(parts, parts[1:]):
        assert a[1] == b[0]
    loads = [w[a:b].sum() for a, b in parts]
    assert max(loads) - min(loads) <= w.max()
    assert shard.partition_qpoints(5, 8)[-1] == (5, 5) or sum(b - a for a, b in shard.partition_qpoints(5, 8)) == 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import helpers as H
        import oracle as O

        s = H.cached_solve("diamond", (4, 4, 4))
        parts = shard.partition_qpoints(s.nlist, world)
        m0, m1 = shard.mode_range(parts[rank], s.nb)
        rp, rm, _, _ = O.Oracle(s).rta3(m0, m1)
        full = shard.gather_modes(rp + rm, parts[rank], s.nb, s.nlist)
        tmax = shard.reduce_max(float(rank + 1))
        if rank == 0:
            np.save(out, np.concatenate([full, [tmax]]))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_matches_single_process(tmp_path):
    import helpers as H
    import oracle as O

    out = str(tmp_path / "r.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    got = np.load(out)
    s = H.cached_solve("diamond", (4, 4, 4))
    rp, rm, _, _ = O.Oracle(s).rta3()
    assert np.array_equal(got[:-1], rp + rm)
    assert got[-1] == 2.0
