"""Sharding and result merging across ranks (gloo, world size 2, CPU only).

The GPU work of each rank is independent; these tests cover the host logic:
contiguous shard ranges that keep global shot indices, the counts merge
(dense histogram all-reduce and the object-gather path for wide registers)
and the per-set row gather used for batched energies/gradients.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dqsim_bosonic_b200.dist import counts_to_hist, hist_to_counts, shard_range


def test_shard_range_covers_everything_once():
    for total in (0, 1, 5, 4096, 4097):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shard_range(total, r, world)
                assert 0 <= lo <= hi <= total
                seen.extend(range(lo, hi))
            assert seen == list(range(total))
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def test_hist_roundtrip():
    counts = {"000": 3, "101": 2, "111": 1}
    h = counts_to_hist(counts, 3)
    assert h.tolist() == [3, 0, 0, 0, 0, 2, 0, 1]
    assert hist_to_counts(h, 3) == counts
    assert hist_to_counts(counts_to_hist({"": 7}, 0), 0) == {"": 7}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from dqsim_bosonic_b200.dist import gather_rows, merge_counts

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each rank counted its own shots
        local = {"00": 1 + rank, "11": 2} if rank == 0 else {"01": 5, "11": 1}
        merged = merge_counts(local, 2)
        wide = merge_counts({"1" * 30: 1, "0" * 30: rank}, 30)
        total = 5
        lo, hi = (0, 3) if rank == 0 else (3, 5)
        rows = gather_rows(np.arange(lo, hi, dtype=np.float64)[:, None] * [1.0, 10.0], total)
        q.put((rank, merged, wide, rows.tolist()))
    finally:
        dist.destroy_process_group()


def test_merge_across_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, merged, wide, rows in results:
        assert merged == {"00": 1, "01": 5, "11": 3}
        assert wide == {"1" * 30: 2, "0" * 30: 1}
        assert rows == [[float(i), 10.0 * i] for i in range(5)]
