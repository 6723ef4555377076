"""Multi-rank host logic on CPU (gloo, world size 2): channel partitioning
over ranks, the max-over-ranks timing reduction, gathering results on rank
0, and the replica semantics (each rank correlates its own channels with the
oracle; together they equal the single-process result)."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from ftd_b200.shard import (gather_to_rank0, max_over_ranks, partition_channels,  # noqa: E402
                            rank_load)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, shapes, seeds, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle
        parts = partition_channels(shapes, world)
        mine = parts[rank]
        results = {}
        for c in mine:
            n, k = shapes[c]
            qc = oracle.gaussian_qc(seeds[c], 1, n, k)
            results[c] = oracle.herk_qc(qc, n, k, 1)[0]
        t = max_over_ranks(10.0 + rank, dist)
        gathered = gather_to_rank0(results, dist)
        if rank == 0:
            merged = {}
            for r in gathered:
                merged.update(r)
            out_q.put((t, parts, merged))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    shapes = [(int(rng.integers(64, 512)), int(rng.integers(1, 16)) * 64) for _ in range(37)]
    for world in (1, 2, 3, 8):
        parts = partition_channels(shapes, world)
        flat = sorted(c for p in parts for c in p)
        assert flat == list(range(len(shapes)))
        loads = [rank_load(shapes, p) for p in parts]
        biggest = max(8.0 * n * (n + 1) / 2 * k for n, k in shapes)
        assert max(loads) - min(loads) <= biggest  # LPT bound
    with pytest.raises(ValueError):
        partition_channels(shapes, 0)


def test_two_gloo_ranks_replicas():
    shapes = [(48, 64), (96, 128), (40, 32), (130, 64), (64, 256), (17, 16)]
    seeds = [100 + c for c in range(len(shapes))]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, shapes, seeds, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, parts, merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert t == 11.0                      # the slower rank's time
    assert sorted(parts[0] + parts[1]) == list(range(len(shapes)))
    from oracle import oracle
    for c, (n, k) in enumerate(shapes):  # replicas == one process
        ref = oracle.herk_qc(oracle.gaussian_qc(seeds[c], 1, n, k), n, k, 1)[0]
        assert np.array_equal(merged[c], ref)
