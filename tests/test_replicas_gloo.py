"""Multi-rank host logic of the replica / query-shard path, as two gloo ranks
on CPU (no GPU): shard ranges, max-over-ranks timing, result gathering, and
index_shard with a stand-in indexing function."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ebsdtorch_b200.replicas import gather_shards, index_shard, max_over_ranks, shard_range


def test_shard_range_covers_exactly():
    for n in (0, 1, 7, 262144, 1001):
        for w in (1, 2, 3, 8):
            ranges = [shard_range(n, r, w) for r in range(w)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a1 == b0 for (_, b0), (a1, _) in zip(ranges, ranges[1:]))
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _fake_index(master_patterns, geometry, experiment_patterns, **kw):
    """Stand-in for the GPU indexer: orientation = (pattern mean, 0, 0, 0)."""
    m = experiment_patterns.patterns.flatten(1).mean(1)
    q = torch.stack((m, torch.zeros_like(m), torch.zeros_like(m), torch.zeros_like(m)), 1)
    experiment_patterns.set_raw_indexing_results(q[:, None, :], m[:, None], phase_id=0)
    experiment_patterns.combine_indexing_results(higher_is_better=True)


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert max_over_ranks(1.0 + rank) == float(world)
        n = 11
        a, b = shard_range(n, rank, world)
        full = gather_shards(torch.arange(a, b, dtype=torch.float32).view(-1, 1).repeat(1, 3), n)
        assert torch.equal(full[:, 0], torch.arange(n, dtype=torch.float32))
        from ebsdtorch_b200.ebsd.experiment_pats import ExperimentPatterns

        pats = torch.arange(n, dtype=torch.float32).view(n, 1, 1).repeat(1, 4, 4)
        exp = ExperimentPatterns(pats)
        sa, sb = index_shard(_fake_index, exp, master_patterns=None, geometry=None)
        assert (sa, sb) == (a, b)
        assert torch.equal(exp.orientations[:, 0], torch.arange(n, dtype=torch.float32))
        assert exp.raw_indexing_results[0][0].shape[0] == b - a
        out[rank] = 1
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert dict(out) == {0: 1, 1: 1}
