"""The multi-GPU (replica) host logic on CPU: two gloo ranks in child
processes.  Shards cover the segments once; the whole-job rate uses the
slowest rank's time on every rank; gathered skies arrive in segment order
on rank 0 (complex tensors included)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from sphradiometer_b200.replicas import gather_skies, shard_range, whole_job_rate


def test_shards_cover_every_segment_once():
    for n_seg in (0, 1, 7, 64, 4097):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                a, b = shard_range(n_seg, r, world)
                assert 0 <= b - a <= n_seg // world + 1
                got.extend(range(a, b))
            assert got == list(range(n_seg))
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, n_seg, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r "took" 10 + 5 r ms for 100 units per step, 3 steps
        rate, slowest = whole_job_rate(100, 3, 10.0 + 5.0 * rank)
        a, b = shard_range(n_seg, rank, world)
        seg = torch.arange(a, b, dtype=torch.float64)
        local = torch.complex(seg[:, None] * torch.ones(1, 4, dtype=torch.float64), -seg[:, None] * torch.ones(1, 4, dtype=torch.float64))
        full = gather_skies(local, n_seg)
        ok = full is None if rank else bool(torch.equal(full.real[:, 0], torch.arange(n_seg, dtype=torch.float64)) and torch.equal(full.imag, -full.real))
        q.put((rank, rate, slowest, ok))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, n_seg = 2, 11
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n_seg, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, slowest, ok in res:
        assert slowest == 15.0
        assert rate == pytest.approx(world * 100 * 3 / 0.015)
        assert ok
