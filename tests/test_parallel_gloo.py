"""The multi-rank path of a sharded batch, as world-size-2 gloo ranks on the
CPU: the partition covers every buffer once and balances bytes, the
max-over-ranks reduction and the result gather work, and the containers
the ranks produce for their shares equal a single process's.  The per-buffer
codec here is the CPU oracle (no GPU in this test); on the GPU each rank runs
the batched path on its share, with no collective on the data path."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from huffman_coding_gap_arrays_b200 import parallel as PL


def _sizes(count=37, seed=3):
    rng = np.random.default_rng(seed)
    return [int(x) for x in np.exp(rng.uniform(np.log(100), np.log(200000), count))]


def _buffer(i, n):
    rng = np.random.default_rng(1000 + i)
    return rng.choice(256, size=n, p=np.arange(256, 0, -1) / np.arange(256, 0, -1).sum()).astype(np.uint8)


def _container(i, n):
    from oracle import oracle as O
    x = _buffer(i, n)
    cb = O.codebook(O.histogram(x))
    bits, gaps, total = O.encode(x, cb)
    return O.container(cb, n, bits, gaps, (total + 127) // 128)


def test_partition_covers_and_balances():
    sizes = _sizes(200)
    for world in (1, 2, 3, 8):
        parts = PL.shard_by_bytes(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
        assert parts == PL.shard_by_bytes(sizes, world)  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = PL.shard_by_bytes(sizes, world)[rank]
        local = {i: _container(i, sizes[i]) for i in mine}
        slowest = PL.max_over_ranks(float(rank + 1))
        merged = PL.gather_results(local)
        if rank == 0:
            q.put((slowest, sorted(merged), {k: len(v) for k, v in merged.items()},
                   {k: v for k, v in merged.items() if k < 4}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_a_batch():
    sizes = _sizes()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        slowest, keys, lens, some = q.get(timeout=300)
    finally:
        for p in procs:
            p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert slowest == 2.0
    assert keys == list(range(len(sizes)))
    for i in range(len(sizes)):
        assert lens[i] == len(_container(i, sizes[i]))
    for i, v in some.items():
        assert v == _container(i, sizes[i])
