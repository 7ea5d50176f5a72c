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


# ------------------------------------------------------------------------------
# One buffer split across ranks (parallel.compress_split): each rank holds a
# contiguous byte range; the ranks sum their histograms, scan their bit counts
# and gather their encoded windows to rank 0, which ORs them together.  The
# per-part encoder here is the oracle's whole-stream encoding cut down to what
# the part owns (its bits [bit0, end) and the gap entries k with
# bit0 < 128(k+1) <= end) -- the contract hgap_encode_part_prepared keeps on
# the GPU (tests/test_gpu_split.py checks that side).

def _split_data(n=300_003, seed=11):
    rng = np.random.default_rng(seed)
    p = 1.0 / np.arange(1, 257) ** 1.1
    return rng.choice(256, size=n, p=p / p.sum()).astype(np.uint8)


def _cuts(n, world, seed=5):
    rng = np.random.default_rng(seed)
    inner = sorted(int(c) for c in rng.integers(0, n, size=world - 1))
    return [0] + inner + [n]


class _OraclePartCodec:
    def __init__(self, full):
        from oracle import oracle as O
        self.O = O
        self.full = full
        self.cb = O.codebook(O.histogram(full))
        self.bits, self.gaps, self.total = O.encode(full, self.cb)

    def histogram(self, x):
        return self.O.histogram(x.numpy())

    def encode(self, x, book, bit0, part_bits):
        import torch
        end = bit0 + part_bits
        w0, w1 = bit0 >> 5, (end + 31) // 32
        words = np.asarray(self.bits[w0:w1], np.uint64).copy()
        for i in range(len(words)):
            lo = max(bit0, 32 * (w0 + i)) - 32 * (w0 + i)
            hi = min(end, 32 * (w0 + i) + 32) - 32 * (w0 + i)
            words[i] &= ((1 << (hi - lo)) - 1) << (32 - hi)
        g0, g1 = bit0 >> 10, ((end + 127) // 128 + 7) // 8
        gw = np.asarray(self.gaps[g0:g1], np.uint64).copy()
        for i in range(len(gw)):
            keep = 0
            for j in range(8):
                k = 8 * (g0 + i) + j
                if bit0 < 128 * (k + 1) <= end:
                    keep |= 0xF << (4 * j)
            gw[i] &= keep
        if not x.numel():
            words, gw = words[:0], gw[:0]
        to = lambda a: torch.from_numpy(a.astype(np.uint32).view(np.int32).copy())
        return w0, to(words), g0, to(gw)


def _split_rank(rank, world, port, q):
    import torch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full = _split_data()
        cuts = _cuts(full.size, world)
        part = torch.from_numpy(full[cuts[rank]:cuts[rank + 1]].copy())
        out = PL.compress_split(part, codec=_OraclePartCodec(full))
        if rank == 0:
            book, n, sizes, bits, gaps = out
            q.put((n, sizes.bits, bits.numpy().tobytes(), gaps.numpy().tobytes()))
        else:
            assert out is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_split_one_buffer(world):
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        n, nbits, bits, gaps = q.get(timeout=300)
    finally:
        for p in procs:
            p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    full = _split_data()
    cb = O.codebook(O.histogram(full))
    ref_bits, ref_gaps, total = O.encode(full, cb)
    assert n == full.size and nbits == total
    assert bits == np.asarray(ref_bits, np.uint32).tobytes()
    assert gaps == np.asarray(ref_gaps, np.uint32).tobytes()


def test_part_starts_and_stitch_on_cpu():
    import torch
    assert PL.part_starts([5, 0, 7, 3]) == [0, 5, 5, 12]
    a = torch.tensor([0x0F000000], dtype=torch.int32)
    b = torch.tensor([0x00F00000, 7], dtype=torch.int32)
    bits, gaps = PL.stitch_parts([(1, a, 0, a[:0]), (1, b, 0, b[:0])], 3, 0)
    assert bits.tolist() == [0, 0x0FF00000, 7]
