"""Multi-GPU: a batch of independent buffers shards across ranks by bytes.

Buffers are independent (each has its own codebook and stream), so the
batched path needs no collective on its data path: every rank compresses
and decompresses its own share, one process per GPU.  The only exchanges
are the launch-time agreement on the partition (computed identically on
every rank from the sizes, no message), the max-over-ranks of the device
time, and -- if a caller wants every result on one rank -- a gather of the
finished containers.

One buffer can also be split across ranks (compress_split): each rank encodes
its contiguous byte range from the stream bit where it starts, after a sum of
the 256-bin histograms and a scan of the ranks' bit counts.
"""
from __future__ import annotations

import heapq

import numpy as np

import torch
import torch.distributed as dist


def shard_by_bytes(sizes, world: int) -> list:
    """Deterministic partition of buffer indices over `world` ranks that
    balances bytes: largest buffers first, each to the least-loaded rank
    (ties to the lowest rank); each rank's indices ascend."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over the process group (the slowest rank's time)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: dict, dst: int = 0):
    """Gathers {buffer index: bytes} from every rank to rank `dst`; returns
    the merged dict there (None elsewhere).  Off the timed path."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    out = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(local, out, dst=dst)
    if dist.get_rank() != dst:
        return None
    merged = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"buffer {k} produced by two ranks")
            merged[k] = v
    return merged


# ------------------------------------------------------------------------------
# One buffer split across devices: each rank holds and encodes a contiguous
# byte range.  The exchanges are the 256-bin histogram sum (one codebook for
# all parts), an 8-byte-per-rank scan of the parts' bit counts (where each
# part starts in the stream), and the gather of the encoded windows; the words
# and gap words two neighbouring parts share are joined by OR.

class DevicePartCodec:
    """The per-rank codec of a split buffer: libhgap.so on this rank's GPU."""

    def __init__(self):
        self._enc = None

    def histogram(self, x):
        from .codec import Encoder
        n = x.numel()
        self._enc = Encoder(max(n, 1), x.device)
        return self._enc.histogram(x).cpu().numpy().astype(np.uint32)

    def encode(self, x, book, bit0: int, part_bits: int):
        return self._enc.encode_part(x, book, bit0, part_bits)


def part_starts(part_bits) -> list:
    """Exclusive prefix sum: the stream bit where each part starts."""
    out, acc = [], 0
    for b in part_bits:
        out.append(acc)
        acc += int(b)
    return out


def stitch_parts(parts, words: int, gap_words: int, device=None):
    """The stream from its parts' windows: parts = [(first word, words,
    first gap word, gap words)]; every word is the OR of the parts' words at
    that place (a part's boundary words hold only its own bits)."""
    bits = torch.zeros(max(words, 1), dtype=torch.int32, device=device)
    gaps = torch.zeros(max(gap_words, 1), dtype=torch.int32, device=device)
    for w0, bw, g0, gw in parts:
        if bw.numel():
            bits[w0:w0 + bw.numel()] |= bw.to(bits.device)
        if gw.numel():
            gaps[g0:g0 + gw.numel()] |= gw.to(gaps.device)
    return bits[:words], gaps[:gap_words]


def compress_split(x_local, codec=None, dst: int = 0, group=None):
    """Compresses one buffer held as contiguous parts by the ranks of the
    process group (rank r holds part r, in order).  Returns, on rank ``dst``,
    (book, n, sizes, bits, gaps) -- identical to compressing the whole buffer
    on one device -- and None elsewhere.  ``codec`` (DevicePartCodec by
    default) supplies the per-part histogram and encode."""
    from .codec import Codebook
    codec = codec or DevicePartCodec()
    multi = dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1
    world = dist.get_world_size(group) if multi else 1
    rank = dist.get_rank(group) if multi else 0
    dev = x_local.device
    cdev = torch.device("cpu") if not multi or dist.get_backend(group) == "gloo" else dev
    hist = np.asarray(codec.histogram(x_local), np.uint32)
    ghist = torch.from_numpy(hist.astype(np.int64)).to(cdev)
    if multi:
        dist.all_reduce(ghist, op=dist.ReduceOp.SUM, group=group)
    book, sizes = Codebook.from_histogram(ghist.cpu().numpy())
    mine = torch.tensor([book.encoded_bits(hist), x_local.numel()], dtype=torch.int64, device=cdev)
    if multi:
        every = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(every, mine, group=group)
    else:
        every = [mine]
    counts = [(int(t[0]), int(t[1])) for t in every]
    starts = part_starts([c[0] for c in counts])
    n_total = sum(c[1] for c in counts)
    w0, bw, g0, gw = codec.encode(x_local, book, starts[rank], counts[rank][0])
    if not multi:
        bits, gaps = stitch_parts([(w0, bw, g0, gw)], sizes.words, sizes.gap_words, dev)
        return book, n_total, sizes, bits, gaps
    # every rank knows every part's window sizes from the counts: pad to the largest
    lens = []
    for r in range(world):
        b0, end = starts[r], starts[r] + counts[r][0]
        lens.append(((end + 31) // 32 - (b0 >> 5) if counts[r][1] else 0,
                     ((end + 127) // 128 + 7) // 8 - (b0 >> 10) if counts[r][1] else 0))
    wmax = max(1, max(l[0] for l in lens))
    gmax = max(1, max(l[1] for l in lens))
    pb = torch.zeros(wmax, dtype=torch.int32, device=cdev)
    pg = torch.zeros(gmax, dtype=torch.int32, device=cdev)
    pb[:bw.numel()] = bw.to(cdev)
    pg[:gw.numel()] = gw.to(cdev)
    lb = [torch.empty_like(pb) for _ in range(world)] if rank == dst else None
    lg = [torch.empty_like(pg) for _ in range(world)] if rank == dst else None
    dist.gather(pb, lb, dst=dst, group=group)
    dist.gather(pg, lg, dst=dst, group=group)
    if rank != dst:
        return None
    parts = [(starts[r] >> 5, lb[r][:lens[r][0]], starts[r] >> 10, lg[r][:lens[r][1]]) for r in range(world)]
    bits, gaps = stitch_parts(parts, sizes.words, sizes.gap_words, dev)
    return book, n_total, sizes, bits, gaps


__all__ = ["shard_by_bytes", "max_over_ranks", "gather_results", "DevicePartCodec", "part_starts",
           "stitch_parts", "compress_split"]
