"""Serving: a request loop with continuous batching (no counterpart in the
reference).

Requests -- compress a device buffer, or decompress a stream produced by the
batched path -- arrive over time.  The loop, running on the host:

  * admits arrived requests, oldest first, into the next batch while the
    batch stays under ``max_batch`` requests and the device memory the
    in-flight batches hold stays under the HBM budget (a batch is admitted on
    an upper bound of its allocations from the library's own size queries,
    and then charged the bytes it really allocated);
  * launches each batch as one batched compress and/or one batched
    decompress on its own stream (up to ``max_inflight`` batches at once,
    so requests that arrive while others are on the GPU start as soon as a
    slot and memory free up, and their work overlaps on the device);
  * retires batches whose completion event has fired, releasing their
    memory and stamping their requests' completion times.

Codebooks and decoder tables are built on the device inside each batch and
never leave it.  Payloads and results stay in HBM (the latency is queueing
plus GPU service, not network or PCIe time).  The launch shape of each batch
comes from a ``LearnedTuner`` (its features: the batch's own size and byte
statistics -- a decompress request's from its codebook and stream size, a
compress request's from the traffic compressed so far), from one fixed shape,
or -- for comparison -- requests run one by one through the plain
single-buffer path.
"""
from __future__ import annotations

import ctypes as C
import gc
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import codec
from ._lib import BatchEntry, check, lib
from .batch import ENTRY_BYTES, BatchCodec, LaunchConfig, _upload
from .codec import _stream


@dataclass
class Request:
    rid: int
    arrival: float                      # seconds after the start of the run
    kind: str                           # "compress" | "decompress"
    data: torch.Tensor | None = None    # compress: uint8 device buffer
    stream: "EncodedStream | None" = None  # decompress: what to decode
    # filled by the server
    start: float = float("nan")         # launch time of its batch
    done: float = float("nan")          # completion time
    result: object = None

    @property
    def nbytes(self) -> int:
        return int(self.data.numel()) if self.kind == "compress" else int(self.stream.entry.n)


def entry_features(e) -> np.ndarray:
    """Byte statistics of one encoded stream from its entry alone: code bits
    per byte (the code's mean length, within a bit of the entropy), the
    longest code, and the share of bytes with codes longer than the decoder's
    11-bit level-1 prefix, as the code itself implies (a code of length l
    stands for probability 2^-l)."""
    lens = np.array([e.symbols[k].length for k in range(e.symbol_count)], np.float64)
    if e.n == 0 or lens.size == 0:
        return np.zeros(3, np.float32)
    return np.array([e.bits / e.n, lens.max(), float(np.exp2(-lens[lens > 11]).sum())], np.float32)


@dataclass
class EncodedStream:
    """One buffer's encoded stream in device memory, as the batched path
    produced it (entry with sizes and codebook, bitstream and gap array)."""
    entry: BatchEntry
    bits: torch.Tensor   # int32 view of u32 words, 16-byte aligned start
    gaps: torch.Tensor
    owner: object = None  # keeps the arenas the views point into alive
    features: np.ndarray | None = None
    class_bit: int = 0    # 1 << its decoder class (hgap_batch_decoder_class), 0 when empty

    def __post_init__(self):
        if self.features is None:
            self.features = entry_features(self.entry)
        e = self.entry
        c = int(lib().hgap_batch_decoder_class(e.symbols, e.symbol_count)) if e.symbol_count else 255
        self.class_bit = 1 << c if c < 8 else 0

    @property
    def book(self) -> "codec.Codebook":
        """Its codebook on the host (built once: payloads are decoded many times)."""
        b = getattr(self, "_book", None)
        if b is None:
            e = self.entry
            syms = np.array([e.symbols[k].symbol for k in range(e.symbol_count)], np.uint8)
            lens = np.array([e.symbols[k].length for k in range(e.symbol_count)], np.uint8)
            b = self._book = codec.Codebook.from_symbols(syms, lens)
        return b

    def to_compressed(self):
        e = self.entry
        sizes = codec.StreamSizes(int(e.bits), int(e.words), int(e.segments), int(e.gap_words))
        return codec.Compressed(self.book, int(e.n), sizes, self.bits, self.gaps)


# The batch features the tuner sees in serving, on a coarse grid: log2 bytes in
# 1/8 steps, code bits per byte to a whole bit, the longest code in three bands
# (11 or less: no level-2 lookups; 12-13; 14 and up), the level-2 share as
# none or some, and log2 of the request count to a whole step.  The server
# fills the tuner's memo for the whole grid before the clock starts, so no
# batch waits for a forward pass.
FEATURE_ENTROPY = tuple(float(e) for e in range(0, 9))
FEATURE_MAXLEN = (11.0, 13.0, 16.0)
FEATURE_L2 = (0.0, 0.125)


def quantize_features(f) -> np.ndarray:
    f = np.asarray(f, np.float64)
    size = np.round(f[0] * 8) / 8
    ent = float(np.clip(np.round(f[1]), 0, 8))
    maxlen = 11.0 if f[2] <= 11 else (13.0 if f[2] <= 13 else 16.0)
    l2 = 0.0 if f[3] < 0.0625 else 0.125
    count = float(np.clip(np.round(f[4]), 0, 16)) if f.size > 4 else 0.0
    return np.array([size, ent, maxlen, l2, count], np.float32)


def precompute_grid(tuner, sizes, max_batch: int) -> None:
    """Fills the tuner's memo for every batch a run over requests of `sizes`
    can form, before the clock starts: all batch sizes from the smallest
    request to the largest `max_batch` requests together, over the grid of
    `quantize_features` (byte statistics and log2 of the request count)."""
    if not len(sizes):
        return
    lo = np.log2(max(1, min(sizes)))
    hi = np.log2(max(1, sum(sorted(sizes)[-max_batch:])))
    for e in FEATURE_ENTROPY:
        for m in FEATURE_MAXLEN:
            for l2 in FEATURE_L2:
                for k in range(int(np.round(np.log2(max_batch))) + 1):
                    tuner.precompute(np.array([e, m, l2], np.float32), lo, hi, float(k))


ALLOC_GRAIN = 512  # the caching allocator rounds every block up to a multiple of this
# ...and a block of 1 MiB or more may keep an unsplit remainder of up to 1 MiB
# (the allocator splits a large block only when more than 1 MiB would be left)
ALLOC_SLACK = ALLOC_GRAIN + (1 << 20)


def _allocated(device: torch.device) -> int:
    """Bytes the caching allocator has handed out on `device` -- the figure
    torch.cuda.memory_allocated reports, read from the allocator's nested
    statistics directly (memory_allocated flattens the whole statistics tree
    first: ~0.2 ms a call, most of a small batch's host time)."""
    idx = device.index if device.index is not None else torch.cuda.current_device()
    try:
        return int(torch._C._cuda_memoryStats(idx)["allocated_bytes"]["all"]["current"])
    except (AttributeError, KeyError, TypeError):
        return int(torch.cuda.memory_allocated(device))


def _grain(n: int) -> int:
    return (int(n) + ALLOC_GRAIN - 1) // ALLOC_GRAIN * ALLOC_GRAIN


def _q(fn, sizes) -> int:
    a = np.ascontiguousarray(np.asarray(sizes, np.uint64))
    return int(fn(len(a), a.ctypes.data_as(C.POINTER(C.c_uint64))))


@dataclass
class _Batch:
    reqs: list
    stream: torch.cuda.Stream
    event: torch.cuda.Event
    reserved: int
    keep: list = field(default_factory=list)
    entries_host: torch.Tensor | None = None
    plan: BatchCodec | None = None
    dec_ws: torch.Tensor | None = None
    status_host: torch.Tensor | None = None  # the workspaces' status words, copied after the launches
    lone: tuple | None = None                # a lone compress request's (request, book, sizes, bits, gaps)
    shape: str = ""                          # its launch shape, for the per-shape statistics


class Server:
    """Continuous-batching request loop on one GPU."""

    def __init__(self, policy: str = "batched", tuner=None, config: LaunchConfig | None = None,
                 hbm_budget: float = 40e9, max_batch: int = 64, max_inflight: int = 3,
                 traffic_features=(5.0, 12.0, 0.05), device="cuda", keep_results: bool = False,
                 reserve_bytes: int = 8 << 30, tuner_min_bytes: int = 64 << 20):
        if policy not in ("batched", "plain"):
            raise ValueError("policy is 'batched' or 'plain'")
        self.policy = policy
        self.tuner = tuner
        # below this many bytes a batch's kernels are a small part of its service time (host
        # work dominates), and shapes the tuner predicts faster on the GPU measured slower in
        # service: such batches keep the tuner's default shape
        self.tuner_min_bytes = int(tuner_min_bytes)
        self.config = config or LaunchConfig()
        self.budget = float(hbm_budget)
        self.max_batch = int(max_batch)
        self.max_inflight = int(max_inflight)
        self.traffic = np.asarray(traffic_features, np.float32)
        self.device = torch.device(device)
        if self.device.index is None:  # resolved once: device lookups on every call add up
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.keep_results = keep_results
        self.current = torch.cuda.current_stream(self.device)  # where batches allocate and upload
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(self.max_inflight)]
        self.free_streams = list(self.streams)  # a new batch only goes to a stream with nothing queued
        # per stream: pinned room for its batch's two status words (compress, decompress),
        # copied there behind the launches, so retiring a batch needs no synchronization
        self.status_host = {s: torch.zeros(2, dtype=torch.int32, pin_memory=True) for s in self.streams}
        if reserve_bytes and self.policy == "batched":
            # one large cached block up front: per-batch allocations of varying size are
            # then carved from it instead of each new size reaching the driver mid-run.
            # Every batch allocates on the current stream (one pool; see _launch).
            blk = torch.empty(int(reserve_bytes), dtype=torch.uint8, device=self.device)
            del blk
        self.held = 0
        self.peak_held = 0
        self.batches = 0
        self.mem_waits = 0        # admissions stopped by the HBM budget
        self.slot_waits = 0       # loop passes with requests ready but every slot busy
        self.bound_misses = 0     # batches that allocated more than their admission bound
        self.tuner_misses = 0     # batches whose launch shape needed a forward pass of the tuner
        self.shapes = {}          # launch shape -> [batches, bytes, summed service seconds]
        # a batch's fixed part per kind: the workspace header, and the allocator's
        # rounding of each of its shared tensors (8 for compress, 3 for decompress)
        L = lib()
        cfg = LaunchConfig(region_chunks=1).cstruct()
        self._fixed = {"compress": int(L.hgap_batch_compress_workspace_bytes(0, None, C.byref(cfg)))
                       + 8 * ALLOC_SLACK,
                       "decompress": int(L.hgap_batch_decompress_workspace_bytes(0, None)) + 3 * ALLOC_SLACK}

    def reset_counters(self) -> None:
        """Zeroes the statistics (after a warm-up run)."""
        self.batches = self.peak_held = self.mem_waits = self.slot_waits = self.bound_misses = 0
        self.tuner_misses = 0
        self.shapes = {}

    # --------------------------------------------------------------- memory
    def request_bytes(self, r: Request) -> int:
        """Upper bound of the device bytes a request adds to its batch, from
        the library's own size queries: for compress, its share of the
        encoder workspace (whose region count depends on the launch shape:
        the smallest region is assumed), its worst-case bitstream and gap
        arena share (16 bits per byte), its entry and pointer slots; for
        decompress, its output (a tensor of its own, with the allocator's
        rounding), its share of the decoder workspace, its entry and pointer
        slots; plus the 256-byte alignment of every per-buffer array.  The
        batch's shared tensors add their rounding once (the fixed part)."""
        b = getattr(r, "_bytes", None)
        if b is not None:
            return b
        L = lib()
        n = [r.nbytes]
        if r.kind == "compress":
            one = LaunchConfig(region_chunks=1).cstruct()
            ws = int(L.hgap_batch_compress_workspace_bytes(1, np.asarray(n, np.uint64).ctypes.data_as(
                C.POINTER(C.c_uint64)), C.byref(one))) - int(L.hgap_batch_compress_workspace_bytes(
                    0, None, C.byref(one)))
            b = ws + 4 * (_q(L.hgap_batch_bits_capacity, n) + _q(L.hgap_batch_gaps_capacity, n))
            b += ENTRY_BYTES + 3 * 8 + 6 * 256
        else:
            ws = _q(L.hgap_batch_decompress_workspace_bytes, n) - int(L.hgap_batch_decompress_workspace_bytes(0, None))
            b = max(r.nbytes, 1) + ALLOC_SLACK + ws + ENTRY_BYTES + 8 + 6 * 256
        r._bytes = int(b)
        return r._bytes

    def _features(self, reqs) -> np.ndarray:
        """The batch's own features: log2 of its bytes and the byte-weighted
        statistics of its requests (a decompress request's from its entry, a
        compress request's from the traffic compressed so far)."""
        total = max(1, sum(r.nbytes for r in reqs))
        acc = np.zeros(3, np.float64)
        for r in reqs:
            acc += r.nbytes * (r.stream.features if r.kind == "decompress" else self.traffic)
        return quantize_features(np.concatenate([[np.log2(total)], acc / total, [np.log2(len(reqs))]]))

    def _config_for(self, reqs) -> LaunchConfig:
        if self.tuner is None:
            return self.config
        if sum(r.nbytes for r in reqs) < self.tuner_min_bytes:
            return getattr(self.tuner, "default", self.config)
        f = self._features(reqs)
        memo = getattr(self.tuner, "_memo", None)
        if memo is not None and tuple((np.round(f * 8) / 8).astype(np.float32).tolist()) not in memo:
            self.tuner_misses += 1  # a forward pass inside the loop
        return self.tuner.choose(f)

    # -------------------------------------------------------------- batches
    def _launch(self, reqs, t0) -> _Batch:
        s = self.free_streams.pop()
        self.batches += 1
        now = time.perf_counter() - t0
        for r in reqs:
            r.start = now
        bound = self._bound(reqs)
        before = _allocated(self.device)
        b = _Batch(reqs, s, torch.cuda.Event(), 0)
        cfg = self._config_for(reqs)
        b.shape = (f"r{cfg.region_chunks}/h{cfg.hist_ctas_per_sm}/e{cfg.enc_ctas_per_sm}"
                   f"/d{cfg.dec_ctas_per_sm}/t{cfg.dec_tile_segs}")
        comp = [r for r in reqs if r.kind == "compress"]
        dec = [r for r in reqs if r.kind == "decompress"]
        # Allocations and uploads on the current stream: the caching allocator keeps one
        # pool per stream, and a batch's blocks taken from one shared pool (freed only
        # after the batch's event has fired) never send a new size to the driver mid-run
        # just because the batch landed on another stream than the last one of that size.
        plan = ent = lone = None
        if len(comp) == 1 and not dec and comp[0].nbytes > 0:
            # one compress request alone: the single-buffer path (its histogram pass on the
            # batch's stream, the codebook on the host from the 1 KiB histogram, the encoder)
            # costs less host work than a batch plan and five launches
            lone = self._lone_prepare(comp[0], s)
        elif comp:
            plan = BatchCodec([r.data.numel() for r in comp], cfg, device=self.device, decompress=False,
                              inputs=[r.data for r in comp])
            ent = torch.empty(plan.entries.numel(), dtype=torch.uint8, pin_memory=True)
        # one decompress request alone: the single-buffer decoder (one call: its table
        # from the payload's codebook, a workspace memset, one kernel) is a far shorter
        # launch sequence than a batch's table, setup and class kernels
        single = len(dec) == 1 and not comp and dec[0].nbytes > 0
        dprep = None
        if single:
            dprep = self._single_prepare(dec[0])
        elif dec:
            dprep = self._decompress_prepare(dec)
        # the batch is charged what it really holds on the device
        b.reserved = _allocated(self.device) - before
        if b.reserved > bound:
            self.bound_misses += 1
        s.wait_stream(self.current)
        b.status_host = self.status_host[s]
        b.status_host.zero_()
        with torch.cuda.stream(s):
            if lone is not None:
                self._lone_launch(comp[0], lone, s, b)
                b.status_host[0:1].copy_(lone[0].workspace.view(torch.int32)[0:1], non_blocking=True)
            elif comp:
                plan.compress(stream=s)
                ent.copy_(plan.entries, non_blocking=True)
                b.status_host[0:1].copy_(plan.enc_ws.view(torch.int32)[0:1], non_blocking=True)
                b.plan, b.entries_host = plan, ent
                b.keep.append((comp, plan, ent))
            if single:
                self._single_launch(dec[0], dprep, s, b)
                b.status_host[1:2].copy_(b.dec_ws.view(torch.int32)[0:1], non_blocking=True)
            elif dec:
                self._decompress_launch(dec, dprep, cfg, s, b)
                b.status_host[1:2].copy_(b.dec_ws.view(torch.int32)[0:1], non_blocking=True)
        b.event.record(s)
        return b

    def _bound(self, reqs) -> int:
        kinds = {r.kind for r in reqs}
        return sum(self.request_bytes(r) for r in reqs) + sum(self._fixed[k] for k in kinds)

    def _lone_prepare(self, r, s):
        """The encoder's histogram pass for one request on stream s, its codebook
        on the host, and the stream's buffers (allocated on the current stream)."""
        enc = codec.Encoder(r.nbytes, self.device)
        hist = torch.empty(256, dtype=torch.int32, device=self.device)
        s.wait_stream(self.current)
        enc.histogram(r.data, out=hist, stream=s)
        hist_host = torch.empty(256, dtype=torch.int32, pin_memory=True)
        with torch.cuda.stream(s):
            hist_host.copy_(hist, non_blocking=True)
        s.synchronize()
        book, sizes = codec.Codebook.from_histogram(hist_host)
        bits = torch.empty(max(sizes.words, 1), dtype=torch.int32, device=self.device)
        gaps = torch.empty(max(sizes.gap_words, 1), dtype=torch.int32, device=self.device)
        return enc, hist, book, sizes, bits, gaps

    def _lone_launch(self, r, prep, s, b) -> None:
        enc, hist, book, sizes, bits, gaps = prep
        enc.encode(r.data, book, sizes, bits=bits, gaps=gaps, stream=s, check_status=False, prepared=True)
        b.lone = (r, book, sizes, bits[:sizes.words], gaps[:sizes.gap_words])
        b.keep.append(prep)

    def _single_prepare(self, r):
        """Output and workspace of one request decoded by the single-buffer path."""
        out = torch.empty(r.nbytes, dtype=torch.uint8, device=self.device)
        nbytes = lib().hgap_decode_workspace_bytes(int(r.stream.entry.segments))
        ws = torch.empty((nbytes + 7) // 8, dtype=torch.int64, device=self.device)
        r.stream.book  # built before the launch, on the host
        return out, ws

    def _single_launch(self, r, prep, s, b) -> None:
        out, ws = prep
        e = r.stream.entry
        check(lib().hgap_decode(r.stream.bits.data_ptr(), int(e.words), r.stream.gaps.data_ptr(), int(e.segments),
                                C.byref(r.stream.book.cstruct), out.data_ptr(), r.nbytes, ws.data_ptr(),
                                ws.numel() * 8, _stream(s)), "hgap_decode")
        r.result = out
        b.keep.append((r, out, ws))
        b.dec_ws = ws

    def _decompress_prepare(self, reqs):
        """One batched decompress over streams that live anywhere in device
        memory: each entry's offsets are rebased on the lowest address.  The
        outputs, tables and workspace, allocated and uploaded on the current stream."""
        count = len(reqs)
        outs = [torch.empty(max(r.nbytes, 1), dtype=torch.uint8, device=self.device) for r in reqs]
        base_b = min(r.stream.bits.data_ptr() for r in reqs) & ~15
        base_g = min(r.stream.gaps.data_ptr() for r in reqs) & ~3
        arr = (BatchEntry * count)()
        for i, r in enumerate(reqs):
            C.memmove(C.byref(arr[i]), C.byref(r.stream.entry), ENTRY_BYTES)
            arr[i].bits_offset = (r.stream.bits.data_ptr() - base_b) // 4
            arr[i].gaps_offset = (r.stream.gaps.data_ptr() - base_g) // 4
        # the entries (576 bytes each) and the output pointers after them, in one upload
        host = np.empty(count * ENTRY_BYTES + 8 * count, np.uint8)
        host[:count * ENTRY_BYTES] = np.frombuffer(bytes(arr), np.uint8)
        host[count * ENTRY_BYTES:].view(np.int64)[:] = [o.data_ptr() for o in outs]
        meta = _upload(host, torch.uint8, device=self.device)
        d_ent, d_out = meta[:count * ENTRY_BYTES], meta[count * ENTRY_BYTES:]
        sizes = np.array([r.nbytes for r in reqs], np.uint64)
        nbytes = lib().hgap_batch_decompress_workspace_bytes(count, sizes.ctypes.data_as(C.POINTER(C.c_uint64)))
        ws = torch.empty((nbytes + 7) // 8, dtype=torch.int64, device=self.device)
        mask = 0
        for r in reqs:
            mask |= r.stream.class_bit
        return outs, base_b, base_g, d_ent, d_out, ws, mask

    def _decompress_launch(self, reqs, prep, cfg, s, b) -> None:
        outs, base_b, base_g, d_ent, d_out, ws, mask = prep
        c = cfg.cstruct()
        c.dec_class_mask = mask  # the requests' books are known here: empty classes cost no launch
        check(lib().hgap_batch_decompress(len(reqs), d_ent.data_ptr(), base_b, base_g, d_out.data_ptr(),
                                          ws.data_ptr(), ws.numel() * 8, C.byref(c), _stream(s)),
              "hgap_batch_decompress")
        for r, o in zip(reqs, outs):
            r.result = o[:r.nbytes]
        b.keep.append((reqs, d_ent, d_out, ws, outs))
        b.dec_ws = ws

    def _retire(self, b: _Batch, now: float) -> None:
        # device status of the batch's launches, copied to pinned memory before its event
        words = b.status_host.tolist()
        if b.plan is not None or b.lone is not None:
            check(lib().hgap_status_from_word(words[0] & 0xffffffff), "served compress")
        if b.dec_ws is not None:
            check(lib().hgap_status_from_word(words[1] & 0xffffffff), "served decompress")
        for r in b.reqs:
            r.done = now
        st = self.shapes.setdefault(b.shape, [0, 0, 0.0])
        st[0] += 1
        st[1] += sum(r.nbytes for r in b.reqs)
        st[2] += now - b.reqs[0].start
        self.free_streams.append(b.stream)
        if b.plan is not None:
            comp = [r for r in b.reqs if r.kind == "compress"]
            raw = b.entries_host.numpy().tobytes()
            arr = (BatchEntry * len(comp)).from_buffer_copy(raw[:ENTRY_BYTES * len(comp)])
            for i, r in enumerate(comp):
                e = arr[i]
                bits = b.plan.bits[e.bits_offset:e.bits_offset + e.words]
                gaps = b.plan.gaps[e.gaps_offset:e.gaps_offset + e.gap_words]
                r.result = EncodedStream(e, bits, gaps, b.plan) if self.keep_results else int(e.words)
                # the traffic's byte statistics, for the next batches' features
                w = min(1.0, r.nbytes / (64 << 20))
                self.traffic = ((1 - 0.5 * w) * self.traffic + 0.5 * w * entry_features(e)).astype(np.float32)
        if b.lone is not None:
            r, book, sizes, bits, gaps = b.lone
            r.result = codec.Compressed(book, r.nbytes, sizes, bits, gaps) if self.keep_results else int(sizes.words)
            lens = book.lengths.astype(np.float64)
            f = np.array([sizes.bits / r.nbytes, lens.max(), float(np.exp2(-lens[lens > 11]).sum())], np.float32)
            w = min(1.0, r.nbytes / (64 << 20))
            self.traffic = ((1 - 0.5 * w) * self.traffic + 0.5 * w * f).astype(np.float32)
        if not self.keep_results:
            for r in b.reqs:
                if r.kind == "decompress":
                    r.result = None  # the output is released with the batch
        self.held -= b.reserved

    # ---------------------------------------------------------------- loop
    def run(self, requests) -> dict:
        """Serves `requests` (sorted by arrival) in real time; returns the
        latency and throughput statistics."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        if self.policy != "plain" and self.tuner is not None and hasattr(self.tuner, "precompute"):
            precompute_grid(self.tuner, [r.nbytes for r in reqs], self.max_batch)
        # the cyclic garbage collector stays off while the clock runs: a full pass over
        # the run's objects stalled a launch for ~100 ms and every request queued behind it
        gc_on = gc.isenabled()
        gc.collect()
        gc.disable()
        try:
            return self._run_plain(reqs) if self.policy == "plain" else self._loop(reqs)
        finally:
            if gc_on:
                gc.enable()

    def _loop(self, reqs) -> dict:
        pending = deque(reqs)
        queue = deque()
        inflight = []
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        while pending or queue or inflight:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            for b in list(inflight):
                if b.event.query():
                    inflight.remove(b)
                    self._retire(b, time.perf_counter() - t0)
            if queue and len(inflight) >= self.max_inflight:
                self.slot_waits += 1
            if queue and len(inflight) < self.max_inflight:
                take, kinds, mem = [], set(), 0
                while queue and len(take) < self.max_batch:
                    r = queue[0]
                    f = self.request_bytes(r) + (0 if r.kind in kinds else self._fixed[r.kind])
                    if self.held + mem + f > self.budget and (take or inflight):
                        self.mem_waits += 1
                        break  # wait for memory to free up
                    take.append(queue.popleft())
                    kinds.add(r.kind)
                    mem += f
                if take:
                    b = self._launch(take, t0)
                    self.held += b.reserved
                    self.peak_held = max(self.peak_held, self.held)
                    inflight.append(b)
                    continue
            if not queue and not inflight and pending:
                time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 1e-3)))
        t_end = time.perf_counter() - t0
        return self._stats(reqs, t_end)

    def _run_plain(self, reqs) -> dict:
        """Each request alone through the single-buffer path, in arrival order."""
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        for r in reqs:
            now = time.perf_counter() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
            r.start = time.perf_counter() - t0
            if r.kind == "compress":
                c = codec.compress(r.data)
                r.result = c if self.keep_results else int(c.sizes.words)
            else:
                y = codec.decompress(r.stream.to_compressed())
                r.result = y if self.keep_results else None  # the output is released at once
            torch.cuda.synchronize(self.device)
            r.done = time.perf_counter() - t0
        return self._stats(reqs, time.perf_counter() - t0)

    def _stats(self, reqs, t_end) -> dict:
        lat = np.array([r.done - r.arrival for r in reqs]) * 1e3
        svc = np.array([r.done - r.start for r in reqs]) * 1e3
        total = sum(r.nbytes for r in reqs)
        return {"requests": len(reqs), "bytes": total, "seconds": round(t_end, 4),
                "sustained_gbs": round(total / t_end / 1e9, 3),
                "p50_ms": round(float(np.percentile(lat, 50)), 3),
                "p99_ms": round(float(np.percentile(lat, 99)), 3),
                "mean_ms": round(float(lat.mean()), 3),
                "service_p50_ms": round(float(np.percentile(svc, 50)), 3),
                "service_p99_ms": round(float(np.percentile(svc, 99)), 3), "batches": self.batches,
                "peak_hbm_gb": round(self.peak_held / 1e9, 3), "budget_gb": round(self.budget / 1e9, 3),
                "mem_waits": self.mem_waits, "slot_waits": self.slot_waits,
                "bound_misses": self.bound_misses, "tuner_misses": self.tuner_misses,
                "shapes": self._shape_stats()}

    def _shape_stats(self) -> dict:
        """The launch shapes the batches took (region chunks / histogram,
        encoder, decoder CTAs per SM / decoder tile), most used first: batches,
        mean MB per batch, mean service ms."""
        top = sorted(self.shapes.items(), key=lambda kv: -kv[1][0])[:8]
        return {k: [v[0], round(v[1] / v[0] / 1e6, 2), round(1e3 * v[2] / v[0], 3)] for k, v in top}


def poisson_requests(count: int, rate_gbs: float, pool: torch.Tensor, streams: list, seed: int = 5,
                     lo: int = 64 << 10, hi: int = 64 << 20, decompress_frac: float = 0.5) -> list:
    """`count` requests with log-uniform sizes in [lo, hi], Poisson arrivals at
    `rate_gbs` of offered load; compress requests are slices of `pool`,
    decompress requests pick one of the pre-encoded `streams`."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    mean = float(sizes.mean())
    lam = rate_gbs * 1e9 / mean
    t = np.cumsum(rng.exponential(1.0 / lam, count))
    out = []
    for i in range(count):
        if streams and rng.random() < decompress_frac:
            s = streams[int(rng.integers(len(streams)))]
            out.append(Request(i, float(t[i]), "decompress", stream=s))
        else:
            n = int(min(sizes[i], pool.numel()))
            off = int(rng.integers(0, pool.numel() - n + 1))
            out.append(Request(i, float(t[i]), "compress", data=pool[off:off + n]))
    return out


def encode_streams(buffers, config: LaunchConfig | None = None) -> list:
    """Pre-encodes buffers with the batched path (the decompress payloads)."""
    plan = BatchCodec([b.numel() for b in buffers], config)
    plan.bind(buffers)
    plan.compress()
    plan.check_compress()
    ents = plan.entries_host()
    return [EncodedStream(e, plan.bits[e.bits_offset:e.bits_offset + e.words],
                          plan.gaps[e.gaps_offset:e.gaps_offset + e.gap_words], plan) for e in ents]


__all__ = ["Server", "Request", "EncodedStream", "poisson_requests", "encode_streams", "quantize_features",
           "precompute_grid"]
