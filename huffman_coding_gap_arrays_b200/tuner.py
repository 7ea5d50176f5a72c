"""Launch-configuration autotuner for the batched path.

The batched kernels take a launch shape (``LaunchConfig``: encoder region
size, CTAs per SM of the histogram, encoder and decoder grids) that never
changes their output.  The autotuner times candidate shapes on the caller's
own buffers with CUDA events and keeps every measurement as a record
(buffer features, config, time), which is also the training set of the
learned tuner (``mlp.py``).

Features of a buffer (cheap, from its histogram and codebook):
  log2 of its size, its entropy in bits per byte, its longest code length and
  the fraction of its bytes whose code is longer than the decoder's 11-bit
  level-1 prefix (level-2 lookups, the decoder's slow path).  A batch has the
  same four, over all its bytes: log2 of its total size and the byte-weighted
  means of the other three; and a fifth, log2 of its buffer count (0 for one
  buffer), which tells one 64 MiB buffer from 4096 buffers of 16 KiB.
"""
from __future__ import annotations

import ctypes as C
import itertools
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from .batch import BatchCodec, LaunchConfig

REGIONS = (1, 2, 4, 8, 16, 32)
HIST_CTAS = (2, 4)
ENC_CTAS = (1, 2)
# decoder CTAs per SM; each decoder is clamped to what fits it (5 for 256-segment tiles, 4 for
# 512-segment ones, 3 for 32 stage rows), and 0 takes that maximum
DEC_CTAS = (1, 2, 3, 4, 0)
DEC_TILES = (0, 256, 512)  # decoder tile: by the book's shortest code (0), or 256 / 512 segments for all
DEC_SPACE = tuple(itertools.product(DEC_CTAS, DEC_TILES))  # (CTAs per SM, tile) pairs


def with_dec(cfg: LaunchConfig, dec) -> LaunchConfig:
    """cfg with the decoder shape `dec` = (CTAs per SM, tile segments)."""
    return LaunchConfig(cfg.region_chunks, cfg.hist_ctas_per_sm, cfg.enc_ctas_per_sm, dec[0], dec[1])


def compress_space():
    return [LaunchConfig(region_chunks=r, hist_ctas_per_sm=h, enc_ctas_per_sm=e)
            for r, h, e in itertools.product(REGIONS, HIST_CTAS, ENC_CTAS)]


def features_from_hist(n: int, hist: np.ndarray, lengths: np.ndarray) -> np.ndarray:
    """[log2 n, entropy (bits/byte), max code length, level-2 byte fraction]."""
    h = np.asarray(hist, np.float64)
    tot = h.sum()
    if tot <= 0:
        return np.array([math.log2(max(n, 1)), 0.0, 0.0, 0.0], np.float32)
    p = h[h > 0] / tot
    ent = float(-(p * np.log2(p)).sum())
    ln = np.asarray(lengths, np.float64)
    maxlen = float(ln.max()) if ln.size else 0.0
    l2 = float(h[ln > 11].sum() / tot)
    return np.array([math.log2(max(n, 1)), ent, maxlen, l2], np.float32)


def buffer_features(x: torch.Tensor) -> np.ndarray:
    """Features of one uint8 CUDA buffer (histogram on the device)."""
    from . import codec
    n = x.numel()
    if n == 0:
        return np.zeros(5, np.float32)
    hist = codec.histogram(x).cpu().numpy().view(np.uint32)
    book, _ = codec.Codebook.from_histogram(hist)
    return np.concatenate([features_from_hist(n, hist, book.length), [0.0]]).astype(np.float32)


def batch_features(inputs) -> np.ndarray:
    """Features of a batch of uint8 CUDA buffers: the histograms by this
    library's histogram kernel, the codebooks by its device builder (one warp
    per histogram), the per-buffer statistics vectorised over the batch."""
    from . import codec
    from ._lib import CCodebook, check, lib
    sizes = np.array([int(t.numel()) for t in inputs], np.int64)
    total = int(sizes.sum())
    if total == 0:
        return np.zeros(5, np.float32)
    dev = next(t.device for t in inputs if t.numel())
    hs = torch.zeros((len(inputs), 256), dtype=torch.int32, device=dev)
    for i, t in enumerate(inputs):
        if t.numel():
            codec.histogram(t, out=hs[i])
    books = torch.empty(len(inputs) * C.sizeof(CCodebook), dtype=torch.uint8, device=dev)
    bsizes = torch.empty(len(inputs) * 4, dtype=torch.int64, device=dev)
    check(lib().hgap_codebook_build_device(len(inputs), hs.data_ptr(), books.data_ptr(), bsizes.data_ptr(),
                                           codec._stream(None)), "hgap_codebook_build_device")
    h = hs.cpu().numpy().view(np.uint32).astype(np.float64)
    # per-byte code lengths: hgap_codebook.table[b].length
    off = CCodebook.table.offset
    raw = books.cpu().numpy().reshape(len(inputs), C.sizeof(CCodebook))[:, off:off + 8 * 256]
    lens = np.ascontiguousarray(raw).view(np.uint32).reshape(len(inputs), 256, 2)[:, :, 1].astype(np.float64)
    n = h.sum(axis=1)
    ok = n > 0
    p = np.where(h > 0, h / np.maximum(n, 1)[:, None], 1.0)
    ent = -(np.where(h > 0, p * np.log2(p), 0.0)).sum(axis=1)
    maxlen = np.where(h > 0, lens, 0.0).max(axis=1)
    l2 = np.where(lens > 11, h, 0.0).sum(axis=1) / np.maximum(n, 1)
    w = np.where(ok, sizes, 0).astype(np.float64)
    acc = np.array([(w * ent).sum(), (w * maxlen).sum(), (w * l2).sum()])
    return np.concatenate([[math.log2(total)], acc / total, [math.log2(len(sizes))]]).astype(np.float32)


@dataclass
class Record:
    features: np.ndarray   # of the tuned input (one buffer, or a batch)
    config: LaunchConfig
    compress_ms: float
    decompress_ms: float


@dataclass
class TuneResult:
    compress: LaunchConfig
    decompress: tuple  # (CTAs per SM, tile segments)
    compress_ms: float
    decompress_ms: float
    records: list = field(default_factory=list)

    @property
    def config(self) -> LaunchConfig:
        return with_dec(self.compress, self.decompress)


def _time(fn, reps: int, warmup: int) -> float:
    for _ in range(warmup):
        fn()
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(reps):
        fn()
    b.record(s)
    b.synchronize()
    return a.elapsed_time(b) / reps


class Autotuner:
    """Exhaustive search of the launch space on the caller's buffers."""

    def __init__(self, reps: int = 3, warmup: int = 1, space=None, dec_space=DEC_SPACE):
        self.reps = reps
        self.warmup = warmup
        self.space = list(space) if space is not None else compress_space()
        self.dec_space = tuple(dec_space)
        self.records: list[Record] = []

    def tune(self, inputs, outputs, features: np.ndarray | None = None,
             plan: BatchCodec | None = None) -> TuneResult:
        """Times every compress shape, then every decoder shape (grid and
        tile size) on the best compress output; every run is checked by the
        device status."""
        sizes = [int(t.numel()) for t in inputs]
        if plan is None:
            base = min(c.region_chunks for c in self.space)
            plan = BatchCodec(sizes, LaunchConfig(region_chunks=base))
            plan.bind(inputs, outputs)
        feats = features if features is not None else np.zeros(4, np.float32)
        best_c, best_ms = None, float("inf")
        for cfg in self.space:
            plan.config = cfg
            ms = _time(plan.compress, self.reps, self.warmup)
            plan.check_compress()
            self.records.append(Record(feats, cfg, ms, float("nan")))
            if ms < best_ms:
                best_c, best_ms = cfg, ms
        plan.config = best_c
        plan.compress()
        plan.check_compress()
        best_d, best_dms = None, float("inf")
        for d in self.dec_space:
            plan.config = with_dec(best_c, d)
            ms = _time(plan.decompress, self.reps, self.warmup)
            plan.check_decompress()
            self.records.append(Record(feats, plan.config, float("nan"), ms))
            if ms < best_dms:
                best_d, best_dms = d, ms
        plan.config = with_dec(best_c, best_d)
        return TuneResult(best_c, best_d, best_ms, best_dms, list(self.records))


__all__ = ["Autotuner", "TuneResult", "Record", "compress_space", "buffer_features", "batch_features",
           "features_from_hist", "with_dec",
           "REGIONS", "HIST_CTAS", "ENC_CTAS", "DEC_CTAS", "DEC_TILES", "DEC_SPACE"]
