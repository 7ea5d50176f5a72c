"""Batched path: thousands of buffers, each with its own codebook, in one
fixed sequence of launches (no counterpart in the reference).

    plan = BatchCodec(sizes)                      # workspaces and arenas, once
    plan.bind(inputs, outputs)                    # device pointer tables, once
    plan.compress()                               # histogram -> books -> encode
    plan.decompress()                             # books -> tables -> decode
    g = plan.capture()                            # both as one CUDA graph

Each buffer's bitstream and gap array are exactly what ``codec.compress`` makes
for it alone (same codebook, same bits); ``container(i)`` writes buffer i in
the reference's file format.  Every computation is a libhgap.so call.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import BatchConfig, BatchEntry, CCodebook, check, lib
from .codec import Codebook, Compressed, StreamSizes, _stream

ENTRY_BYTES = C.sizeof(BatchEntry)
# Kernels one batched call launches (csrc/batch.cu): compress = benc_setup, hist_st, book,
# benc_place, encode; decompress = bdec_table, bdec_setup, bdec_map and one decoder per class (8).
COMPRESS_KERNELS = 5
DECOMPRESS_KERNELS = 11


@dataclass
class LaunchConfig:
    """Launch shape of the batched kernels; no choice changes the output."""
    region_chunks: int = 8      # encoder region = region_chunks x 8 KiB (1..32)
    hist_ctas_per_sm: int = 0   # persistent grids: CTAs per SM (0 = occupancy maximum)
    enc_ctas_per_sm: int = 0
    dec_ctas_per_sm: int = 0
    dec_tile_segs: int = 0      # decoder tile: 256 or 512 segments (0 = by the book's shortest code)
    dec_class_mask: int = 0     # decoder classes to launch (0 = all 8; see decoder_class_mask)

    def cstruct(self) -> BatchConfig:
        return BatchConfig(self.region_chunks, self.hist_ctas_per_sm, self.enc_ctas_per_sm,
                           self.dec_ctas_per_sm, self.dec_tile_segs, self.dec_class_mask)


def decoder_class_mask(entries) -> int:
    """The decoder classes a batch of entries (BatchEntry, host copies) needs,
    as hgap_batch_config.dec_class_mask: an empty class then costs no launch."""
    L = lib()
    mask = 0
    for e in entries:
        if e.symbol_count:
            c = int(L.hgap_batch_decoder_class(e.symbols, e.symbol_count))
            if c < 8:
                mask |= 1 << c
    return mask


def _u64p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _upload(values, dtype, out: torch.Tensor | None = None, device=None) -> torch.Tensor:
    """Host values to the device through pinned memory, ordered on the current
    stream without blocking the host (a pageable copy would wait for the
    stream's earlier work)."""
    host = torch.tensor(np.array(values, copy=True), dtype=dtype).pin_memory()
    if out is None:
        return host.to(device, non_blocking=True)
    out.copy_(host, non_blocking=True)
    return out


class BatchCodec:
    """Workspaces, arenas and pointer tables for a fixed list of buffer sizes."""

    def __init__(self, sizes, config: LaunchConfig | None = None, device=None,
                 region_chunks: np.ndarray | None = None, decompress: bool = True, inputs=None, outputs=None):
        self.sizes = np.ascontiguousarray(np.asarray(sizes, dtype=np.uint64))
        self.count = int(self.sizes.size)
        self.config = config or LaunchConfig()
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        L = lib()
        cfg = self.config.cstruct()
        enc_ws = L.hgap_batch_compress_workspace_bytes(self.count, _u64p(self.sizes), C.byref(cfg))
        # a compress-only plan (decompress=False) holds no decompress workspace
        dec_ws = L.hgap_batch_decompress_workspace_bytes(self.count, _u64p(self.sizes)) if decompress else 8
        self.bits_capacity = int(L.hgap_batch_bits_capacity(self.count, _u64p(self.sizes)))
        self.gaps_capacity = int(L.hgap_batch_gaps_capacity(self.count, _u64p(self.sizes)))
        dev = self.device
        # one device allocation carved into the workspaces, arenas and entries (256-byte aligned)
        parts = [("enc_ws", enc_ws, torch.int64), ("dec_ws", dec_ws, torch.int64),
                 ("bits", 4 * max(self.bits_capacity, 4), torch.int32),
                 ("gaps", 4 * max(self.gaps_capacity, 1), torch.int32),
                 ("entries", max(self.count, 1) * ENTRY_BYTES, torch.uint8)]
        offs, total = [], 0
        for _, nbytes, dt in parts:
            offs.append(total)
            total += (nbytes + 255) & ~255
        self._arena = torch.empty(total, dtype=torch.uint8, device=dev)
        for (name, nbytes, dt), o in zip(parts, offs):
            whole = (nbytes + dt.itemsize - 1) // dt.itemsize * dt.itemsize
            setattr(self, name, self._arena[o:o + whole].view(dt))
        self.entries.zero_()
        # sizes, input pointers and output pointers in one device array, uploaded at once
        k = max(self.count, 1)
        meta = np.zeros(3 * k, np.int64)
        meta[:self.count] = self.sizes.view(np.int64)
        if inputs is not None:
            self._check(inputs, "inputs")
            meta[k:k + self.count] = [t.data_ptr() for t in inputs]
        if outputs is not None:
            self._check(outputs, "outputs")
            meta[2 * k:2 * k + self.count] = [t.data_ptr() for t in outputs]
        self._meta = _upload(meta, torch.int64, device=dev)
        self.d_sizes, self.d_in, self.d_out = self._meta[:k], self._meta[k:2 * k], self._meta[2 * k:]
        self.d_region = None
        if region_chunks is not None:
            rc = np.asarray(region_chunks, np.uint8)
            if rc.size != self.count:
                raise ValueError("one region size per buffer")
            self.d_region = _upload(rc, torch.uint8, device=dev)
        self._inputs = list(inputs) if inputs is not None else None
        self._outputs = list(outputs) if outputs is not None else None

    # ---------------------------------------------------------------- binding
    def bind(self, inputs=None, outputs=None) -> None:
        """Device pointer tables of the input and output buffers (lists of
        uint8 CUDA tensors, one per size).  The tensors must stay alive."""
        if inputs is not None:
            self._check(inputs, "inputs")
            _upload([t.data_ptr() for t in inputs], torch.int64, out=self.d_in)
            self._inputs = list(inputs)
        if outputs is not None:
            self._check(outputs, "outputs")
            _upload([t.data_ptr() for t in outputs], torch.int64, out=self.d_out)
            self._outputs = list(outputs)

    def _check(self, bufs, name):
        if len(bufs) != self.count:
            raise ValueError(f"{name}: {len(bufs)} buffers for {self.count} sizes")
        for t, n in zip(bufs, self.sizes.tolist()):
            if not t.is_cuda or t.dtype != torch.uint8 or not t.is_contiguous():
                raise ValueError(f"{name} must be contiguous uint8 CUDA tensors")
            if t.numel() < n:
                raise ValueError(f"{name}: a buffer is smaller than its size")

    # ------------------------------------------------------------- launches
    def compress(self, stream=None) -> None:
        if self._inputs is None:
            raise RuntimeError("bind(inputs=...) first")
        cfg = self.config.cstruct()
        check(lib().hgap_batch_compress(
            self.count, self.d_in.data_ptr(), self.d_sizes.data_ptr(),
            self.d_region.data_ptr() if self.d_region is not None else None,
            self.bits.data_ptr(), self.bits_capacity, self.gaps.data_ptr(), self.gaps_capacity,
            self.entries.data_ptr(), self.enc_ws.data_ptr(), self.enc_ws.numel() * 8, C.byref(cfg),
            _stream(stream)), "hgap_batch_compress")

    def decompress(self, stream=None) -> None:
        if self._outputs is None:
            raise RuntimeError("bind(outputs=...) first")
        cfg = self.config.cstruct()
        check(lib().hgap_batch_decompress(
            self.count, self.entries.data_ptr(), self.bits.data_ptr(), self.gaps.data_ptr(),
            self.d_out.data_ptr(), self.dec_ws.data_ptr(), self.dec_ws.numel() * 8, C.byref(cfg),
            _stream(stream)), "hgap_batch_decompress")

    def check(self, stream=None) -> None:
        check(lib().hgap_batch_status(self.enc_ws.data_ptr(), _stream(stream)), "batch compress (device)")
        check(lib().hgap_batch_status(self.dec_ws.data_ptr(), _stream(stream)), "batch decompress (device)")

    def check_compress(self, stream=None) -> None:
        check(lib().hgap_batch_status(self.enc_ws.data_ptr(), _stream(stream)), "batch compress (device)")

    def check_decompress(self, stream=None) -> None:
        check(lib().hgap_batch_status(self.dec_ws.data_ptr(), _stream(stream)), "batch decompress (device)")

    def capture(self, compress: bool = True, decompress: bool = True) -> torch.cuda.CUDAGraph:
        """The launch sequence as one CUDA graph (run it once eagerly first:
        the first call sets kernel attributes, which is not a stream operation)."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                if compress:
                    self.compress(stream=s)
                if decompress:
                    self.decompress(stream=s)
        torch.cuda.current_stream(self.device).wait_stream(s)
        return g

    # ---------------------------------------------------------------- results
    def entries_host(self) -> list:
        raw = self.entries.cpu().numpy()
        arr = (BatchEntry * max(self.count, 1)).from_buffer_copy(raw.tobytes())
        return [arr[i] for i in range(self.count)]

    def book(self, e) -> Codebook:
        syms = np.array([e.symbols[k].symbol for k in range(e.symbol_count)], np.uint8)
        lens = np.array([e.symbols[k].length for k in range(e.symbol_count)], np.uint8)
        if e.symbol_count == 0:
            return Codebook(CCodebook())
        return Codebook.from_symbols(syms, lens)

    def stream(self, i: int, e=None) -> Compressed:
        """Buffer i's encoded stream (views into the arenas)."""
        e = e if e is not None else self.entries_host()[i]
        sizes = StreamSizes(int(e.bits), int(e.words), int(e.segments), int(e.gap_words))
        bits = self.bits[e.bits_offset:e.bits_offset + e.words]
        gaps = self.gaps[e.gaps_offset:e.gaps_offset + e.gap_words]
        return Compressed(self.book(e), int(e.n), sizes, bits, gaps)

    def container(self, i: int, e=None) -> bytes:
        """Buffer i in the reference's container format."""
        return self.stream(i, e).to_container()


def device_codebooks(hists: torch.Tensor, stream=None):
    """Codebooks built on the device, one warp per histogram (count x 256
    int32 counts on the GPU).  Returns (list of Codebook, list of StreamSizes)."""
    if not hists.is_cuda or hists.dim() != 2 or hists.shape[1] != 256:
        raise ValueError("hists must be a CUDA tensor of shape (count, 256)")
    hists = hists.contiguous()
    count = hists.shape[0]
    books = torch.empty(count * C.sizeof(CCodebook), dtype=torch.uint8, device=hists.device)
    sizes = torch.empty(count * 4, dtype=torch.int64, device=hists.device)
    check(lib().hgap_codebook_build_device(count, hists.data_ptr(), books.data_ptr(), sizes.data_ptr(),
                                           _stream(stream)), "hgap_codebook_build_device")
    raw = books.cpu().numpy().tobytes()
    z = sizes.cpu().numpy().reshape(-1, 4)
    out_b, out_s = [], []
    for i in range(count):
        c = CCodebook.from_buffer_copy(raw[i * C.sizeof(CCodebook):(i + 1) * C.sizeof(CCodebook)])
        out_b.append(Codebook(c))
        out_s.append(StreamSizes(*[int(v) for v in z[i]]))
    return out_b, out_s


def device_decode_tables(books: list, device="cuda", stream=None):
    """Decoder tables built on the device from codebooks; returns
    (tables int16 tensor (count, 2048 + 2560) on the host, per-book status)."""
    count = len(books)
    raw = b"".join(bytes(b.cstruct) for b in books)
    d_books = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(device)
    t = torch.empty(count * (2048 + 2560), dtype=torch.int16, device=device)
    st = torch.zeros(count, dtype=torch.int32, device=device)
    check(lib().hgap_decode_table_build_device(count, d_books.data_ptr(), t.data_ptr(), st.data_ptr(),
                                               _stream(stream)), "hgap_decode_table_build_device")
    return t.view(count, -1).cpu(), st.cpu()


def host_decode_table(book: Codebook) -> np.ndarray:
    t1 = np.zeros(2048, np.uint16)
    t2 = np.zeros(2560, np.uint16)
    check(lib().hgap_decode_table_build(C.byref(book.cstruct), t1.ctypes.data, t2.ctypes.data),
          "hgap_decode_table_build")
    return np.concatenate([t1, t2])


__all__ = ["BatchCodec", "LaunchConfig", "device_codebooks", "device_decode_tables", "host_decode_table"]
