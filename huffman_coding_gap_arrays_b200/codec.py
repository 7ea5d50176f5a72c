"""Host-side API over libhgap.so, mirroring the reference's entry points.

The reference path (daisuke-takafuji/Huffman_coding_Gap_arrays) is
``histgram`` -> ``store_symbols``/``qsort``/``boundary_PM`` -> ``encode`` on
the encoder side (encoder/src/huff.cpp:60-99) and ``get_table_info``/
``get_twolevel_table`` -> ``decoder_l1_l2`` on the decoder side
(decoder/src/huff.cpp:154-207).  Here:

    hist = histogram(x)                      # histgram, device -> device
    book, sizes = Codebook.from_histogram(hist.cpu())   # boundary_PM, host
    bits, gaps = Encoder(x.numel()).encode(x, book, sizes)   # encode
    y = Decoder(sizes.segments).decode(bits, gaps, sizes, book, n)   # decoder_l1_l2

``compress``/``decompress`` chain those, and ``Compressed.to_container`` /
``from_container`` read and write the reference's file format
(encoder/src/huff.cpp:111-125, decoder/src/huff.cpp:27-81).

Device memory and streams come from torch (u32 words are held in int32
tensors); every computation is a libhgap.so call -- there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import CCodebook, HgapError, Sizes, SymLen, check, lib


def _stream(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


def _require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


@dataclass
class StreamSizes:
    """B, W, S and the gap-word count of one encoded stream (huff.cpp:84-88)."""
    bits: int
    words: int
    segments: int
    gap_words: int

    @classmethod
    def from_bits(cls, bits: int) -> "StreamSizes":
        z = lib().hgap_sizes_from_bits(int(bits))
        return cls(z.bits, z.words, z.segments, z.gap_words)

    @classmethod
    def from_words(cls, words: int) -> "StreamSizes":
        seg = (words + 3) // 4
        return cls(words * 32, words, seg, (seg + 7) // 8)


class Codebook:
    """Canonical length-limited codebook (reference struct Symbol list +
    struct Codetable, encoder/include/constants.hpp:34-43)."""

    def __init__(self, c: CCodebook):
        self._c = c

    @classmethod
    def from_histogram(cls, hist) -> tuple["Codebook", StreamSizes]:
        h = np.ascontiguousarray(_to_numpy_u32(hist))
        if h.size != 256:
            raise ValueError("histogram must have 256 bins")
        c = CCodebook()
        z = Sizes()
        check(lib().hgap_codebook_build(h.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(c),
                                        C.byref(z)), "hgap_codebook_build")
        return cls(c), StreamSizes(z.bits, z.words, z.segments, z.gap_words)

    @classmethod
    def from_symbols(cls, symbols, lengths) -> "Codebook":
        symbols = np.asarray(symbols, np.uint8)
        lengths = np.asarray(lengths, np.uint8)
        arr = (SymLen * max(1, symbols.size))()
        for i, (s, l) in enumerate(zip(symbols.tolist(), lengths.tolist())):
            arr[i].symbol, arr[i].length = s, l
        c = CCodebook()
        check(lib().hgap_codebook_from_symbols(arr, symbols.size, C.byref(c)),
              "hgap_codebook_from_symbols")
        return cls(c)

    @property
    def symbol_count(self) -> int:
        return int(self._c.symbol_count)

    @property
    def symbols(self) -> np.ndarray:
        return np.array([self._c.symbols[i].symbol for i in range(self.symbol_count)], np.uint8)

    @property
    def lengths(self) -> np.ndarray:
        return np.array([self._c.symbols[i].length for i in range(self.symbol_count)], np.uint8)

    @property
    def code(self) -> np.ndarray:
        return np.array([self._c.table[b].code for b in range(256)], np.uint32)

    @property
    def length(self) -> np.ndarray:
        return np.array([self._c.table[b].length for b in range(256)], np.uint32)

    def encoded_bits(self, hist) -> int:
        h = np.ascontiguousarray(_to_numpy_u32(hist))
        return int(lib().hgap_encoded_bits(C.byref(self._c), h.ctypes.data_as(C.POINTER(C.c_uint32))))

    @property
    def cstruct(self) -> CCodebook:
        return self._c


def _to_numpy_u32(h) -> np.ndarray:
    if isinstance(h, torch.Tensor):
        h = h.detach().cpu().numpy()
    return np.asarray(h).astype(np.uint32, copy=False).view(np.uint32)


def histogram(x: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """256-bin byte histogram on the device (replaces histgram,
    encoder/src/encoder.cu:118-140).  Returns an int32 tensor of u32 counts."""
    _require_cuda(x, "x")
    if out is None:
        out = torch.empty(256, dtype=torch.int32, device=x.device)
    check(lib().hgap_histogram(x.data_ptr(), x.numel() * x.element_size(), out.data_ptr(),
                               _stream(stream)), "hgap_histogram")
    return out


class Encoder:
    """Holds the encoder workspace for inputs of up to ``capacity`` bytes
    (replaces encode, encoder/src/encoder.cu:381-457, without its per-call
    allocations)."""

    def __init__(self, capacity: int, device=None):
        self.capacity = int(capacity)
        dev = torch.device(device) if device is not None else torch.device("cuda")
        nbytes = lib().hgap_encode_workspace_bytes(max(self.capacity, 1))
        self.workspace = torch.empty((nbytes + 7) // 8, dtype=torch.int64, device=dev)

    def histogram(self, x: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """The encoder's histogram pass (hgap_encode_histogram): the global
        histogram, plus per-super-tile histograms kept in this workspace for a
        following ``encode(..., prepared=True)`` of the same tensor."""
        _require_cuda(x, "x")
        n = x.numel() * x.element_size()
        if n > self.capacity:
            raise ValueError(f"input of {n} bytes exceeds encoder capacity {self.capacity}")
        if out is None:
            out = torch.empty(256, dtype=torch.int32, device=x.device)
        ws = self.workspace
        check(lib().hgap_encode_histogram(x.data_ptr(), n, out.data_ptr(), ws.data_ptr(), ws.numel() * 8,
                                          _stream(stream)), "hgap_encode_histogram")
        return out

    def encode(self, x: torch.Tensor, book: Codebook, sizes: StreamSizes, bits: torch.Tensor | None = None,
               gaps: torch.Tensor | None = None, stream=None, check_status: bool = True,
               prepared: bool = False):
        """Encode x.  With prepared=True the per-super-tile histograms from the
        last ``histogram(x)`` on this encoder are reused (one pass over x);
        otherwise the encoder makes them itself (two passes)."""
        _require_cuda(x, "x")
        n = x.numel() * x.element_size()
        if n > self.capacity:
            raise ValueError(f"input of {n} bytes exceeds encoder capacity {self.capacity}")
        if bits is None:
            bits = torch.empty(max(sizes.words, 1), dtype=torch.int32, device=x.device)
        if gaps is None:
            gaps = torch.empty(max(sizes.gap_words, 1), dtype=torch.int32, device=x.device)
        ws = self.workspace
        fn = lib().hgap_encode_prepared if prepared else lib().hgap_encode
        check(fn(x.data_ptr(), n, C.byref(book.cstruct), bits.data_ptr(), sizes.words,
                 gaps.data_ptr(), sizes.segments, ws.data_ptr(), ws.numel() * 8, _stream(stream)),
              "hgap_encode")
        if check_status:
            self.check(stream)
        return bits[:sizes.words], gaps[:sizes.gap_words]

    def encode_part(self, x: torch.Tensor, book: Codebook, bit0: int, part_bits: int, stream=None,
                    check_status: bool = True):
        """One part of a stream split across devices (hgap_encode_part_prepared),
        after ``histogram(x)`` on this encoder: x's codes placed from stream bit
        ``bit0``.  Returns (first stream word, its words, first gap word, its
        gap words); the stream is the OR of all parts' words at those places
        (``parallel.stitch_parts``)."""
        _require_cuda(x, "x")
        n = x.numel() * x.element_size()
        if n > self.capacity:
            raise ValueError(f"input of {n} bytes exceeds encoder capacity {self.capacity}")
        bit0, part_bits = int(bit0), int(part_bits)
        end = bit0 + part_bits
        w_first, g_first = bit0 >> 5, bit0 >> 10
        w_base = w_first & ~3                        # the window starts on a 16-byte boundary
        w_end, g_end = (end + 31) // 32, ((end + 127) // 128 + 7) // 8
        bits = torch.empty(max(w_end - w_base, 1), dtype=torch.int32, device=x.device)
        gaps = torch.empty(max(g_end - g_first, 1), dtype=torch.int32, device=x.device)
        ws = self.workspace
        check(lib().hgap_encode_part_prepared(x.data_ptr(), n, C.byref(book.cstruct), bit0, part_bits,
                                              bits.data_ptr(), w_base, gaps.data_ptr(), g_first,
                                              ws.data_ptr(), ws.numel() * 8, _stream(stream)),
              "hgap_encode_part_prepared")
        if check_status and n:
            self.check(stream)
        if n == 0:
            return w_first, bits[:0], g_first, gaps[:0]
        return w_first, bits[w_first - w_base:w_end - w_base], g_first, gaps[:g_end - g_first]

    def check(self, stream=None) -> None:
        check(lib().hgap_workspace_status(self.workspace.data_ptr(), _stream(stream)), "encode (device)")


class Decoder:
    """Holds the decoder workspace for streams of up to ``segments`` gap
    entries (replaces decoder_l1_l2, decoder/src/decoder.cu:732-815)."""

    def __init__(self, segments: int, device=None):
        self.segments = int(segments)
        dev = torch.device(device) if device is not None else torch.device("cuda")
        nbytes = lib().hgap_decode_workspace_bytes(max(self.segments, 1))
        self.workspace = torch.empty((nbytes + 7) // 8, dtype=torch.int64, device=dev)

    def decode(self, bits: torch.Tensor, gaps: torch.Tensor, sizes: StreamSizes, book: Codebook, n: int,
               out: torch.Tensor | None = None, stream=None, check_status: bool = True) -> torch.Tensor:
        _require_cuda(bits, "bits")
        _require_cuda(gaps, "gaps")
        if sizes.segments > self.segments:
            raise ValueError("stream has more segments than the decoder workspace")
        if out is None:
            out = torch.empty(max(n, 1), dtype=torch.uint8, device=bits.device)
        ws = self.workspace
        check(lib().hgap_decode(bits.data_ptr(), sizes.words, gaps.data_ptr(), sizes.segments,
                                C.byref(book.cstruct), out.data_ptr(), n, ws.data_ptr(),
                                ws.numel() * 8, _stream(stream)), "hgap_decode")
        if check_status:
            self.check(stream)
        return out[:n]

    def check(self, stream=None) -> None:
        check(lib().hgap_workspace_status(self.workspace.data_ptr(), _stream(stream)), "decode (device)")


@dataclass
class Compressed:
    """One encoded buffer: codebook, original length, bitstream and gap array."""
    book: Codebook
    n: int
    sizes: StreamSizes
    bits: torch.Tensor  # int32 view of u32 words (device or host)
    gaps: torch.Tensor

    def to_container(self) -> bytes:
        """Reference container bytes (encoder/src/huff.cpp:111-125)."""
        bits = np.ascontiguousarray(self.bits.cpu().numpy().view(np.uint32))
        gaps = np.ascontiguousarray(self.gaps.cpu().numpy().view(np.uint32))
        size = lib().hgap_container_bytes(self.book.symbol_count, self.sizes.words, self.sizes.segments)
        buf = np.zeros(max(size, 1), np.uint8)
        written = C.c_size_t(0)
        check(lib().hgap_container_write(buf.ctypes.data, size, C.byref(self.book.cstruct), self.n,
                                         self.sizes.words, self.sizes.segments, gaps.ctypes.data,
                                         bits.ctypes.data, C.byref(written)), "hgap_container_write")
        return buf[:written.value].tobytes()

    @classmethod
    def from_container(cls, data: bytes, device=None) -> "Compressed":
        """Parses reference container bytes (decoder/src/huff.cpp:27-81)."""
        raw = np.frombuffer(data, np.uint8)
        c = CCodebook()
        n, W, S = C.c_uint64(), C.c_uint64(), C.c_uint64()
        gp, bp = C.c_void_p(), C.c_void_p()
        check(lib().hgap_container_parse(raw.ctypes.data, raw.size, C.byref(c), C.byref(n), C.byref(W),
                                         C.byref(S), C.byref(gp), C.byref(bp)), "hgap_container_parse")
        base = raw.ctypes.data
        sizes = StreamSizes.from_words(W.value)
        g0 = (gp.value or base) - base
        b0 = (bp.value or base) - base
        gaps = np.frombuffer(raw[g0:g0 + 4 * sizes.gap_words].tobytes(), np.uint32)
        bits = np.frombuffer(raw[b0:b0 + 4 * sizes.words].tobytes(), np.uint32)
        dev = torch.device(device) if device is not None else torch.device("cuda")
        return cls(Codebook(c), n.value, sizes,
                   torch.from_numpy(bits.view(np.int32).copy()).to(dev),
                   torch.from_numpy(gaps.view(np.int32).copy()).to(dev))


def compress(x: torch.Tensor, stream=None) -> Compressed:
    """histogram -> codebook -> encode, as encoder/src/huff.cpp:60-99 does."""
    _require_cuda(x, "x")
    x = x.reshape(-1).view(torch.uint8) if x.dtype != torch.uint8 else x.reshape(-1)
    n = x.numel()
    if n == 0:
        book, sizes = Codebook.from_histogram(np.zeros(256, np.uint32))
        empty = torch.empty(0, dtype=torch.int32, device=x.device)
        return Compressed(book, 0, sizes, empty, empty)
    enc = Encoder(n, x.device)
    hist = enc.histogram(x, stream=stream)
    book, sizes = Codebook.from_histogram(hist.cpu())
    bits, gaps = enc.encode(x, book, sizes, stream=stream, prepared=True)
    return Compressed(book, n, sizes, bits, gaps)


def decompress(c: Compressed, stream=None) -> torch.Tensor:
    if c.n == 0:
        return torch.empty(0, dtype=torch.uint8, device=c.bits.device)
    return Decoder(c.sizes.segments, c.bits.device).decode(c.bits, c.gaps, c.sizes, c.book, c.n,
                                                           stream=stream)


__all__ = ["Codebook", "StreamSizes", "Encoder", "Decoder", "Compressed", "histogram", "compress",
           "decompress", "HgapError"]
