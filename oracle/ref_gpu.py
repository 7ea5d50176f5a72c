"""The reference's own GPU kernels, timed kernel by kernel on the device.

MEASUREMENT AND TEST INFRASTRUCTURE ONLY: ctypes bindings of
oracle/_ref/libref_gpu_time.so, which oracle/Makefile builds from the
reference's unmodified encoder/src/encoder.cu and decoder/src/decoder.cu
(sm_100a) with two small launch-and-time shims (ref_gpu_enc_time.cu,
ref_gpu_dec_time.cu).  This is the "plain reference on B200" of the
measurement plan: cu_histgram + mergeHistogram (encoder/src/encoder.cu:33-140),
cuencoder + cu_get_gaparray (:142-379, with the memsets encode() issues,
:381-457) and gpu_dec_l1_l2 (decoder/src/decoder.cu:454-730, with the memsets
decoder_l1_l2() issues, :732-815).  Only `bench.py --impl reference` and the
tests use it; the library never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_gpu_time.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        vp, u32, i32, f32p = C.c_void_p, C.c_uint32, C.c_int, C.POINTER(C.c_float)
        u8p, u32p = C.POINTER(C.c_uint8), C.POINTER(C.c_uint32)
        L.hgapref_gpu_histogram_time.argtypes = [vp, u32, vp, i32, f32p]
        L.hgapref_gpu_encode_time.argtypes = [vp, u32, u32p, u32p, u32, u32, vp, vp, i32, f32p]
        L.hgapref_gpu_decode_time.argtypes = [vp, u32, u32, u32, u8p, u8p, i32, vp, C.c_size_t, i32, f32p]
        for f in (L.hgapref_gpu_histogram_time, L.hgapref_gpu_encode_time, L.hgapref_gpu_decode_time):
            f.restype = C.c_int
        _lib = L
    return _lib


def _f32(k):
    return np.zeros(k, np.float32)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def padded_input(x, device):
    """x (uint8 tensor) copied into a buffer with 8 KiB + 4 bytes of zeroed
    slack: the reference's histogram reads whole words and cuencoder's idle
    threads of the last tile read before testing the length
    (encoder/src/encoder.cu:52-56,183)."""
    import torch
    buf = torch.zeros(x.numel() + 8192 + 64, dtype=torch.uint8, device=device)
    buf[:x.numel()].copy_(x)
    return buf


def histogram(buf, n: int):
    """One run of the reference histogram kernels on the padded buffer:
    (counts, ms of cu_histgram, ms of mergeHistogram)."""
    import torch
    h = torch.zeros(256, dtype=torch.int32, device=buf.device)
    ms = _f32(2)
    rc = lib().hgapref_gpu_histogram_time(buf.data_ptr(), n, h.data_ptr(), 1, _fp(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU histogram failed ({rc})")
    return h.cpu().numpy().view(np.uint32), float(ms[0]), float(ms[1])


def encode(buf, n: int, cb: "O.Codebook"):
    """One run of the reference encoder kernels: (bits, gaps, ms of the
    memsets, ms of cuencoder, ms of cu_get_gaparray)."""
    import torch
    _, W, S, G = cb.sizes()
    bits = torch.empty(W + 4, dtype=torch.int32, device=buf.device)
    gaps = torch.empty(G + 4, dtype=torch.int32, device=buf.device)
    ms = _f32(3)
    rc = lib().hgapref_gpu_encode_time(buf.data_ptr(), n, cb.code.ctypes.data_as(C.POINTER(C.c_uint32)),
                                       cb.length.ctypes.data_as(C.POINTER(C.c_uint32)), W, S,
                                       bits.data_ptr(), gaps.data_ptr(), 1, _fp(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU encode failed ({rc})")
    return bits[:W], gaps[:G], float(ms[0]), float(ms[1]), float(ms[2])


class DecodeBuffers:
    """The reference decoder's input (gap array then bitstream, with spare
    words after it) and its oversized output (it writes past n and memsets
    4 * (gap words + words) bytes, decoder/src/decoder.cu:529,763).

    The output starts zeroed, as the fresh cudaMalloc of decoder_l1_l2 is in
    practice: the reference clears only 4 * (gap words + words) bytes of it
    before each launch (decoder.cu:763, less than n for any compressing
    stream) yet ORs every thread's first and last output word into place
    (decoder.cu:704,727), so stale bytes beyond its memset would corrupt its
    output (a reference defect this harness does not trigger; between
    repetitions that tail holds the previous, identical decode)."""

    def __init__(self, bits, gaps, n: int):
        import torch
        W, G = bits.numel(), gaps.numel()
        self.words, self.gap_words, self.n = W, G, n
        self.input = torch.zeros(G + W + 16, dtype=torch.int32, device=bits.device)
        self.input[:G].copy_(gaps)
        self.input[G:G + W].copy_(bits)
        self.out_bytes = max(n + 512, 4 * (G + W)) + 4096
        self.out = torch.zeros(self.out_bytes, dtype=torch.uint8, device=bits.device)


def whole_block_prefix(x, cb: "O.Codebook") -> int:
    """The longest prefix of x (a uint8 device tensor) whose stream under
    codebook cb fills whole 128-segment blocks of the reference decoder.

    gpu_dec_l1_l2 runs one thread per segment in blocks of 128 and guards
    the whole body -- warp shuffles and block barriers included -- with
    `input_ptr < gap_element_num` (decoder/src/decoder.cu:501-520, shuffles
    and barriers at :571-653), so in a last block that is not full, lanes
    skip shuffles and barriers the others execute; on B200 its output near
    the end of such streams is wrong.  On a stream of whole blocks it decodes
    exactly.  Only the last few thousand bytes are examined: at most 128
    segments (16 Ki bits) are dropped."""
    import torch
    n = x.numel()
    lens = torch.from_numpy(cb.length.astype(np.int64)).to(x.device)
    tail = min(n, 1 << 17)
    tl = lens[x[n - tail:].long()]
    total = int(cb.total_bits)
    # bits of the stream when the last k bytes are dropped, k = 0 .. tail
    drop = torch.cat([torch.zeros(1, dtype=torch.int64, device=x.device), torch.cumsum(tl.flip(0), 0)])
    bits = total - drop
    segs = (bits + 127) // 128
    ok = torch.nonzero((segs % 128 == 0) & (bits > 0)).flatten()
    if ok.numel() == 0:
        return 0
    return n - int(ok[0].item())


def with_total_bits(cb: "O.Codebook", bits: int) -> "O.Codebook":
    """cb for a shorter input: same codes, `bits` stream bits."""
    return O.Codebook(cb.symbols, cb.lengths, cb.code, cb.length, bits)


def decode(bufs: DecodeBuffers, segments: int, cb: "O.Codebook"):
    """One run of gpu_dec_l1_l2: (output view of n bytes, ms of the memsets,
    ms of the kernel), or None where the reference's own level-1 boundary is
    wrong for this book (decoder/src/get_table.cpp:20-27; not run then)."""
    ms = _f32(2)
    rc = lib().hgapref_gpu_decode_time(bufs.input.data_ptr(), bufs.words, bufs.n, segments,
                                       cb.symbols.ctypes.data_as(C.POINTER(C.c_uint8)),
                                       cb.lengths.ctypes.data_as(C.POINTER(C.c_uint8)), cb.count,
                                       bufs.out.data_ptr(), bufs.out_bytes, 1, _fp(ms))
    if rc == -2:
        return None
    if rc != 0:
        raise RuntimeError(f"reference GPU decode failed ({rc})")
    return bufs.out[:bufs.n], float(ms[0]), float(ms[1])
