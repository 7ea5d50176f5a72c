"""ctypes bindings of the C oracle (liboracle.so) and of the reference's own
sources compiled into oracle/_ref (libref_encoder.so, libref_decoder_host.so).

Test infrastructure only: the checker, never the thing measured or shipped.
Functions mirror hgap_oracle.h; see there for the reference file:line each
one restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)


class OrcSizes(C.Structure):
    _fields_ = [("bits", C.c_uint64), ("words", C.c_uint64),
                ("segments", C.c_uint64), ("gap_words", C.c_uint64)]


class OrcSymbol(C.Structure):
    _fields_ = [("symbol", C.c_uint8), ("length", C.c_uint8), ("count", C.c_uint32)]


class OrcTableInfo(C.Structure):
    _fields_ = [("l1table_size", C.c_uint32), ("l2table_size", C.c_uint32),
                ("ptrtable_size", C.c_uint32)]


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and oracle/_ref where the reference is present)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def _ptr(a, t):
    return a.ctypes.data_as(t)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_histogram.argtypes = [_u8p, C.c_uint64, _u32p]
        L.orc_codebook.argtypes = [_u32p, C.POINTER(OrcSymbol), _u32p, _u32p]
        L.orc_codebook.restype = C.c_int
        L.orc_canonical_codes.argtypes = [_u8p, _u8p, C.c_int, _u32p, _u32p]
        L.orc_sizes_from_bits.argtypes = [C.c_uint64]
        L.orc_sizes_from_bits.restype = OrcSizes
        L.orc_encode.argtypes = [_u8p, C.c_uint64, _u32p, _u32p, _u32p, C.c_uint64,
                                 _u32p, C.c_uint64, _u64p]
        L.orc_encode.restype = C.c_int
        L.orc_decode.argtypes = [_u32p, C.c_uint64, _u32p, C.c_uint64, _u8p, _u8p, C.c_int,
                                 _u8p, C.c_uint64]
        L.orc_decode.restype = C.c_int
        L.orc_ref_table_info.argtypes = [_u8p, _u8p, C.c_int, C.c_uint32,
                                         C.POINTER(OrcTableInfo), C.c_int]
        L.orc_ref_table_info.restype = C.c_uint32
        L.orc_ref_twolevel_table.argtypes = [C.c_void_p, C.c_uint32, _u8p, _u8p, C.c_int,
                                             OrcTableInfo]
        L.orc_ref_twolevel_table.restype = C.c_uint32
        L.orc_ref_table_bytes.argtypes = [OrcTableInfo]
        L.orc_ref_table_bytes.restype = C.c_size_t
        L.orc_container_bytes.argtypes = [C.c_int, C.c_uint64, C.c_uint64]
        L.orc_container_bytes.restype = C.c_size_t
        L.orc_container_write.argtypes = [_u8p, _u8p, _u8p, C.c_int, C.c_uint32, C.c_uint32,
                                          C.c_uint32, _u32p, _u32p]
        L.orc_container_write.restype = C.c_size_t
        L.orc_mt_encode.argtypes = [_u8p, C.c_uint64, _u32p, _u32p, _u32p, C.c_uint64, _u32p,
                                    C.c_uint64, C.c_int]
        L.orc_mt_encode.restype = C.c_int
        L.orc_mt_histogram.argtypes = [_u8p, C.c_uint64, _u32p, C.c_int]
        L.orc_mt_histogram.restype = C.c_int
        L.orc_mt_decode.argtypes = [_u32p, C.c_uint64, _u32p, C.c_uint64, _u8p, _u8p, C.c_int,
                                    _u8p, C.c_uint64, C.c_int]
        L.orc_mt_decode.restype = C.c_int
        _lib = L
    return _lib


class Codebook:
    """Oracle codebook: container-order list plus per-byte code/length tables."""

    def __init__(self, symbols, lengths, code, length, total_bits):
        self.symbols = np.ascontiguousarray(symbols, dtype=np.uint8)
        self.lengths = np.ascontiguousarray(lengths, dtype=np.uint8)
        self.code = np.ascontiguousarray(code, dtype=np.uint32)
        self.length = np.ascontiguousarray(length, dtype=np.uint32)
        self.total_bits = int(total_bits)

    @property
    def count(self) -> int:
        return int(self.symbols.size)

    def sizes(self):
        z = lib().orc_sizes_from_bits(self.total_bits)
        return z.bits, z.words, z.segments, z.gap_words


def histogram(data: np.ndarray) -> np.ndarray:
    data = np.ascontiguousarray(data, dtype=np.uint8)
    h = np.zeros(256, np.uint32)
    lib().orc_histogram(_ptr(data, _u8p), data.size, _ptr(h, _u32p))
    return h


def histogram_mt(data: np.ndarray, threads: int) -> np.ndarray:
    data = np.ascontiguousarray(data, dtype=np.uint8)
    h = np.zeros(256, np.uint32)
    lib().orc_mt_histogram(_ptr(data, _u8p), data.size, _ptr(h, _u32p), threads)
    return h


def codebook(hist: np.ndarray) -> Codebook:
    hist = np.ascontiguousarray(hist, dtype=np.uint32)
    sorted_ = (OrcSymbol * 256)()
    code = np.zeros(256, np.uint32)
    length = np.zeros(256, np.uint32)
    n = lib().orc_codebook(_ptr(hist, _u32p), sorted_, _ptr(code, _u32p), _ptr(length, _u32p))
    syms = np.array([sorted_[n - 1 - i].symbol for i in range(n)], np.uint8)
    lens = np.array([sorted_[n - 1 - i].length for i in range(n)], np.uint8)
    bits = int(sum(int(length[b]) * int(hist[b]) for b in range(256)))
    return Codebook(syms, lens, code, length, bits)


def codebook_from_list(symbols, lengths, total_bits: int = 0) -> Codebook:
    symbols = np.ascontiguousarray(symbols, dtype=np.uint8)
    lengths = np.ascontiguousarray(lengths, dtype=np.uint8)
    code = np.zeros(256, np.uint32)
    length = np.zeros(256, np.uint32)
    lib().orc_canonical_codes(_ptr(symbols, _u8p), _ptr(lengths, _u8p), symbols.size,
                              _ptr(code, _u32p), _ptr(length, _u32p))
    return Codebook(symbols, lengths, code, length, total_bits)


def encode(data: np.ndarray, cb: Codebook):
    """Serial encode; returns (bitstream u32[W], gap u32[ceil(S/8)], bits)."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    bits_total = int(sum(int(cb.length[b]) * c for b, c in enumerate(histogram(data).tolist())))
    z = lib().orc_sizes_from_bits(bits_total)
    bits = np.zeros(max(z.words, 1), np.uint32)
    gaps = np.zeros(max(z.gap_words, 1), np.uint32)
    out_bits = C.c_uint64(0)
    rc = lib().orc_encode(_ptr(data, _u8p), data.size, _ptr(cb.code, _u32p),
                          _ptr(cb.length, _u32p), _ptr(bits, _u32p), z.words,
                          _ptr(gaps, _u32p), z.gap_words, C.byref(out_bits))
    if rc != 0:
        raise ValueError(f"oracle encode failed ({rc})")
    return bits[:z.words], gaps[:z.gap_words], bits_total


def encode_mt(data: np.ndarray, cb: Codebook, bits_total: int, threads: int):
    data = np.ascontiguousarray(data, dtype=np.uint8)
    z = lib().orc_sizes_from_bits(bits_total)
    bits = np.zeros(max(z.words, 1), np.uint32)
    gaps = np.zeros(max(z.gap_words, 1), np.uint32)
    rc = lib().orc_mt_encode(_ptr(data, _u8p), data.size, _ptr(cb.code, _u32p),
                             _ptr(cb.length, _u32p), _ptr(bits, _u32p), z.words,
                             _ptr(gaps, _u32p), z.gap_words, threads)
    if rc != 0:
        raise ValueError(f"oracle mt encode failed ({rc})")
    return bits[:z.words], gaps[:z.gap_words]


def decode(bits: np.ndarray, gaps: np.ndarray, segments: int, cb: Codebook, n: int) -> np.ndarray:
    bits = np.ascontiguousarray(bits, dtype=np.uint32)
    gaps = np.ascontiguousarray(gaps, dtype=np.uint32)
    out = np.zeros(max(n, 1), np.uint8)
    rc = lib().orc_decode(_ptr(bits, _u32p), bits.size, _ptr(gaps, _u32p), segments,
                          _ptr(cb.symbols, _u8p), _ptr(cb.lengths, _u8p), cb.count,
                          _ptr(out, _u8p), n)
    if rc != 0:
        raise ValueError(f"oracle decode failed ({rc})")
    return out[:n]


def decode_mt(bits, gaps, segments: int, cb: Codebook, n: int, threads: int) -> np.ndarray:
    bits = np.ascontiguousarray(bits, dtype=np.uint32)
    gaps = np.ascontiguousarray(gaps, dtype=np.uint32)
    out = np.zeros(max(n, 1), np.uint8)
    rc = lib().orc_mt_decode(_ptr(bits, _u32p), bits.size, _ptr(gaps, _u32p), segments,
                             _ptr(cb.symbols, _u8p), _ptr(cb.lengths, _u8p), cb.count,
                             _ptr(out, _u8p), n, threads)
    if rc != 0:
        raise ValueError(f"oracle mt decode failed ({rc})")
    return out[:n]


def container(cb: Codebook, n: int, bits: np.ndarray, gaps: np.ndarray, segments: int) -> bytes:
    bits = np.ascontiguousarray(bits, dtype=np.uint32)
    gaps = np.ascontiguousarray(gaps, dtype=np.uint32)
    size = lib().orc_container_bytes(cb.count, bits.size, gaps.size)
    buf = np.zeros(size, np.uint8)
    w = lib().orc_container_write(_ptr(buf, _u8p), _ptr(cb.symbols, _u8p),
                                  _ptr(cb.lengths, _u8p), cb.count, n, bits.size, segments,
                                  _ptr(gaps, _u32p), _ptr(bits, _u32p))
    assert w == size
    return buf.tobytes()


def ref_table(cb: Codebook, prefix_bit: int = 10, reference_bug: bool = False):
    """The reference-format two-level LUT blob (decoder/src/get_table.cpp)."""
    info = OrcTableInfo()
    p = lib().orc_ref_table_info(_ptr(cb.symbols, _u8p), _ptr(cb.lengths, _u8p), cb.count,
                                 prefix_bit, C.byref(info), int(reference_bug))
    if reference_bug:
        return p, (info.l1table_size, info.l2table_size, info.ptrtable_size), None, None
    blob = np.zeros(lib().orc_ref_table_bytes(info), np.uint8)
    boundary = lib().orc_ref_twolevel_table(blob.ctypes.data, p, _ptr(cb.symbols, _u8p),
                                            _ptr(cb.lengths, _u8p), cb.count, info)
    return p, (info.l1table_size, info.l2table_size, info.ptrtable_size), blob, boundary


# ---------------------------------------------------------------- reference ---

_ref_enc = None
_ref_dec = None


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_encoder.so"))


def ref_encoder():
    global _ref_enc
    if _ref_enc is None:
        L = C.CDLL(os.path.join(REF_DIR, "libref_encoder.so"))
        L.hgapref_codebook.argtypes = [_u32p, _u8p, _u8p, _u32p, _u32p, _u64p]
        L.hgapref_codebook.restype = C.c_int
        L.hgapref_gpu_encode.argtypes = [_u8p, C.c_uint32, _u32p, _u32p, _u32p, C.c_uint32,
                                         C.c_uint32, _u32p]
        L.hgapref_gpu_encode.restype = C.c_int
        _ref_enc = L
    return _ref_enc


def ref_decoder_host():
    global _ref_dec
    if _ref_dec is None:
        L = C.CDLL(os.path.join(REF_DIR, "libref_decoder_host.so"))
        L.hgapref_twolevel_table.argtypes = [_u8p, _u8p, C.c_int, C.c_int, _u32p, _u8p,
                                             C.c_uint64, _u32p]
        L.hgapref_twolevel_table.restype = C.c_int
        _ref_dec = L
    return _ref_dec


def ref_codebook(hist: np.ndarray):
    """Reference codebook (store_symbols + qsort(compare) + boundary_PM)."""
    hist = np.ascontiguousarray(hist, dtype=np.uint32)
    syms = np.zeros(256, np.uint8)
    lens = np.zeros(256, np.uint8)
    code = np.zeros(256, np.uint32)
    length = np.zeros(256, np.uint32)
    bits = C.c_uint64(0)
    n = ref_encoder().hgapref_codebook(_ptr(hist, _u32p), _ptr(syms, _u8p), _ptr(lens, _u8p),
                                       _ptr(code, _u32p), _ptr(length, _u32p), C.byref(bits))
    if n < 2:
        return None
    return Codebook(syms[:n], lens[:n], code, length, bits.value)


def ref_twolevel_table(cb: Codebook, prefix_bit: int = 10):
    info = np.zeros(3, np.uint32)
    cap = 1 << 20
    blob = np.zeros(cap, np.uint8)
    boundary = C.c_uint32(0)
    p = ref_decoder_host().hgapref_twolevel_table(
        _ptr(cb.symbols, _u8p), _ptr(cb.lengths, _u8p), cb.count, prefix_bit, _ptr(info, _u32p),
        _ptr(blob, _u8p), cap, C.byref(boundary))
    size = int(info[2]) * 4 + 256 + int(info[0]) + int(info[1])
    return p, tuple(int(x) for x in info), (blob[:size] if p >= 0 else None), boundary.value


def ref_gpu_encode(data: np.ndarray, cb: Codebook):
    """The reference's own GPU histgram()+encode() (needs a GPU)."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    _, W, S, G = cb.sizes()
    out = np.zeros(W + G + 1, np.uint32)
    hist = np.zeros(256, np.uint32)
    rc = ref_encoder().hgapref_gpu_encode(_ptr(data, _u8p), data.size, _ptr(hist, _u32p),
                                          _ptr(cb.code, _u32p), _ptr(cb.length, _u32p), W, S,
                                          _ptr(out, _u32p))
    if rc != 0:
        raise RuntimeError(f"reference GPU encode failed ({rc})")
    return hist, out[:W], out[W:W + G]
