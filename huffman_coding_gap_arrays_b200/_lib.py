"""ctypes binding of libhgap.so (include/hgap.h).

The library is the product: there is no Python or CPU fallback.  If the
shared object is missing the import fails loudly with the command that builds
it.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhgap.so")

HGAP_OK = 0
STATUS_NAMES = {
    0: "HGAP_OK", 1: "HGAP_ERR_INVALID_ARG", 2: "HGAP_ERR_CUDA", 3: "HGAP_ERR_TIMEOUT",
    4: "HGAP_ERR_CORRUPT", 5: "HGAP_ERR_SIZE", 6: "HGAP_ERR_WORKSPACE", 7: "HGAP_ERR_NO_CODE",
    8: "HGAP_ERR_UNSUPPORTED",
}

# Every symbol include/hgap.h declares (checked by tests/test_abi.py).
EXPORTS = [
    "hgap_status_string", "hgap_histogram", "hgap_codebook_build", "hgap_codebook_from_symbols",
    "hgap_sizes_from_bits", "hgap_encoded_bits", "hgap_encode_workspace_bytes", "hgap_encode",
    "hgap_encode_histogram", "hgap_encode_prepared", "hgap_encode_part_prepared",
    "hgap_decode_workspace_bytes", "hgap_decode", "hgap_workspace_status", "hgap_container_bytes",
    "hgap_container_write", "hgap_container_parse", "histgram", "hgap_ref_encode",
    "hgap_ref_decoder_l1_l2", "hgap_decode_noalloc", "hgap_codebook_build_device",
    "hgap_decode_table_build", "hgap_decode_table_build_device", "hgap_batch_compress_workspace_bytes",
    "hgap_batch_decompress_workspace_bytes", "hgap_batch_bits_capacity", "hgap_batch_gaps_capacity",
    "hgap_batch_compress", "hgap_batch_decompress", "hgap_batch_status", "hgap_mlp_forward",
    "hgap_mlp_loss_grad", "hgap_mlp_adam", "hgap_encode_hold", "hgap_decode_hold", "hgap_status_from_word",
    "hgap_batch_decoder_class",
]


class HgapError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}")


class SymLen(C.Structure):
    _fields_ = [("symbol", C.c_uint8), ("length", C.c_uint8)]


class Codeword(C.Structure):
    _fields_ = [("code", C.c_uint32), ("length", C.c_uint32)]


class CCodebook(C.Structure):
    _fields_ = [("symbol_count", C.c_uint32), ("symbols", SymLen * 256), ("table", Codeword * 256)]


class Sizes(C.Structure):
    _fields_ = [("bits", C.c_uint64), ("words", C.c_uint64), ("segments", C.c_uint64),
                ("gap_words", C.c_uint64)]


class BatchEntry(C.Structure):
    _fields_ = [("n", C.c_uint64), ("bits", C.c_uint64), ("words", C.c_uint64),
                ("segments", C.c_uint64), ("gap_words", C.c_uint64), ("bits_offset", C.c_uint64),
                ("gaps_offset", C.c_uint64), ("symbol_count", C.c_uint32), ("status", C.c_uint32),
                ("symbols", SymLen * 256)]


class BatchConfig(C.Structure):
    _fields_ = [("region_chunks", C.c_uint32), ("hist_ctas_per_sm", C.c_uint32),
                ("enc_ctas_per_sm", C.c_uint32), ("dec_ctas_per_sm", C.c_uint32),
                ("dec_tile_segs", C.c_uint32), ("dec_class_mask", C.c_uint32)]


DEC_T1_ENTRIES = 2048
DEC_T2_ENTRIES = 2560
MLP_IN, MLP_HIDDEN, MLP_OUT = 10, 32, 2
MLP_PARAMS = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_OUT * MLP_HIDDEN + MLP_OUT


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with "
            "`python -m huffman_coding_gap_arrays_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    vp, u32p, u64 = C.c_void_p, C.POINTER(C.c_uint32), C.c_uint64
    L.hgap_status_string.argtypes = [C.c_int]
    L.hgap_status_string.restype = C.c_char_p
    L.hgap_histogram.argtypes = [vp, u64, vp, vp]
    L.hgap_codebook_build.argtypes = [u32p, C.POINTER(CCodebook), C.POINTER(Sizes)]
    L.hgap_codebook_from_symbols.argtypes = [C.POINTER(SymLen), C.c_uint32, C.POINTER(CCodebook)]
    L.hgap_sizes_from_bits.argtypes = [u64]
    L.hgap_sizes_from_bits.restype = Sizes
    L.hgap_encoded_bits.argtypes = [C.POINTER(CCodebook), u32p]
    L.hgap_encoded_bits.restype = u64
    L.hgap_encode_workspace_bytes.argtypes = [u64]
    L.hgap_encode_workspace_bytes.restype = C.c_size_t
    L.hgap_encode.argtypes = [vp, u64, C.POINTER(CCodebook), vp, u64, vp, u64, vp, C.c_size_t, vp]
    L.hgap_encode_prepared.argtypes = L.hgap_encode.argtypes
    L.hgap_encode_histogram.argtypes = [vp, u64, vp, vp, C.c_size_t, vp]
    L.hgap_encode_part_prepared.argtypes = [vp, u64, C.POINTER(CCodebook), u64, u64, vp, u64, vp, u64, vp,
                                            C.c_size_t, vp]
    L.hgap_decode_workspace_bytes.argtypes = [u64]
    L.hgap_decode_workspace_bytes.restype = C.c_size_t
    L.hgap_decode.argtypes = [vp, u64, vp, u64, C.POINTER(CCodebook), vp, u64, vp, C.c_size_t, vp]
    L.hgap_workspace_status.argtypes = [vp, vp]
    L.hgap_status_from_word.argtypes = [C.c_uint32]
    L.hgap_encode_hold.argtypes = L.hgap_encode.argtypes + [u64, u64]
    L.hgap_decode_hold.argtypes = L.hgap_decode.argtypes + [u64, u64]
    L.hgap_decode_noalloc.argtypes = [vp, u64, vp, u64, C.POINTER(CCodebook), vp, u64, vp]
    L.hgap_container_bytes.argtypes = [C.c_uint32, u64, u64]
    L.hgap_container_bytes.restype = C.c_size_t
    L.hgap_container_write.argtypes = [vp, C.c_size_t, C.POINTER(CCodebook), u64, u64, u64, vp, vp,
                                       C.POINTER(C.c_size_t)]
    L.hgap_container_parse.argtypes = [vp, C.c_size_t, C.POINTER(CCodebook), C.POINTER(u64),
                                       C.POINTER(u64), C.POINTER(u64), C.POINTER(vp), C.POINTER(vp)]
    L.histgram.argtypes = [vp, vp, C.c_uint32]
    L.histgram.restype = None
    L.hgap_ref_encode.argtypes = [vp, C.c_uint32, vp, C.c_uint32, C.c_uint32, C.POINTER(Codeword)]
    L.hgap_ref_decoder_l1_l2.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int, C.c_uint32,
                                         C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
    u64p = C.POINTER(C.c_uint64)
    L.hgap_codebook_build_device.argtypes = [C.c_uint32, vp, vp, vp, vp]
    L.hgap_decode_table_build.argtypes = [C.POINTER(CCodebook), vp, vp]
    L.hgap_decode_table_build_device.argtypes = [C.c_uint32, vp, vp, vp, vp]
    L.hgap_batch_compress_workspace_bytes.argtypes = [C.c_uint32, u64p, C.POINTER(BatchConfig)]
    L.hgap_batch_compress_workspace_bytes.restype = C.c_size_t
    L.hgap_batch_decompress_workspace_bytes.argtypes = [C.c_uint32, u64p]
    L.hgap_batch_decompress_workspace_bytes.restype = C.c_size_t
    L.hgap_batch_bits_capacity.argtypes = [C.c_uint32, u64p]
    L.hgap_batch_bits_capacity.restype = u64
    L.hgap_batch_gaps_capacity.argtypes = [C.c_uint32, u64p]
    L.hgap_batch_gaps_capacity.restype = u64
    L.hgap_batch_compress.argtypes = [C.c_uint32, vp, vp, vp, vp, u64, vp, u64, vp, vp, C.c_size_t,
                                      C.POINTER(BatchConfig), vp]
    L.hgap_batch_decompress.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, C.c_size_t,
                                        C.POINTER(BatchConfig), vp]
    L.hgap_batch_status.argtypes = [vp, vp]
    L.hgap_batch_decoder_class.argtypes = [C.POINTER(SymLen), C.c_uint32]
    L.hgap_batch_decoder_class.restype = C.c_uint32
    L.hgap_mlp_forward.argtypes = [vp, vp, C.c_uint32, vp, vp]
    L.hgap_mlp_loss_grad.argtypes = [vp, vp, vp, C.c_uint32, C.c_float, vp, vp, vp]
    L.hgap_mlp_adam.argtypes = [vp, vp, vp, vp, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float,
                                C.c_float, vp]
    for name in ("hgap_codebook_build_device", "hgap_decode_table_build", "hgap_decode_table_build_device",
                 "hgap_batch_compress", "hgap_batch_decompress", "hgap_batch_status", "hgap_mlp_forward",
                 "hgap_mlp_loss_grad", "hgap_mlp_adam"):
        getattr(L, name).restype = C.c_int
    for name in ("hgap_histogram", "hgap_codebook_build", "hgap_codebook_from_symbols",
                 "hgap_encode", "hgap_encode_histogram", "hgap_encode_prepared", "hgap_encode_part_prepared",
                 "hgap_decode", "hgap_workspace_status", "hgap_container_write",
                 "hgap_container_parse", "hgap_ref_encode", "hgap_ref_decoder_l1_l2",
                 "hgap_decode_noalloc", "hgap_status_from_word"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != HGAP_OK:
        raise HgapError(status, where)
