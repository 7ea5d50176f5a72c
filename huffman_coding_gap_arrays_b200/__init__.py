"""B200-native Huffman coding with gap arrays.

A drop-in for the hot path of daisuke-takafuji/Huffman_coding_Gap_arrays
(byte histogram, length-limited canonical codebook, gap-array encoder,
segment-parallel decoder) in the reference's compressed format.  The compute
runs in hand-written sm_100a kernels inside libhgap.so, called through the C
ABI declared in include/hgap.h; this package is the host-side binding.
"""
from ._lib import HgapError, lib  # noqa: F401  (fails loudly if libhgap.so is missing)
from .codec import (Codebook, Compressed, Decoder, Encoder, StreamSizes, compress,  # noqa: F401
                    decompress, histogram)
