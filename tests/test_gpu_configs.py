"""The benchmark configs at full size on the GPU: the 16 MiB Zipf(1.2)
buffer, the 1 GiB mixed Zipf/Gaussian buffer and the two BF16 byte planes of
256M weights.  Bitstream and gap array are compared with the threaded CPU
oracle byte for byte, and decode(encode(x)) == x on the device."""
import os

import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import workloads as WL
from oracle import oracle as O

pytestmark = pytest.mark.gpu
THREADS = max(1, min(64, len(os.sched_getaffinity(0))))


def round_trip_against_oracle(x: torch.Tensor):
    n = x.numel()
    hist = H.histogram(x)
    xh = x.cpu().numpy()
    h_o = O.histogram_mt(xh, THREADS)
    assert np.array_equal(hist.cpu().numpy().view(np.uint32), h_o)
    book, sizes = H.Codebook.from_histogram(hist.cpu())
    cb = O.codebook(h_o)
    assert np.array_equal(book.lengths, cb.lengths) and np.array_equal(book.symbols, cb.symbols)
    bits, gaps = H.Encoder(n).encode(x, book, sizes)
    bits_o, gaps_o = O.encode_mt(xh, cb, cb.total_bits, THREADS)
    assert np.array_equal(bits.cpu().numpy().view(np.uint32), bits_o)
    assert np.array_equal(gaps.cpu().numpy().view(np.uint32), gaps_o)
    y = H.Decoder(sizes.segments).decode(bits, gaps, sizes, book, n)
    assert torch.equal(y, x)
    return book, sizes


def test_zipf_16m(cuda):
    x = WL.zipf_buffer(16 << 20, 1.2, seed=1)
    book, sizes = round_trip_against_oracle(x)
    assert 5.0 < sizes.bits / x.numel() < 5.6


def test_mixed_1g(cuda):
    x = WL.mixed_buffer(1 << 30, seed=2)
    book, sizes = round_trip_against_oracle(x)
    assert 7.0 < sizes.bits / x.numel() < 8.0


def test_bf16_planes(cuda):
    exp, sm = WL.bf16_planes(256 << 20, seed=3)
    book_e, sizes_e = round_trip_against_oracle(exp)
    assert book_e.lengths.max() == 16 and book_e.symbol_count < 40   # highly skewed plane
    del exp
    torch.cuda.empty_cache()
    book_m, sizes_m = round_trip_against_oracle(sm)
    assert sizes_m.bits / sm.numel() > 7.9                           # near-uniform plane expands
