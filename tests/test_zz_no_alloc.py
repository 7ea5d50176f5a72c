"""hgap_decode_noalloc: the decoder for callers that cannot allocate device
memory (their device memory belongs to a framework's pool, or they are only
handed the input and output buffers), with its scratch in a fixed array
inside libhgap.so.  Called through the C ABI, it must give exactly what
hgap_decode with a caller workspace gives, on two calls in a row (the shared
array keeps the previous call's contents, so the second call also checks
that the decoder clears what must start at zero).  Kept in its own file, named
to be collected last."""
import ctypes as C

import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import _lib

pytestmark = pytest.mark.gpu

SCRATCH = 256 * 1024


def _encoded(seed: int, n: int):
    rng = np.random.default_rng(seed)
    r = np.arange(1, 257); p = r ** -1.15; p /= p.sum()
    x = torch.from_numpy(rng.choice(256, size=n, p=p).astype(np.uint8)).to("cuda")
    return x, H.compress(x)


def _noalloc(c, out) -> int:
    L = _lib.lib()
    return L.hgap_decode_noalloc(c.bits.data_ptr(), c.sizes.words, c.gaps.data_ptr(),
                                 c.sizes.segments, C.byref(c.book.cstruct), out.data_ptr(), c.n,
                                 torch.cuda.current_stream().cuda_stream)


def test_noalloc_matches_workspace_decoder_twice(cuda):
    for call, (seed, n) in enumerate([(1, 3_000_001), (2, 1_234_567)]):
        x, c = _encoded(seed, n)
        want = H.Decoder(c.sizes.segments).decode(c.bits, c.gaps, c.sizes, c.book, c.n)
        got = torch.full((n + 8,), 0xEE, dtype=torch.uint8, device="cuda")
        assert _noalloc(c, got) == 0, f"call {call}"
        assert torch.equal(got[:n], want) and torch.equal(got[:n], x)
        assert bool((got[n:] == 0xEE).all())


def test_noalloc_rejects_streams_beyond_its_scratch(cuda):
    L = _lib.lib()
    segs = 1
    while L.hgap_decode_workspace_bytes(segs) <= SCRATCH:
        segs *= 2
    words = 4 * segs
    book = _lib.CCodebook()
    rc = L.hgap_decode_noalloc(None, words, None, segs, C.byref(book), None, 10, None)
    assert rc == 6  # HGAP_ERR_WORKSPACE, before any argument is touched
