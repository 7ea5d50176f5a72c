"""Parity with the reference's own GPU kernels, run on the same B200: its
histogram (cu_histgram + mergeHistogram), its encoder (cuencoder +
cu_get_gaparray) and its decoder (gpu_dec_l1_l2), built unmodified for
sm_100a into oracle/_ref/libref_gpu_time.so.  This library's histogram,
bitstream and gap array must equal the reference kernels' output, and the
reference decoder must restore the input.  The reference decoder runs only
where its own level-1 table boundary is right (decoder/src/get_table.cpp:20-27)
and on a stream of whole 128-segment blocks (ref_gpu.whole_block_prefix: its
last, partial block runs shuffles and barriers with lanes that skipped them)."""
import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import workloads as WL
from oracle import oracle as O
from oracle import ref_gpu as RG

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not RG.available(), reason="oracle/_ref/libref_gpu_time.so not built")]


def _cases():
    return {
        "zipf_1m": lambda: WL.zipf_buffer((1 << 20) + 3, 1.2, seed=5),
        "zipf_16m": lambda: WL.zipf_buffer(16 << 20, 1.2, seed=1),
        "mixed_48m": lambda: WL.mixed_buffer((48 << 20) + 1001, seed=2),
        "uniform_3m": lambda: torch.randint(0, 256, ((3 << 20) + 7,), dtype=torch.uint8, device="cuda",
                                            generator=torch.Generator("cuda").manual_seed(9)),
    }


@pytest.mark.parametrize("name", list(_cases()))
def test_reference_kernels_agree_with_ours(cuda, name):
    x = _cases()[name]()
    n = x.numel()
    buf = RG.padded_input(x, x.device)
    h_ref, _, _ = RG.histogram(buf, n)
    h = H.histogram(x).cpu().numpy().view(np.uint32)
    assert np.array_equal(h, h_ref)
    cb = O.ref_codebook(h_ref)
    bits_r, gaps_r, _, _, _ = RG.encode(buf, n, cb)
    book, sizes = H.Codebook.from_histogram(h)
    assert (sizes.words, sizes.gap_words) == (bits_r.numel(), gaps_r.numel())
    bits, gaps = H.Encoder(n).encode(x, book, sizes)
    assert torch.equal(bits, bits_r)
    assert torch.equal(gaps, gaps_r)
    # the reference decoder: on the longest prefix that fills whole blocks, encoded with
    # the same codebook by both encoders
    m = RG.whole_block_prefix(x, cb)
    assert m > 0
    xp = x[:m]
    bits_p = int(torch.from_numpy(cb.length.astype(np.int64)).to(x.device)[xp.long()].sum().item())
    cbp = RG.with_total_bits(cb, bits_p)
    _, W, S, G = cbp.sizes()
    assert S % 128 == 0
    rb, rg, _, _, _ = RG.encode(RG.padded_input(xp, x.device), m, cbp)
    ob, og = H.Encoder(m).encode(xp, book, H.StreamSizes.from_bits(bits_p))
    assert torch.equal(ob, rb) and torch.equal(og, rg)
    res = RG.decode(RG.DecodeBuffers(rb, rg, m), S, cbp)
    if res is None:
        pytest.skip("the reference's level-1 boundary is wrong for this book")
    y, _, _ = res
    assert torch.equal(y, xp)
