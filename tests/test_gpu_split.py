"""One buffer encoded as contiguous parts (hgap_encode_part_prepared, as the
ranks of parallel.compress_split would on their GPUs), on one GPU: the parts
run one after another in this process -- none waits on another -- and their
windows, OR-ed together, must equal the single-device compress of the whole
buffer bit for bit (bitstream and gap array), and decode back to it.  Cut
points cover empty parts, one-byte parts, parts ending inside a word, on a
word, on a segment and on a gap word, and many small parts."""
import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import parallel as PL

pytestmark = pytest.mark.gpu


def _data(dist: str, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if dist == "zipf":
        p = 1.0 / np.arange(1, 257) ** 1.2
        return rng.choice(256, size=n, p=p / p.sum()).astype(np.uint8)
    if dist == "uniform":
        return rng.integers(0, 256, size=n, dtype=np.uint8)
    if dist == "narrow":
        return np.clip(np.round(128 + 0.6 * rng.standard_normal(n)), 0, 255).astype(np.uint8)
    if dist == "deep":
        p = 1.0 / 1.618 ** np.arange(40)
        return (rng.choice(40, size=n, p=p / p.sum()).astype(np.uint8) * 5 + 3).astype(np.uint8)
    raise ValueError(dist)


def _split_encode(x: torch.Tensor, cuts):
    """The per-part steps of compress_split without the collectives."""
    codecs, parts_x, hists = [], [], []
    for a, b in zip(cuts[:-1], cuts[1:]):
        c = PL.DevicePartCodec()
        px = x[a:b]
        hists.append(c.histogram(px))
        codecs.append(c)
        parts_x.append(px)
    ghist = np.sum([h.astype(np.int64) for h in hists], axis=0)
    book, sizes = H.Codebook.from_histogram(ghist)
    counts = [book.encoded_bits(h) for h in hists]
    starts = PL.part_starts(counts)
    windows = [c.encode(px, book, s, k) for c, px, s, k in zip(codecs, parts_x, starts, counts)]
    bits, gaps = PL.stitch_parts(windows, sizes.words, sizes.gap_words, x.device)
    return book, sizes, bits, gaps


def _cut_sets(n, seed):
    rng = np.random.default_rng(seed)
    return [
        [0, n // 2, n],
        [0, 0, n // 3, n // 3, n],                     # empty parts
        [0, 1, 2, n - 1, n],                           # one-byte parts
        [0] + sorted(int(c) for c in rng.integers(0, n, size=7)) + [n],
        [0] + list(range(4096, n, 4096)) + [n],        # many equal parts
    ]


@pytest.mark.parametrize("dist", ["zipf", "uniform", "narrow", "deep"])
@pytest.mark.parametrize("n", [3, 1000, 100_003, 3 * (1 << 20) + 5])
def test_split_parts_equal_whole_buffer(cuda, dist, n):
    x = torch.from_numpy(_data(dist, n, 7)).cuda()
    ref = H.compress(x)
    for cuts in _cut_sets(n, 3):
        if n > 200_000 and len(cuts) > 20:
            cuts = [0] + list(range(1 << 18, n, 1 << 18)) + [n]
        book, sizes, bits, gaps = _split_encode(x, cuts)
        assert sizes.bits == ref.sizes.bits
        assert torch.equal(bits, ref.bits[:sizes.words]), cuts[:6]
        assert torch.equal(gaps, ref.gaps[:sizes.gap_words]), cuts[:6]
        out = H.Decoder(sizes.segments).decode(bits, gaps, sizes, book, n)
        assert torch.equal(out[:n], x)


def test_part_bit_count_mismatch_is_reported(cuda):
    """A part told the wrong bit count (its histogram disagrees) is flagged
    on the device, not silently mis-stitched."""
    x = torch.from_numpy(_data("zipf", 50_000, 2)).cuda()
    c = PL.DevicePartCodec()
    h = c.histogram(x)
    book, _ = H.Codebook.from_histogram(h)
    k = book.encoded_bits(h)
    with pytest.raises(H.HgapError):
        c.encode(x, book, 100, k + 300)


def test_compress_split_single_rank_is_compress(cuda):
    x = torch.from_numpy(_data("narrow", 777_777, 4)).cuda()
    ref = H.compress(x)
    book, n, sizes, bits, gaps = PL.compress_split(x)
    assert n == x.numel() and sizes.bits == ref.sizes.bits
    assert torch.equal(bits, ref.bits[:sizes.words]) and torch.equal(gaps, ref.gaps[:sizes.gap_words])
