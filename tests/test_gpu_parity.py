"""Parity of the sm_100a kernels (through libhgap.so's C ABI) with the CPU
oracle: histogram counts equal, bitstream and gap array byte-equal, decode
bit-exact -- over ragged sizes, every input/output alignment, 1- to 16-bit
codes, single-symbol inputs and the error paths."""
import ctypes as C

import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 4, 5, 15, 16, 17, 31, 33, 100, 1000, 4095, 8191, 8192, 8193, 16384,
         24577, 65536, 100_003, 1 << 20, 3 * (1 << 20) + 7]


def make(dist: str, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if dist == "zipf":
        r = np.arange(1, 257); p = r ** -1.2; p /= p.sum()
        return rng.choice(256, size=n, p=p).astype(np.uint8)
    if dist == "uniform":
        return rng.integers(0, 256, size=n, dtype=np.uint8)
    if dist == "two":
        return rng.integers(0, 2, size=n, dtype=np.uint8)
    if dist == "single":
        return np.full(n, 77, np.uint8)
    if dist == "narrow":  # quantised N(128, 0.6): a 1-bit shortest code, up to three codes per lookup
        return np.clip(np.round(128 + 0.6 * rng.standard_normal(n)), 0, 255).astype(np.uint8)
    if dist == "deep":  # Fibonacci-like skew -> codes up to the 16-bit limit
        p = 1.0 / 1.618 ** np.arange(40); p /= p.sum()
        x = rng.choice(40, size=n, p=p).astype(np.uint8)
        return (x * 5 + 3).astype(np.uint8)
    raise ValueError(dist)


def to_dev(x: np.ndarray, offset: int = 0) -> torch.Tensor:
    """x placed `offset` bytes into a fresh device buffer (unaligned views)."""
    buf = torch.empty(x.size + offset + 16, dtype=torch.uint8, device="cuda")
    buf.fill_(0xA5)
    view = buf[offset:offset + x.size]
    view.copy_(torch.from_numpy(x))
    return view


def u32(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("offset", [0, 1, 7, 15])
@pytest.mark.parametrize("n", [1, 17, 1000, 65536, 1 << 20, 5 * (1 << 20) + 3])
def test_histogram(cuda, n, offset):
    x = make("zipf", n, n + offset)
    h = H.histogram(to_dev(x, offset))
    assert np.array_equal(u32(h), O.histogram(x))


def test_histogram_skewed_and_empty(cuda):
    x = np.zeros(3_000_001, np.uint8)
    assert np.array_equal(u32(H.histogram(to_dev(x))), O.histogram(x))
    empty = torch.empty(0, dtype=torch.uint8, device="cuda")
    assert int(H.histogram(empty).sum()) == 0


@pytest.mark.parametrize("dist", ["zipf", "uniform", "two", "deep", "single", "narrow"])
@pytest.mark.parametrize("n", SIZES)
def test_encode_decode_match_oracle(cuda, dist, n):
    x = make(dist, n, 1000 + n)
    h = O.histogram(x)
    ob = O.codebook(h)
    bits_o, gaps_o, B = O.encode(x, ob)
    book, sizes = H.Codebook.from_histogram(h)
    assert sizes.bits == B
    for off in (0, 5):
        d = to_dev(x, off)
        bits, gaps = H.Encoder(n).encode(d, book, sizes)
        assert np.array_equal(u32(bits), bits_o), f"bitstream differs (offset {off})"
        assert np.array_equal(u32(gaps), gaps_o), f"gap array differs (offset {off})"
    for out_off in (0, 3):
        out = torch.full((n + 32,), 0x5A, dtype=torch.uint8, device="cuda")
        y = H.Decoder(sizes.segments).decode(bits, gaps, sizes, book, n, out=out[out_off:])
        assert np.array_equal(y.cpu().numpy(), x)
        guard = out.cpu().numpy()
        assert (guard[:out_off] == 0x5A).all() and (guard[out_off + n:] == 0x5A).all()


def test_code_lengths_reach_16_bits(cuda):
    f = [1, 1]
    while len(f) < 24:
        f.append(f[-1] + f[-2])
    x = np.concatenate([np.full(c, i * 7, np.uint8) for i, c in enumerate(f)])
    np.random.default_rng(0).shuffle(x)
    h = O.histogram(x)
    book, sizes = H.Codebook.from_histogram(h)
    assert book.lengths.max() == 16
    bits_o, gaps_o, _ = O.encode(x, O.codebook(h))
    bits, gaps = H.Encoder(x.size).encode(to_dev(x, 3), book, sizes)
    assert np.array_equal(u32(bits), bits_o) and np.array_equal(u32(gaps), gaps_o)
    y = H.Decoder(sizes.segments).decode(bits, gaps, sizes, book, x.size)
    assert np.array_equal(y.cpu().numpy(), x)


def test_segment_boundary_cases(cuda):
    # 4-bit codes only (16 equiprobable symbols): every codeword ends on a
    # 128-bit boundary, so every gap entry is 0
    x = np.tile(np.arange(16, dtype=np.uint8), 4096)
    h = O.histogram(x)
    book, sizes = H.Codebook.from_histogram(h)
    assert set(book.lengths.tolist()) == {4}
    bits, gaps = H.Encoder(x.size).encode(to_dev(x), book, sizes)
    assert not u32(gaps).any()
    bits_o, gaps_o, _ = O.encode(x, O.codebook(h))
    assert np.array_equal(u32(bits), bits_o) and np.array_equal(u32(gaps), gaps_o)
    y = H.Decoder(sizes.segments).decode(bits, gaps, sizes, book, x.size)
    assert np.array_equal(y.cpu().numpy(), x)


def test_reused_workspace_and_side_stream(cuda):
    enc = H.Encoder(1 << 20)
    dec = H.Decoder(1 << 16)
    s = torch.cuda.Stream()
    for seed in range(4):
        x = make("zipf" if seed % 2 else "uniform", (1 << 20) - seed * 1001, seed)
        h = O.histogram(x)
        book, sizes = H.Codebook.from_histogram(h)
        d = to_dev(x, seed)
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            bits, gaps = enc.encode(d, book, sizes, stream=s)
            y = dec.decode(bits, gaps, sizes, book, x.size, stream=s)
        s.synchronize()
        bits_o, gaps_o, _ = O.encode(x, O.codebook(h))
        assert np.array_equal(u32(bits), bits_o) and np.array_equal(u32(gaps), gaps_o)
        assert np.array_equal(y.cpu().numpy(), x)


@pytest.mark.parametrize("cap_chunks,n_chunks", [(300, 296), (600, 592), (9500, 9400)])
def test_workspace_for_capacity_serves_smaller_inputs(cuda, cap_chunks, n_chunks):
    """An encoder workspace sized for `capacity` bytes takes any smaller input,
    also one the super-tile rule splits into more super-tiles than the
    capacity itself (296 chunks: 296 one-chunk super-tiles; 300 chunks: 150
    two-chunk ones), at every alignment."""
    cap = cap_chunks * 8192 - 100
    enc = H.Encoder(cap)
    for off in (0, 5):
        n = n_chunks * 8192 - 100 - off
        x = make("zipf", n, n_chunks + off)
        h = O.histogram(x)
        book, sizes = H.Codebook.from_histogram(h)
        bits, gaps = enc.encode(to_dev(x, off), book, sizes)
        bits_o, gaps_o, _ = O.encode(x, O.codebook(h))
        assert np.array_equal(u32(bits), bits_o) and np.array_equal(u32(gaps), gaps_o)


def test_compress_container_round_trip(cuda):
    x = make("zipf", 777_777, 9)
    c = H.compress(to_dev(x))
    blob = c.to_container()
    cb = O.codebook(O.histogram(x))
    bits_o, gaps_o, B = O.encode(x, cb)
    assert blob == O.container(cb, x.size, bits_o, gaps_o, (B + 127) // 128)
    back = H.Compressed.from_container(blob)
    assert np.array_equal(H.decompress(back).cpu().numpy(), x)


# ----------------------------------------------------------------- errors ---

def test_corrupt_gap_array_is_reported(cuda):
    x = make("uniform", 200_000, 4)
    h = O.histogram(x)
    book, sizes = H.Codebook.from_histogram(h)
    bits, gaps = H.Encoder(x.size).encode(to_dev(x), book, sizes)
    bad = gaps.clone()
    bad[10] ^= 0x1
    with pytest.raises(H.HgapError) as e:
        H.Decoder(sizes.segments).decode(bits, bad, sizes, book, x.size)
    assert e.value.status == 4  # HGAP_ERR_CORRUPT


def test_truncated_stream_is_reported(cuda):
    x = make("zipf", 100_000, 5)
    h = O.histogram(x)
    book, sizes = H.Codebook.from_histogram(h)
    bits, gaps = H.Encoder(x.size).encode(to_dev(x), book, sizes)
    with pytest.raises(H.HgapError) as e:
        H.Decoder(sizes.segments).decode(bits, gaps, sizes, book, x.size + 1000)
    assert e.value.status == 5  # HGAP_ERR_SIZE: fewer symbols than n


def test_byte_without_codeword_is_reported(cuda):
    x = make("two", 50_000, 6)          # symbols 0 and 1 only
    h = O.histogram(x)
    y = x.copy()
    y[-1] = 200                           # a byte the book has no codeword for
    book, _ = H.Codebook.from_histogram(h)
    bits_total = book.encoded_bits(O.histogram(y))
    sizes = H.StreamSizes.from_bits(bits_total)
    with pytest.raises(H.HgapError) as e:
        H.Encoder(y.size).encode(to_dev(y), book, sizes)
    assert e.value.status == 7  # HGAP_ERR_NO_CODE


def test_wrong_sizes_are_reported(cuda):
    x = make("zipf", 50_000, 7)
    book, sizes = H.Codebook.from_histogram(O.histogram(x))
    small = H.StreamSizes.from_bits(sizes.bits - 1000)
    with pytest.raises(H.HgapError) as e:
        H.Encoder(x.size).encode(to_dev(x), book, small,
                                 bits=torch.empty(sizes.words + 64, dtype=torch.int32, device="cuda"),
                                 gaps=torch.empty(sizes.gap_words + 8, dtype=torch.int32, device="cuda"))
    assert e.value.status == 5


# ------------------------------------------------- reference-signature entries

def test_histgram_compat(cuda):
    x = make("zipf", 123_457, 8)
    words = torch.zeros((x.size + 3) // 4 + 1, dtype=torch.int32, device="cuda")
    words.view(torch.uint8)[:x.size].copy_(torch.from_numpy(x))
    hist = torch.zeros(256, dtype=torch.int32, device="cuda")
    _lib.lib().histgram(hist.data_ptr(), words.data_ptr(), x.size)
    torch.cuda.synchronize()
    assert np.array_equal(u32(hist), O.histogram(x))


def _cudart():
    import ctypes.util
    path = ctypes.util.find_library("cudart") or "/usr/local/cuda/lib64/libcudart.so"
    rt = C.CDLL(path)
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return rt


def test_ref_encode_and_decode_compat(cuda):
    x = make("zipf", 300_001, 9)
    h = O.histogram(x)
    cb = O.codebook(h)
    bits_o, gaps_o, B = O.encode(x, cb)
    W, S, G = bits_o.size, (B + 127) // 128, gaps_o.size
    L = _lib.lib()
    # encode(out_host, W, d_in, n, S, codetable) takes ownership of d_in and
    # cudaFree()s it like the reference: hand it a plain cudaMalloc'd copy.
    rt = _cudart()
    d_in = C.c_void_p()
    assert rt.cudaMalloc(C.byref(d_in), x.size + 16) == 0
    assert rt.cudaMemcpy(d_in, x.ctypes.data, x.size, 1) == 0
    table = (_lib.Codeword * 256)()
    for b in range(256):
        table[b].code, table[b].length = int(cb.code[b]), int(cb.length[b])
    out = np.zeros(W + G, np.uint32)
    assert L.hgap_ref_encode(out.ctypes.data, W, d_in, x.size, S, table) == 0
    assert np.array_equal(out[:W], bits_o) and np.array_equal(out[W:], gaps_o)
    # decoder_l1_l2 with a reference-format LUT blob (get_twolevel_table layout)
    p, info, blob, _ = O.ref_table(cb, 10)
    inp = np.concatenate([gaps_o, bits_o]).astype(np.uint32)
    dec = np.zeros((x.size + 3) // 4, np.uint32)
    rc = L.hgap_ref_decoder_l1_l2(inp.ctypes.data, W, dec.ctypes.data, x.size, S,
                                  blob.ctypes.data, blob.size, p, cb.count, *info)
    assert rc == 0
    assert np.array_equal(dec.view(np.uint8)[:x.size], x)


# ------------------------------------------- encoder histogram pass + prepared

@pytest.mark.parametrize("n,off", [(1, 0), (1000, 3), (1 << 20, 0), (5 * (1 << 20) + 3, 9),
                                   (40 * (1 << 20) + 5, 1)])
def test_encode_histogram_then_prepared(cuda, n, off):
    x = make("zipf" if n % 2 else "uniform", n, n)
    d = to_dev(x, off)
    enc = H.Encoder(n)
    hist = enc.histogram(d)
    h = O.histogram(x)
    assert np.array_equal(u32(hist), h)
    book, sizes = H.Codebook.from_histogram(u32(hist))
    bits, gaps = enc.encode(d, book, sizes, prepared=True)
    bits_o, gaps_o, _ = O.encode(x, O.codebook(h))
    assert np.array_equal(u32(bits), bits_o) and np.array_equal(u32(gaps), gaps_o)


def test_prepared_with_foreign_workspace_is_rejected(cuda):
    x = make("zipf", 300_000, 1)
    y = make("zipf", 300_000, 2)
    enc = H.Encoder(x.size)
    dx, dy = to_dev(x), to_dev(y)
    enc.histogram(dx)
    book, sizes = H.Codebook.from_histogram(O.histogram(y))
    with pytest.raises(H.HgapError) as e:
        enc.encode(dy, book, sizes, prepared=True)   # histograms belong to x, not y
    assert e.value.status == 1  # HGAP_ERR_INVALID_ARG
