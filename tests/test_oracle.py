"""The CPU oracle, pinned against the reference's own host sources
(oracle/_ref: store_symbols + qsort(compare) + boundary_PM from
encoder/src/*.cpp, get_table_info + get_twolevel_table from
decoder/src/get_table.cpp), plus its own round-trip properties."""
import numpy as np
import pytest

from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (reference absent)")


def _hists(seed, count):
    rng = np.random.default_rng(seed)
    for it in range(count):
        k = int(rng.integers(2, 257))
        h = np.zeros(256, np.uint64)
        idx = rng.choice(256, size=k, replace=False)
        mode = it % 6
        if mode == 0:
            v = rng.integers(1, 10, size=k)            # heavy ties
        elif mode == 1:
            v = rng.integers(1, 1_000_000, size=k)
        elif mode == 2:
            v = (2.0 ** rng.uniform(0, 30, size=k)).astype(np.int64) + 1
        elif mode == 3:
            f = [1, 1]
            while len(f) < k:
                f.append(f[-1] + f[-2])
            v = np.minimum(np.array(f[:k], dtype=object), 2 ** 24).astype(np.int64)
        elif mode == 4:
            v = np.full(k, rng.integers(1, 100))
        else:
            v = rng.zipf(1.3, size=k).astype(np.int64)
        h[idx] = np.minimum(v, 2 ** 26)
        yield h.astype(np.uint32)


@needs_ref
def test_codebook_matches_reference_boundary_pm():
    n16 = 0
    for h in _hists(11, 3000):
        mine = O.codebook(h)
        ref = O.ref_codebook(h)
        assert np.array_equal(mine.symbols, ref.symbols)
        assert np.array_equal(mine.lengths, ref.lengths)
        assert np.array_equal(mine.code, ref.code)
        assert np.array_equal(mine.length, ref.length)
        assert mine.total_bits == ref.total_bits
        n16 += int(mine.lengths.max() == 16)
    assert n16 > 100  # the 16-bit length limit is exercised


@needs_ref
def test_reference_output_size_overflows_in_u32():
    # get_outputfilesize multiplies u8 length by u32 count in 32 bits
    # (encoder/src/symbols.cpp:52); the oracle keeps 64 bits.
    h = np.zeros(256, np.uint32)
    h[:3] = [3_000_000_000, 2_900_000_000, 1_000_000_000]
    ref = O.ref_codebook(h)
    mine = O.codebook(h)
    assert np.array_equal(mine.lengths, ref.lengths)
    exact = sum(int(mine.length[b]) * int(h[b]) for b in range(256))
    assert mine.total_bits == exact and ref.total_bits != exact


def test_single_and_empty_books():
    h = np.zeros(256, np.uint32)
    assert O.codebook(h).count == 0
    h[42] = 1000
    cb = O.codebook(h)
    assert cb.count == 1 and cb.length[42] == 1 and cb.code[42] == 0


@needs_ref
@pytest.mark.parametrize("prefix", [8, 10, 12])
def test_twolevel_table_matches_reference_where_boundary_is_right(prefix):
    checked = buggy = 0
    for h in _hists(5, 600):
        cb = O.codebook(h)
        p_ref, info_ref, blob_ref, boundary_ref = O.ref_twolevel_table(cb, prefix)
        p, info, blob, boundary = O.ref_table(cb, prefix)
        p_bug, info_bug, _, _ = O.ref_table(cb, prefix, reference_bug=True)
        assert (p_bug, info_bug) == (p_ref, info_ref)          # get_table_info restated exactly
        assert boundary == boundary_ref                        # get_twolevel_table's own boundary
        if info_ref == info and blob_ref is not None:
            assert np.array_equal(blob, blob_ref)              # byte-identical table
            checked += 1
        if info_ref[0] != info[0]:
            buggy += 1                                         # get_table.cpp:20 off-by-one-code
    assert checked > 100


def test_reference_table_bug_on_exponent_plane_shape():
    # A book shaped like the BF16 exponent plane (few symbols, lengths up to 16):
    # get_table_info's l1 boundary comes from the *next* code (get_table.cpp:20).
    lens = np.array([1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 16], np.uint8)
    cb = O.codebook_from_list(np.arange(17, dtype=np.uint8), lens)
    _, info_bug, _, _ = O.ref_table(cb, 10, reference_bug=True)
    _, info, _, boundary = O.ref_table(cb, 10)
    assert info_bug[0] != boundary and info[0] == boundary


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 31, 32, 33, 127, 128, 129, 1000, 4096, 65537])
@pytest.mark.parametrize("dist", ["zipf", "uniform", "two"])
def test_oracle_round_trip(n, dist):
    rng = np.random.default_rng(n)
    if dist == "zipf":
        r = np.arange(1, 257); p = r ** -1.2; p /= p.sum()
        x = rng.choice(256, size=n, p=p).astype(np.uint8)
    elif dist == "uniform":
        x = rng.integers(0, 256, size=n).astype(np.uint8)
    else:
        x = rng.integers(0, 2, size=n).astype(np.uint8)
    cb = O.codebook(O.histogram(x))
    bits, gaps, B = O.encode(x, cb)
    _, W, S, G = O.lib().orc_sizes_from_bits(B).bits, bits.size, (B + 127) // 128, gaps.size
    assert np.array_equal(O.decode(bits, gaps, S, cb, n), x)
    assert np.array_equal(O.decode_mt(bits, gaps, S, cb, n, 4), x)
    b2, g2 = O.encode_mt(x, cb, B, 4)
    assert np.array_equal(b2, bits) and np.array_equal(g2, gaps)


def test_gap_entries_follow_reference_semantics():
    # 3 symbols with codes 0, 10, 11: bit layout is easy to follow by hand
    x = np.array([0, 1, 2] * 100, np.uint8)
    cb = O.codebook_from_list(np.array([0, 1, 2], np.uint8), np.array([1, 2, 2], np.uint8))
    bits, gaps, B = O.encode(x, cb)
    assert B == 500
    stream = "".join(format(int(w), "032b") for w in bits)[:B]
    assert stream.startswith("01011" * 3)
    # gap[k] = end of the code that crosses/ends at 128(k+1), minus 128(k+1)
    ends, pos = [], 0
    for s in x:
        pos += 1 if s == 0 else 2
        ends.append(pos)
    for k in range((B + 127) // 128 - 1):
        b = 128 * (k + 1)
        e = min(e for e in ends if e >= b)
        assert (int(gaps[k // 8]) >> (4 * (k % 8))) & 15 == e - b


def test_corrupt_gap_is_detected():
    rng = np.random.default_rng(1)
    x = rng.integers(0, 256, size=4000).astype(np.uint8)
    cb = O.codebook(O.histogram(x))
    bits, gaps, B = O.encode(x, cb)
    S = (B + 127) // 128
    bad = gaps.copy()
    bad[0] ^= 0x3
    with pytest.raises(ValueError):
        O.decode(bits, bad, S, cb, x.size)


def test_container_layout():
    x = np.frombuffer(b"abracadabra" * 50, np.uint8)
    cb = O.codebook(O.histogram(x))
    bits, gaps, B = O.encode(x, cb)
    S = (B + 127) // 128
    blob = O.container(cb, x.size, bits, gaps, S)
    assert int.from_bytes(blob[:8], "little") == cb.count
    off = 8 + 2 * cb.count
    n, W, S2 = np.frombuffer(blob[off:off + 12], np.uint32)
    assert (n, W, S2) == (x.size, bits.size, S)
    assert blob[off + 12:off + 12 + 4 * gaps.size] == gaps.tobytes()
    assert blob[-4 * bits.size:] == bits.tobytes()
