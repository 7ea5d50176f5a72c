"""libhgap.so without a GPU: it loads, exports every symbol include/hgap.h
declares, and its host half (codebook, container, argument checks) matches
the oracle and the reference's own host code."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import _lib
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "hgap.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b([A-Za-z_]\w*)\s*\(", text))
    return sorted(n for n in names if n.startswith("hgap_") or n == "histgram")


def test_every_declared_symbol_is_exported():
    L = _lib.lib()
    declared = _declared()
    assert len(declared) >= 15
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == declared


def test_status_strings():
    L = _lib.lib()
    for s in range(9):
        assert L.hgap_status_string(s)
    assert L.hgap_status_string(0) == b"ok"


def test_codebook_matches_oracle_and_reference():
    rng = np.random.default_rng(7)
    for it in range(500):
        h = rng.integers(0, 2000, size=256).astype(np.uint32)
        h[rng.random(256) < rng.random()] = 0
        if it % 7 == 0:
            h = np.zeros(256, np.uint32)
            f = [1, 1]
            while len(f) < 40:
                f.append(f[-1] + f[-2])
            h[rng.choice(256, 40, replace=False)] = f
        if (h > 0).sum() == 0:
            continue
        book, sizes = H.Codebook.from_histogram(h)
        cb = O.codebook(h)
        assert np.array_equal(book.symbols, cb.symbols)
        assert np.array_equal(book.lengths, cb.lengths)
        assert np.array_equal(book.code, cb.code) and np.array_equal(book.length, cb.length)
        assert sizes.bits == cb.total_bits
        if O.ref_available() and (h > 0).sum() >= 2:
            ref = O.ref_codebook(h)
            assert np.array_equal(book.lengths, ref.lengths) and np.array_equal(book.code, ref.code)


def test_single_symbol_book_is_defined():
    h = np.zeros(256, np.uint32)
    h[200] = 12345
    book, sizes = H.Codebook.from_histogram(h)
    assert book.symbol_count == 1 and book.length[200] == 1 and book.code[200] == 0
    assert (sizes.bits, sizes.words, sizes.segments) == (12345, 386, 97)


@pytest.mark.parametrize("syms,lens", [
    ([1, 2, 3], [2, 1, 2]),        # lengths not monotone
    ([1, 1], [1, 1]),              # duplicate symbol
    ([1, 2, 3], [1, 1, 1]),        # Kraft sum > 1
    ([1], [17]),                   # longer than 16 bits
])
def test_bad_symbol_lists_rejected(syms, lens):
    with pytest.raises(H.HgapError):
        H.Codebook.from_symbols(syms, lens)


def test_symbol_lists_accepted_exactly_when_valid():
    """Random container-order symbol lists: accepted exactly when the symbols
    are distinct, the lengths within 1..16 and non-decreasing, and the Kraft
    sum at most 1; an accepted book's codes are canonical (each code the
    previous one plus one, shifted to the next length) and prefix-free."""
    rng = np.random.default_rng(31)
    for it in range(1500):
        k = int(rng.integers(1, 40))
        syms = rng.choice(256, size=k, replace=bool(it % 7 == 0))
        lens = np.sort(rng.integers(1, 18, size=k)) if it % 5 else rng.integers(1, 17, size=k)
        valid = (len(set(syms.tolist())) == k and lens.min() >= 1 and lens.max() <= 16
                 and bool(np.all(np.diff(lens) >= 0)) and sum(2.0 ** -int(v) for v in lens) <= 1.0)
        if not valid:
            with pytest.raises(H.HgapError):
                H.Codebook.from_symbols(syms, lens)
            continue
        book = H.Codebook.from_symbols(syms, lens)
        assert book.symbol_count == k
        code = prev_len = None
        for sym, ln in zip(syms.tolist(), lens.tolist()):
            assert book.length[sym] == ln
            code = 0 if code is None else (code + 1) << (ln - prev_len)
            assert book.code[sym] == code
            prev_len = ln
        words = sorted(format(int(book.code[v]), f"0{int(book.length[v])}b") for v in syms.tolist())
        assert all(not b.startswith(a) for a, b in zip(words, words[1:]))


def test_container_write_matches_oracle_bytes():
    rng = np.random.default_rng(3)
    r = np.arange(1, 257); p = r ** -1.2; p /= p.sum()
    x = rng.choice(256, size=50_000, p=p).astype(np.uint8)
    h = O.histogram(x)
    cb = O.codebook(h)
    bits, gaps, B = O.encode(x, cb)
    S = (B + 127) // 128
    expect = O.container(cb, x.size, bits, gaps, S)
    book, sizes = H.Codebook.from_histogram(h)
    import torch
    c = H.Compressed(book, x.size, sizes, torch.from_numpy(bits.view(np.int32)),
                     torch.from_numpy(gaps.view(np.int32)))
    blob = c.to_container()
    assert blob == expect
    back = H.Compressed.from_container(blob, device="cpu")
    assert back.n == x.size
    assert (back.sizes.words, back.sizes.segments, back.sizes.gap_words) == (sizes.words, sizes.segments, sizes.gap_words)
    assert np.array_equal(back.book.symbols, book.symbols)
    assert np.array_equal(back.bits.numpy().view(np.uint32), bits)
    assert np.array_equal(back.gaps.numpy().view(np.uint32), gaps)


def test_container_parse_rejects_damage():
    x = np.frombuffer(b"hello gap arrays " * 40, np.uint8)
    cb = O.codebook(O.histogram(x))
    bits, gaps, B = O.encode(x, cb)
    blob = O.container(cb, x.size, bits, gaps, (B + 127) // 128)
    for cut in (0, 7, 20, len(blob) - 1):
        with pytest.raises(H.HgapError):
            H.Compressed.from_container(blob[:cut], device="cpu")
    bad = bytearray(blob)
    bad[0] = 0xFF  # symbol count > 256
    with pytest.raises(H.HgapError):
        H.Compressed.from_container(bytes(bad), device="cpu")


def test_argument_checks_need_no_gpu():
    L = _lib.lib()
    cb = _lib.CCodebook()
    # n == 0 with W == S == 0 is a no-op; anything else is a size error
    assert L.hgap_encode(None, 0, C.byref(cb), None, 0, None, 0, None, 0, None) == 0
    assert L.hgap_encode(None, 0, C.byref(cb), None, 1, None, 1, None, 0, None) == 5
    assert L.hgap_encode(None, 10, C.byref(cb), None, 1, None, 1, None, 0, None) == 1
    assert L.hgap_decode(None, 0, None, 0, C.byref(cb), None, 0, None, 0, None) == 0
    assert L.hgap_decode(None, 3, None, 1, C.byref(cb), None, 10, None, 0, None) == 1
    assert L.hgap_histogram(None, 10, None, None) == 1
    # workspace sizes grow with the input
    assert L.hgap_encode_workspace_bytes(1 << 30) > L.hgap_encode_workspace_bytes(1 << 20)
    assert L.hgap_decode_workspace_bytes(1 << 20) > L.hgap_decode_workspace_bytes(1 << 10)


def test_encoded_bits_is_64bit():
    h = np.zeros(256, np.uint32)
    h[:3] = [3_000_000_000, 2_900_000_000, 1_000_000_000]
    book, sizes = H.Codebook.from_histogram(h)
    assert sizes.bits == sum(int(book.length[b]) * int(h[b]) for b in range(3))


def test_batch_host_queries():
    """The batched path's host-side size queries (no GPU needed)."""
    import ctypes as C
    from huffman_coding_gap_arrays_b200._lib import BatchConfig, BatchEntry
    L = _lib.lib()
    assert C.sizeof(BatchEntry) == 576
    sizes = np.array([0, 1, 4096, 8192 * 8 + 1, 1 << 22], np.uint64)
    p = sizes.ctypes.data_as(C.POINTER(C.c_uint64))
    cfg = BatchConfig(8, 0, 0, 0)
    enc = L.hgap_batch_compress_workspace_bytes(sizes.size, p, C.byref(cfg))
    dec = L.hgap_batch_decompress_workspace_bytes(sizes.size, p)
    # regions: ceil((n + 15) / 64 KiB) per non-empty buffer
    regions = sum(int(-(-(int(n) + 15) // 65536)) for n in sizes if n)
    assert enc >= regions * (8 + 1024)
    assert dec >= sum(int(-(-int(n) // 2048)) for n in sizes) * 40
    cfg1 = BatchConfig(1, 0, 0, 0)
    assert L.hgap_batch_compress_workspace_bytes(sizes.size, p, C.byref(cfg1)) > enc
    # worst case 16 bits per byte, each bitstream rounded up to 16 bytes
    assert L.hgap_batch_bits_capacity(sizes.size, p) == sum(((int(n) * 16 + 31) // 32 + 3) & ~3 for n in sizes)
    assert L.hgap_batch_gaps_capacity(sizes.size, p) == sum(((int(n) * 16 + 127) // 128 + 7) // 8 for n in sizes)


def test_status_from_word():
    """A device status word read on the host maps to the status
    hgap_workspace_status returns: timeout above no-code above corrupt above
    size above plan (no GPU needed)."""
    L = _lib.lib()
    f = L.hgap_status_from_word
    assert f(0) == 0
    assert f(1) == 3 and f(2) == 4 and f(4) == 7 and f(8) == 5 and f(16) == 1
    assert f(2 | 8) == 4 and f(1 | 2 | 4 | 8) == 3 and f(4 | 8) == 7 and f(8 | 16) == 5
    assert f(1 << 20) == 0  # bits no kernel sets


def test_batch_decoder_class():
    """Decoder class from a symbol list on the host: 2 * stage + complete."""
    from huffman_coding_gap_arrays_b200._lib import SymLen
    L = _lib.lib()

    def cls(lengths):
        arr = (SymLen * max(len(lengths), 1))()
        for i, n in enumerate(lengths):
            arr[i].symbol, arr[i].length = i, n
        return L.hgap_batch_decoder_class(arr, len(lengths))

    assert cls([]) == 255
    assert cls([1, 1]) == 7            # complete, shortest code 1 bit
    assert cls([1]) == 6               # one symbol: Kraft sum 1/2
    assert cls([2, 2, 2, 2]) == 5
    assert cls([3, 3, 3, 3]) == 2      # incomplete (Kraft 1/2), 3 bits
    assert cls([4] * 16) == 1
    assert cls([8] * 256) == 1
    assert cls([5] * 8) == 0


def test_container_parse_survives_random_damage():
    """The container reader on thousands of damaged containers (bytes flipped,
    cut short, lengthened): it rejects them or accepts a consistent one, whose
    stream and gap pointers lie inside the buffer and whose book is valid --
    never a read past the buffer."""
    L = _lib.lib()
    rng = np.random.default_rng(21)
    blobs = []
    for n, dist in ((5000, "zipf"), (777, "few"), (1, "one")):
        if dist == "zipf":
            p = np.arange(1, 257, dtype=np.float64) ** -1.2
            x = rng.choice(256, size=n, p=p / p.sum()).astype(np.uint8)
        elif dist == "few":
            x = rng.integers(0, 5, n).astype(np.uint8)
        else:
            x = np.array([42], np.uint8)
        cb = O.codebook(O.histogram(x))
        bits, gaps, B = O.encode(x, cb)
        blobs.append(O.container(cb, x.size, bits, gaps, (B + 127) // 128))
    accepted = 0
    for it in range(3000):
        blob = bytearray(blobs[it % len(blobs)])
        kind = it % 3
        if kind == 0:
            for _ in range(int(rng.integers(1, 4))):
                blob[int(rng.integers(0, len(blob)))] ^= 1 << int(rng.integers(0, 8))
        elif kind == 1:
            blob = blob[:int(rng.integers(0, len(blob)))]
        else:
            blob += bytes(rng.integers(0, 256, int(rng.integers(1, 64))).astype(np.uint8))
        buf = (C.c_uint8 * max(len(blob), 1)).from_buffer_copy(bytes(blob) or b"\0")
        base = C.addressof(buf)
        cb = _lib.CCodebook()
        n, w, s = C.c_uint64(), C.c_uint64(), C.c_uint64()
        g, b = C.c_void_p(), C.c_void_p()
        st = L.hgap_container_parse(buf, len(blob), C.byref(cb), C.byref(n), C.byref(w), C.byref(s),
                                    C.byref(g), C.byref(b))
        if st != 0:
            continue
        accepted += 1
        assert 1 <= cb.symbol_count <= 256
        assert s.value == (w.value + 3) // 4
        gap_bytes = 4 * ((s.value + 7) // 8)
        assert base <= g.value and g.value + gap_bytes <= base + len(blob)
        assert base <= b.value and b.value + 4 * w.value <= base + len(blob)
        lens = [cb.symbols[i].length for i in range(cb.symbol_count)]
        assert all(1 <= v <= 16 for v in lens) and lens == sorted(lens)
        assert sum(2.0 ** -v for v in lens) <= 1.0
    assert accepted > 0  # flips inside the payload leave valid containers


def _table_lookup(t1, t2, v):
    """The decoder's two-level lookup of 16-bit windows v (MSB first): level 1
    on the top 11 bits; a pointer entry (bit 15: width << 12 | offset) reads
    level 2 at offset + the next `width` bits.  Returns (symbol, length,
    invalid) per window."""
    e = t1[v >> 5].astype(np.int64)
    ptr = (e & 0x8000) != 0
    w = (e >> 12) & 7
    idx = np.where(ptr, (e & 0xFFF) + ((v >> (5 - w)) & ((1 << w) - 1)), 0)
    e = np.where(ptr, t2[idx].astype(np.int64), e)
    return e & 0xFF, ((e >> 8) & 15) + 1, (e & 0x4000) != 0


def test_host_decode_table_decodes_every_window():
    """For books from random histograms (complete) and cut-down lists
    (incomplete), every 16-bit window decodes through the host-built table to
    the symbol whose code begins it, with that code's length -- and to an
    invalid entry where no code begins it."""
    L = _lib.lib()
    rng = np.random.default_rng(41)
    v = np.arange(1 << 16, dtype=np.int64)
    for it in range(120):
        h = np.zeros(256, np.uint32)
        k = int(rng.integers(2, 257))
        h[rng.choice(256, size=k, replace=False)] = (rng.pareto(0.6 + 1.5 * rng.random(), k) * 50 + 1).astype(np.uint32)
        book, _ = H.Codebook.from_histogram(h)
        syms, lens = book.symbols, book.lengths
        if it % 3 == 0 and len(syms) > 2:  # drop codes from the end: an incomplete book
            cut = int(rng.integers(1, len(syms) - 1))
            book = H.Codebook.from_symbols(syms[:-cut], lens[:-cut])
            syms, lens = syms[:-cut], lens[:-cut]
        t1 = np.zeros(2048, np.uint16)
        t2 = np.zeros(2560, np.uint16)
        assert L.hgap_decode_table_build(C.byref(book.cstruct), t1.ctypes.data, t2.ctypes.data) == 0
        codes = np.array([int(book.code[s]) for s in syms], np.int64)
        la = codes << (16 - lens.astype(np.int64))  # left-aligned, ascending in container order
        i = np.searchsorted(la, v, side="right") - 1
        inside = (i >= 0) & (v - la[np.maximum(i, 0)] < (1 << (16 - lens[np.maximum(i, 0)].astype(np.int64))))
        sym, ln, bad = _table_lookup(t1, t2, v)
        assert np.array_equal(bad, ~inside)
        assert np.array_equal(sym[inside], syms[i[inside]].astype(np.int64))
        assert np.array_equal(ln[inside], lens[i[inside]].astype(np.int64))
