"""Batched path and device codebooks on the GPU, through the C ABI.

Every batched stream must equal the single-buffer path's stream for the same
buffer (itself pinned to the oracle and the reference's GPU encoder), and
every device-built codebook and decoder table must equal the host builder's.
"""
import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import HgapError
from huffman_coding_gap_arrays_b200 import batch as B
from huffman_coding_gap_arrays_b200 import workloads as WL
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _hists(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        k = i % 8
        if k == 0:   # Fibonacci counts: lengths hit the 16-bit limit
            h = np.zeros(256, np.uint32)
            f = [1, 1]
            while len(f) < 40:
                f.append(f[-1] + f[-2])
            h[rng.choice(256, 40, replace=False)] = np.array(f, np.uint64).astype(np.uint32)
        elif k == 1:  # one symbol
            h = np.zeros(256, np.uint32)
            h[rng.integers(256)] = rng.integers(1, 10**6)
        elif k == 2:  # two symbols
            h = np.zeros(256, np.uint32)
            h[rng.choice(256, 2, replace=False)] = rng.integers(1, 1000, 2)
        elif k == 3:  # all equal: ties everywhere
            h = np.full(256, rng.integers(1, 100), np.uint32)
        elif k == 4:  # Zipf counts
            s = rng.uniform(0.8, 1.6)
            h = (1e7 * np.arange(1, 257, dtype=np.float64) ** -s).astype(np.uint32)
            rng.shuffle(h)
        elif k == 5:  # sparse random with repeated counts
            h = rng.integers(0, 5, 256).astype(np.uint32)
        elif k == 6:  # empty
            h = np.zeros(256, np.uint32)
        else:
            h = rng.integers(0, 2**31, 256).astype(np.uint32)
            h[rng.random(256) < rng.random()] = 0
        out.append(h)
    return np.stack(out)


def test_device_codebooks_match_host():
    hs = _hists(1200, 11)
    books, sizes = B.device_codebooks(torch.from_numpy(hs.view(np.int32)).cuda())
    for h, b, z in zip(hs, books, sizes):
        if (h > 0).sum() == 0:
            assert b.symbol_count == 0 and z.bits == 0
            continue
        hb, hz = H.Codebook.from_histogram(h)
        assert np.array_equal(b.symbols, hb.symbols)
        assert np.array_equal(b.lengths, hb.lengths)
        assert np.array_equal(b.code, hb.code) and np.array_equal(b.length, hb.length)
        assert (z.bits, z.words, z.segments, z.gap_words) == (hz.bits, hz.words, hz.segments, hz.gap_words)


def test_device_decode_tables_match_host():
    hs = [h for h in _hists(400, 12) if (h > 0).sum() > 0]
    books = [H.Codebook.from_histogram(h)[0] for h in hs]
    t, st = B.device_decode_tables(books)
    assert int(st.abs().sum()) == 0
    for i, b in enumerate(books):
        assert np.array_equal(t[i].numpy().view(np.uint16), B.host_decode_table(b)), i


def _make_buffers(sizes, seed, device="cuda"):
    bufs = []
    for i, n in enumerate(sizes):
        x = WL.batch_buffer(max(n, 1), seed * 100003 + i, device=device)[:n] if n else \
            torch.empty(0, dtype=torch.uint8, device=device)
        bufs.append(x)
    return bufs


def _packed(bufs, offset=3):
    """The same buffers packed back to back (unaligned) in one allocation."""
    total = sum(b.numel() for b in bufs) + offset + 16
    flat = torch.zeros(total, dtype=torch.uint8, device=bufs[0].device if bufs else "cuda")
    views, p = [], offset
    for b in bufs:
        v = flat[p:p + b.numel()]
        v.copy_(b)
        views.append(v)
        p += b.numel()
    return flat, views


SIZES = [0, 1, 2, 15, 16, 17, 255, 4095, 4096, 8191, 8192, 8193, 65537, 300001, (1 << 20) + 3]


def _roundtrip(sizes, cfg=None, packed=True, region=None, seed=5):
    bufs = _make_buffers(sizes, seed)
    keep = None
    if packed:
        keep, ins = _packed(bufs)
    else:
        ins = bufs
    outs = [torch.full((max(n, 1),), 0xA5, dtype=torch.uint8, device="cuda") for n in sizes]
    plan = B.BatchCodec(sizes, cfg, region_chunks=region)
    plan.bind(ins, outs)
    plan.compress()
    plan.check_compress()
    plan.decompress()
    plan.check_decompress()
    ents = plan.entries_host()
    for i, (x, e) in enumerate(zip(bufs, ents)):
        n = sizes[i]
        assert e.n == n and e.status == 0
        assert torch.equal(outs[i][:n], x), f"buffer {i} (n={n}) round trip"
        if n == 0:
            assert e.words == 0 and e.symbol_count == 0
            continue
        ref = H.compress(x)
        got = plan.stream(i, e)
        assert np.array_equal(got.book.symbols, ref.book.symbols)
        assert np.array_equal(got.book.lengths, ref.book.lengths)
        assert got.sizes.words == ref.sizes.words and got.sizes.segments == ref.sizes.segments
        assert torch.equal(got.bits, ref.bits), f"buffer {i} (n={n}) bitstream"
        assert torch.equal(got.gaps, ref.gaps), f"buffer {i} (n={n}) gap array"
        assert e.bits_offset % 4 == 0
    return plan, bufs, ins, outs, keep


def test_batch_matches_single_path_packed():
    _roundtrip(SIZES)


def test_batch_matches_single_path_separate():
    _roundtrip(SIZES, packed=False, seed=6)


def test_batch_small_buffers_match_oracle():
    sizes = [1, 7, 100, 4096 + 5, 20000]
    plan, bufs, *_ = _roundtrip(sizes, seed=9)
    for i, (x, e) in enumerate(zip(bufs, plan.entries_host())):
        xs = x.cpu().numpy()
        cb = O.codebook(np.bincount(xs, minlength=256).astype(np.uint32))
        bits, gaps, _ = O.encode(xs, cb)
        got = plan.stream(i, e)
        assert np.array_equal(got.bits.cpu().numpy().view(np.uint32), bits)
        assert np.array_equal(got.gaps.cpu().numpy().view(np.uint32), gaps)


@pytest.mark.parametrize("cfg", [B.LaunchConfig(region_chunks=1), B.LaunchConfig(region_chunks=32),
                                 B.LaunchConfig(region_chunks=2, hist_ctas_per_sm=1, enc_ctas_per_sm=1,
                                                dec_ctas_per_sm=1),
                                 B.LaunchConfig(dec_tile_segs=256), B.LaunchConfig(dec_tile_segs=512),
                                 B.LaunchConfig(dec_ctas_per_sm=2, dec_tile_segs=512)])
def test_batch_launch_configs_same_output(cfg):
    _roundtrip(SIZES[3:], cfg, seed=7)


def test_batch_per_buffer_region_sizes():
    sizes = SIZES[1:]
    rng = np.random.default_rng(3)
    _roundtrip(sizes, B.LaunchConfig(region_chunks=1), region=rng.integers(1, 33, len(sizes)), seed=8)


def test_batch_log_uniform_mix():
    sizes = WL.batch_sizes(96, hi=2 << 20, seed=21)
    _roundtrip(sizes, seed=22)


def test_batch_graph_replay_follows_new_input():
    sizes = [5000, 70000, 123457, 1 << 20]
    bufs = _make_buffers(sizes, 31)
    ins = [b.clone() for b in bufs]
    outs = [torch.empty(n, dtype=torch.uint8, device="cuda") for n in sizes]
    plan = B.BatchCodec(sizes)
    plan.bind(ins, outs)
    plan.compress()
    plan.decompress()
    plan.check()
    g = plan.capture()
    for rep in range(2):
        new = _make_buffers(sizes, 40 + rep)
        for a, b in zip(ins, new):
            a.copy_(b)
        for o in outs:
            o.zero_()
        g.replay()
        torch.cuda.synchronize()
        plan.check()
        for i, (o, x) in enumerate(zip(outs, new)):
            assert torch.equal(o, x), (rep, i)
            ref = H.compress(x)
            got = plan.stream(i)
            assert torch.equal(got.bits, ref.bits) and torch.equal(got.gaps, ref.gaps)


def test_batch_container_matches_single_path():
    sizes = [3000, 50000]
    plan, bufs, *_ = _roundtrip(sizes, seed=12)
    for i, x in enumerate(bufs):
        assert plan.container(i) == H.compress(x).to_container()


def test_batch_arena_too_small_is_reported():
    sizes = [100000, 200000]
    bufs = _make_buffers(sizes, 50)
    outs = [torch.empty(n, dtype=torch.uint8, device="cuda") for n in sizes]
    plan = B.BatchCodec(sizes)
    plan.bits_capacity = 100  # words: far too few
    plan.bind(bufs, outs)
    plan.compress()
    with pytest.raises(HgapError) as ei:
        plan.check_compress()
    assert ei.value.status == 5  # HGAP_ERR_SIZE
    ents = plan.entries_host()
    assert ents[0].status == 5 or ents[1].status == 5


def test_batch_corrupt_entry_is_reported():
    sizes = [40000, 40000]
    bufs = _make_buffers(sizes, 60)
    outs = [torch.empty(n, dtype=torch.uint8, device="cuda") for n in sizes]
    plan = B.BatchCodec(sizes)
    plan.bind(bufs, outs)
    plan.compress()
    plan.check_compress()
    raw = plan.entries.view(len(sizes), -1)
    # buffer 1: a length of 17 is not a valid code length
    sym0_len = 7 * 8 + 8 + 1  # offset of symbols[0].length
    raw[1, sym0_len] = 17
    plan.decompress()
    with pytest.raises(HgapError) as ei:
        plan.check_decompress()
    assert ei.value.status == 4  # HGAP_ERR_CORRUPT
    assert torch.equal(outs[0], bufs[0])  # the healthy buffer still decodes


def test_batch_class_mask_launches_only_named_classes():
    """dec_class_mask from the host copies of the entries decodes exactly; a
    mask that leaves out a class in use is reported (HGAP_ERR_INVALID_ARG) and
    the buffers of the classes it names still decode."""
    sizes = [70000, 50000, 30000, 90000, 4096, 0]
    bufs = _make_buffers(sizes, 61)
    # a 1-bit shortest code (class 6/7) beside the mixed generator's books
    bufs[2] = torch.from_numpy(np.where(np.random.default_rng(1).random(30000) < 0.8, 7, 9)
                               .astype(np.uint8)).cuda()
    outs = [torch.full((max(n, 1),), 0xA5, dtype=torch.uint8, device="cuda") for n in sizes]
    plan = B.BatchCodec(sizes)
    plan.bind(bufs, outs)
    plan.compress()
    plan.check_compress()
    ents = plan.entries_host()
    mask = B.decoder_class_mask(ents)
    assert mask >> 6 & 3  # the two-symbol buffer's class
    plan.config = B.LaunchConfig(dec_class_mask=mask)
    plan.decompress()
    plan.check_decompress()
    for x, o, n in zip(bufs, outs, sizes):
        assert torch.equal(o[:n], x)
    c2 = 1 << (mask.bit_length() - 1)  # leave out the highest class in use
    for o in outs:
        o.fill_(0xA5)
    plan.config = B.LaunchConfig(dec_class_mask=mask & ~c2)
    plan.decompress()
    with pytest.raises(HgapError) as ei:
        plan.check_decompress()
    assert ei.value.status == 1  # HGAP_ERR_INVALID_ARG
    lib = B.lib()
    for x, o, n, e in zip(bufs, outs, sizes, ents):
        if n and not (1 << lib.hgap_batch_decoder_class(e.symbols, e.symbol_count)) & c2:
            assert torch.equal(o[:n], x)


def test_batch_bf16_planes():
    exp, sm = WL.bf16_planes(1 << 20, seed=3)
    sizes = [exp.numel(), sm.numel()]
    outs = [torch.empty(n, dtype=torch.uint8, device="cuda") for n in sizes]
    plan = B.BatchCodec(sizes)
    plan.bind([exp, sm], outs)
    plan.compress()
    plan.decompress()
    plan.check()
    assert torch.equal(outs[0], exp) and torch.equal(outs[1], sm)
    for i, x in enumerate((exp, sm)):
        ref = H.compress(x)
        got = plan.stream(i)
        assert torch.equal(got.bits, ref.bits) and torch.equal(got.gaps, ref.gaps)


def test_batch_features_match_per_buffer_host_books():
    """tuner.batch_features (device histograms and codebooks, vectorised)
    equals the per-buffer statistics from host codebooks."""
    import math
    from huffman_coding_gap_arrays_b200 import tuner as TU
    sizes = [0, 1, 300, 4096, 70000, 1 << 20]
    bufs = _make_buffers(sizes, 62)
    bufs[2] = torch.full((300,), 7, dtype=torch.uint8, device="cuda")  # one symbol
    f = TU.batch_features(bufs)
    acc, total = np.zeros(3), sum(sizes)
    for x in bufs:
        if x.numel() == 0:
            continue
        h = H.histogram(x).cpu().numpy().view(np.uint32)
        book, _ = H.Codebook.from_histogram(h)
        acc += x.numel() * TU.features_from_hist(x.numel(), h, book.length)[1:]
    want = np.concatenate([[math.log2(total)], acc / total, [math.log2(len(sizes))]])
    assert np.allclose(f, want, rtol=1e-5, atol=1e-6), (f, want)
