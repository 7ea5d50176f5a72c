"""The bounded look-back waits, made to run out on purpose without any GPU
fault: one work item withholds its look-back records (hgap_encode_hold /
hgap_decode_hold) and every wait is limited to a few milliseconds.  The
kernels must finish by themselves, report HGAP_ERR_TIMEOUT through the
workspace status, keep every write inside the output buffers, and leave the
workspace usable for the next ordinary call.  Also: a corrupt stream is
reported as corrupt, never as a timeout, whatever the timing."""
import ctypes as C
import time

import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HGAP_ERR_TIMEOUT = 3
HGAP_ERR_CORRUPT = 4
LIMIT_NS = 2_000_000  # 2 ms per wait
GUARD = 4096


def zipf(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    r = np.arange(1, 257)
    p = r ** -1.2
    p /= p.sum()
    return rng.choice(256, size=n, p=p).astype(np.uint8)


def stream_ptr():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("hold", [1, 5])
def test_decoder_wait_runs_out_and_workspace_recovers(cuda, hold):
    x = zipf((1 << 20) + 5, 11 + hold)
    book, sizes = H.Codebook.from_histogram(O.histogram(x))
    d = torch.from_numpy(x).cuda()
    bits, gaps = H.Encoder(x.size).encode(d, book, sizes)
    dec = H.Decoder(sizes.segments)
    ws = dec.workspace
    buf = torch.full((x.size + 2 * GUARD,), 0x5A, dtype=torch.uint8, device="cuda")
    out = buf[GUARD:GUARD + x.size]
    L = _lib.lib()
    t0 = time.perf_counter()
    rc = L.hgap_decode_hold(bits.data_ptr(), sizes.words, gaps.data_ptr(), sizes.segments,
                            C.byref(book.cstruct), out.data_ptr(), x.size, ws.data_ptr(), ws.numel() * 8,
                            stream_ptr(), hold, LIMIT_NS)
    assert rc == 0
    st = L.hgap_workspace_status(ws.data_ptr(), stream_ptr())
    elapsed = time.perf_counter() - t0
    assert st == HGAP_ERR_TIMEOUT
    assert elapsed < 10.0
    g = buf.cpu().numpy()
    assert (g[:GUARD] == 0x5A).all() and (g[GUARD + x.size:] == 0x5A).all()
    # the same workspace and output, an ordinary call: exact again
    y = dec.decode(bits, gaps, sizes, book, x.size, out=out)
    assert np.array_equal(y.cpu().numpy(), x)


@pytest.mark.parametrize("hold", [1, 7])
def test_encoder_wait_runs_out_and_workspace_recovers(cuda, hold):
    x = zipf((1 << 20) + 3, 21 + hold)
    h = O.histogram(x)
    book, sizes = H.Codebook.from_histogram(h)
    d = torch.from_numpy(x).cuda()
    enc = H.Encoder(x.size)
    ws = enc.workspace
    bbuf = torch.full((sizes.words + 2 * GUARD,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
    gbuf = torch.full((sizes.gap_words + 2 * GUARD,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
    L = _lib.lib()
    rc = L.hgap_encode_hold(d.data_ptr(), x.size, C.byref(book.cstruct), bbuf[GUARD:].data_ptr(), sizes.words,
                            gbuf[GUARD:].data_ptr(), sizes.segments, ws.data_ptr(), ws.numel() * 8,
                            stream_ptr(), hold, LIMIT_NS)
    assert rc == 0
    assert L.hgap_workspace_status(ws.data_ptr(), stream_ptr()) == HGAP_ERR_TIMEOUT
    b = bbuf.cpu().numpy().view(np.uint32)
    g = gbuf.cpu().numpy().view(np.uint32)
    assert (b[:GUARD] == 0x5A5A5A5A).all() and (b[GUARD + sizes.words:] == 0x5A5A5A5A).all()
    assert (g[:GUARD] == 0x5A5A5A5A).all() and (g[GUARD + sizes.gap_words:] == 0x5A5A5A5A).all()
    bits, gaps = enc.encode(d, book, sizes, bits=bbuf[GUARD:GUARD + sizes.words],
                            gaps=gbuf[GUARD:GUARD + sizes.gap_words])
    bits_o, gaps_o, _ = O.encode(x, O.codebook(h))
    assert np.array_equal(bits.cpu().numpy().view(np.uint32), bits_o)
    assert np.array_equal(gaps.cpu().numpy().view(np.uint32), gaps_o)


def test_hold_nothing_is_the_ordinary_call(cuda):
    x = zipf(300_001, 5)
    book, sizes = H.Codebook.from_histogram(O.histogram(x))
    d = torch.from_numpy(x).cuda()
    bits, gaps = H.Encoder(x.size).encode(d, book, sizes)
    dec = H.Decoder(sizes.segments)
    out = torch.empty(x.size, dtype=torch.uint8, device="cuda")
    L = _lib.lib()
    rc = L.hgap_decode_hold(bits.data_ptr(), sizes.words, gaps.data_ptr(), sizes.segments,
                            C.byref(book.cstruct), out.data_ptr(), x.size, dec.workspace.data_ptr(),
                            dec.workspace.numel() * 8, stream_ptr(), (1 << 64) - 1, LIMIT_NS)
    assert rc == 0
    assert L.hgap_workspace_status(dec.workspace.data_ptr(), stream_ptr()) == 0
    assert torch.equal(out, d)


def test_corrupt_large_stream_is_corrupt_not_timeout(cuda):
    """An early corrupt gap entry in a stream of many tiles: the tiles still
    waiting on look-back records give up without claiming a timeout."""
    n = 80 << 20
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    d = torch.randint(0, 256, (n,), dtype=torch.uint8, device="cuda", generator=g)
    h = H.histogram(d).cpu()
    book, sizes = H.Codebook.from_histogram(h)
    bits, gaps = H.Encoder(n).encode(d, book, sizes)
    dec = H.Decoder(sizes.segments)
    for word in (3, 1000):
        bad = gaps.clone()
        bad[word] ^= 0x10
        with pytest.raises(H.HgapError) as e:
            dec.decode(bits, bad, sizes, book, n)
        assert e.value.status == HGAP_ERR_CORRUPT
    y = dec.decode(bits, gaps, sizes, book, n)
    assert torch.equal(y, d)
