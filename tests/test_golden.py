"""Golden fixtures written by the REFERENCE's own GPU encoder
(encoder/src/encoder.cu histgram() + encode(), compiled unmodified into
oracle/_ref and run on a B200 by tests/golden/make_golden.py).

CPU: the oracle reproduces every fixture (histogram, bitstream, gap array,
container bytes) -- this pins the oracle's encoder half to the reference.
GPU: libhgap.so reproduces them through its C ABI."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)
from make_golden import make  # noqa: E402

MANIFEST = json.load(open(os.path.join(HERE, "golden.json")))
CASES = MANIFEST["cases"]
IDS = [c["name"] for c in CASES]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_oracle_reproduces_reference_gpu_encoder(case):
    x = make(case["dist"], case["n"], case["seed"])
    h = O.histogram(x)
    assert sha(h) == case["sha_hist"]
    cb = O.codebook(h)
    assert cb.count == case["symbols"] and int(cb.lengths.max()) == case["max_len"]
    bits, gaps, B = O.encode(x, cb)
    assert (B, bits.size) == (case["bits"], case["words"])
    assert sha(bits) == case["sha_bits"]
    assert sha(gaps) == case["sha_gaps"]
    if "container" in case:
        blob = O.container(cb, x.size, bits, gaps, case["segments"])
        ref = open(os.path.join(HERE, case["container"]), "rb").read()
        assert blob == ref
        assert O.decode(bits, gaps, case["segments"], cb, x.size).tobytes() == x.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_kernels_reproduce_reference_gpu_encoder(cuda, case):
    import torch
    import huffman_coding_gap_arrays_b200 as H
    x = make(case["dist"], case["n"], case["seed"])
    d = torch.from_numpy(x).to(cuda)
    hist = H.histogram(d)
    hh = hist.cpu().numpy().view(np.uint32)
    assert sha(hh) == case["sha_hist"]
    book, sizes = H.Codebook.from_histogram(hh)
    bits, gaps = H.Encoder(x.size).encode(d, book, sizes)
    assert sha(bits.cpu().numpy().view(np.uint32)) == case["sha_bits"]
    assert sha(gaps.cpu().numpy().view(np.uint32)) == case["sha_gaps"]
    c = H.Compressed(book, x.size, sizes, bits, gaps)
    if "container" in case:
        assert c.to_container() == open(os.path.join(HERE, case["container"]), "rb").read()
    assert torch.equal(H.decompress(c), d)
