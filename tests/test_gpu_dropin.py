"""Drop-in check: the reference's own bin/encoder and bin/decoder mains
(encoder/src/huff.cpp, decoder/src/huff.cpp and their host helpers, compiled
unmodified by oracle/Makefile `dropin`) linked against libhgap.so instead of
encoder.cu / decoder.cu.  The container they write must equal the oracle's,
and the decoder main must restore the input."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
ENC = os.path.join(REF, "encoder_on_hgap")
DEC = os.path.join(REF, "decoder_on_hgap")


@pytest.mark.skipif(not (os.path.exists(ENC) and os.path.exists(DEC)),
                    reason="reference mains not built (oracle/Makefile dropin)")
@pytest.mark.parametrize("n", [4097, 1 << 20, 5 * (1 << 20) + 1])
def test_reference_mains_on_hgap(cuda, tmp_path, n):
    rng = np.random.default_rng(n)
    r = np.arange(1, 257); p = r ** -1.1; p /= p.sum()
    x = rng.choice(256, size=n, p=p).astype(np.uint8)
    src = tmp_path / "input.bin"
    src.write_bytes(x.tobytes())
    enc = tmp_path / "input.hgap"
    out = subprocess.run([ENC, str(src), str(enc)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    cb = O.codebook(O.histogram(x))
    bits, gaps, B = O.encode(x, cb)
    assert enc.read_bytes() == O.container(cb, n, bits, gaps, (B + 127) // 128)
    out = subprocess.run([DEC, str(enc), "ignored"], capture_output=True, text=True, timeout=120,
                         cwd=tmp_path)
    assert out.returncode == 0, out.stdout + out.stderr
    assert (tmp_path / "decodedfile").read_bytes() == x.tobytes()
