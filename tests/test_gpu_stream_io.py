"""Streaming container I/O on the GPU: file-to-file compress and decompress
through the pipelined batched path; every container file must be the one the
single-buffer path writes for that file alone, and decode back exactly."""
import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import stream_io as SIO
from huffman_coding_gap_arrays_b200 import workloads as WL
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 1000, 70000, 3 << 20, 300005, 65536, 1 << 20, 5, 2 << 20]


def _files(tmp_path, sizes, seed):
    paths, data = [], []
    for i, n in enumerate(sizes):
        x = WL.batch_buffer(max(n, 1), seed + i, device="cpu").numpy()[:n]
        p = tmp_path / f"in{i}.bin"
        x.tofile(p)
        paths.append(str(p))
        data.append(x)
    return paths, data


@pytest.mark.parametrize("group_bytes", [1 << 20, 64 << 20])
def test_files_round_trip_and_match_single_path(tmp_path, group_bytes):
    ins, data = _files(tmp_path, SIZES, 40)
    cont = [str(tmp_path / f"c{i}.hgap") for i in range(len(ins))]
    outs = [str(tmp_path / f"out{i}.bin") for i in range(len(ins))]
    st = SIO.compress_files(ins, cont, group_bytes=group_bytes)
    assert st["files"] == len(ins) and st["bytes_in"] == sum(SIZES)
    for x, c in zip(data, cont):
        got = open(c, "rb").read()
        ref = H.compress(torch.from_numpy(x.copy()).cuda()).to_container() if x.size else \
            H.compress(torch.empty(0, dtype=torch.uint8, device="cuda")).to_container()
        assert got == ref
    st = SIO.decompress_files(cont, outs, group_bytes=group_bytes)
    assert st["bytes_out"] == sum(SIZES)
    for x, o in zip(data, outs):
        assert np.array_equal(np.fromfile(o, np.uint8), x)


def test_container_matches_oracle(tmp_path):
    ins, data = _files(tmp_path, [5000, 123457], 90)
    cont = [str(tmp_path / f"c{i}.hgap") for i in range(len(ins))]
    SIO.compress_files(ins, cont)
    for x, c in zip(data, cont):
        cb = O.codebook(O.histogram(x))
        bits, gaps, total = O.encode(x, cb)
        assert open(c, "rb").read() == O.container(cb, x.size, bits, gaps, (total + 127) // 128)
