"""The batched size queries without a GPU: the properties the serving loop's
admission bound rests on.  The server charges each request its own share of a
batch's workspace and arenas (the query for that one buffer minus the empty
batch's) plus one fixed part per batch, so the queries must be subadditive
over buffers, and the encoder's workspace largest at the smallest region."""
import ctypes as C

import numpy as np
import pytest

from huffman_coding_gap_arrays_b200 import _lib
from huffman_coding_gap_arrays_b200.batch import LaunchConfig

U64P = C.POINTER(C.c_uint64)


def _arr(sizes):
    a = np.ascontiguousarray(np.asarray(sizes, np.uint64))
    return a, a.ctypes.data_as(U64P)


def _comp_ws(sizes, region_chunks):
    L = _lib.lib()
    cfg = LaunchConfig(region_chunks=region_chunks).cstruct()
    a, p = _arr(sizes)
    return int(L.hgap_batch_compress_workspace_bytes(len(a), p if len(a) else None, C.byref(cfg)))


def _dec_ws(sizes):
    L = _lib.lib()
    a, p = _arr(sizes)
    return int(L.hgap_batch_decompress_workspace_bytes(len(a), p if len(a) else None))


def _cap(fn, sizes):
    a, p = _arr(sizes)
    return int(fn(len(a), p if len(a) else None))


def _size_mixes():
    rng = np.random.default_rng(11)
    yield [1]
    yield [0, 1, 15, 16, 17]
    yield [4096] * 3000
    yield [64 << 20, 1 << 30, 3]
    for count in (2, 63, 1000, 5000):
        yield [int(x) for x in np.exp(rng.uniform(np.log(1), np.log(64 << 20), count))]


@pytest.mark.parametrize("sizes", list(_size_mixes()), ids=lambda s: f"{len(s)}-buffers")
def test_compress_workspace_is_subadditive(sizes):
    empty = _comp_ws([], 1)
    share = sum(_comp_ws([n], 1) - empty for n in sizes)
    for rc in (1, 2, 8, 32):
        assert _comp_ws(sizes, rc) <= empty + share
        assert _comp_ws(sizes, rc) <= _comp_ws(sizes, 1)


@pytest.mark.parametrize("sizes", list(_size_mixes()), ids=lambda s: f"{len(s)}-buffers")
def test_decompress_workspace_is_subadditive(sizes):
    empty = _dec_ws([])
    assert _dec_ws(sizes) <= empty + sum(_dec_ws([n]) - empty for n in sizes)


@pytest.mark.parametrize("sizes", list(_size_mixes()), ids=lambda s: f"{len(s)}-buffers")
def test_arena_capacities_add_up(sizes):
    L = _lib.lib()
    for fn in (L.hgap_batch_bits_capacity, L.hgap_batch_gaps_capacity):
        assert _cap(fn, sizes) == sum(_cap(fn, [n]) for n in sizes)
    # every stream fits its share: at most 16 bits a byte, 16-byte aligned starts
    for n in sizes[:50]:
        words = (16 * n + 31) // 32
        assert _cap(L.hgap_batch_bits_capacity, [n]) >= words
        assert _cap(L.hgap_batch_bits_capacity, [n]) % 4 == 0
        assert _cap(L.hgap_batch_gaps_capacity, [n]) >= ((16 * n + 127) // 128 + 7) // 8
