"""The serving loop on the GPU: continuous batching of mixed compress /
decompress requests, under an HBM budget, with results that are the same as
each request run alone through the single-buffer path."""
import numpy as np
import pytest
import torch

import huffman_coding_gap_arrays_b200 as H
from huffman_coding_gap_arrays_b200 import batch as B
from huffman_coding_gap_arrays_b200 import serve as SV
from huffman_coding_gap_arrays_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def _pool(nblocks=24, block=2 << 20, seed=3):
    """A pool of data whose blocks follow the batched workload's distributions."""
    return torch.cat([WL.batch_buffer(block, seed * 1000 + i) for i in range(nblocks)])


def _streams(pool, k=8, seed=4):
    rng = np.random.default_rng(seed)
    bufs = []
    for _ in range(k):
        n = int(np.exp(rng.uniform(np.log(64 << 10), np.log(8 << 20))))
        off = int(rng.integers(0, pool.numel() - n))
        bufs.append(pool[off:off + n])
    return bufs, SV.encode_streams(bufs)


def _check(reqs, originals):
    for r in reqs:
        assert r.done == r.done and r.done >= r.arrival
        if r.kind == "compress":
            got = r.result.to_compressed() if isinstance(r.result, SV.EncodedStream) else r.result
            ref = H.compress(r.data)
            assert got.to_container() == ref.to_container(), f"request {r.rid}: compressed stream"
        else:
            assert torch.equal(r.result, originals[id(r.stream)]), f"request {r.rid}: decompressed bytes"


def _run(server, count, rate_gbs, seed, hi=8 << 20):
    pool = _pool()
    bufs, streams = _streams(pool)
    originals = {id(s): b for s, b in zip(streams, bufs)}
    reqs = SV.poisson_requests(count, rate_gbs, pool, streams, seed=seed, hi=hi)
    stats = server.run(reqs)
    _check(reqs, originals)
    return stats, reqs


def test_results_are_the_same_alone_and_in_the_mix():
    server = SV.Server(keep_results=True, max_batch=16)
    stats, reqs = _run(server, 60, 200.0, seed=11)  # high offered load: requests share batches
    assert stats["requests"] == 60 and stats["batches"] < 60
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    kinds = {r.kind for r in reqs}
    assert kinds == {"compress", "decompress"}


def test_hbm_budget_is_respected():
    """Offered load far above capacity and a budget of a few requests: the
    admission waits on memory, every batch is charged what it really
    allocated, which never exceeds its admission bound nor the budget, and
    every result is still the one the request gets alone."""
    budget = 40 << 20
    server = SV.Server(keep_results=True, hbm_budget=budget, max_batch=64)
    stats, _ = _run(server, 40, 500.0, seed=12, hi=4 << 20)
    assert server.peak_held <= budget, server.peak_held
    assert stats["batches"] > 1
    assert stats["mem_waits"] > 0
    assert stats["bound_misses"] == 0


def test_request_bound_covers_real_allocations():
    pool = _pool(nblocks=4)
    bufs, streams = _streams(pool, k=3)
    server = SV.Server(keep_results=True)
    for kind in ("compress", "decompress"):
        reqs = [SV.Request(i, 0.0, kind, data=b if kind == "compress" else None,
                           stream=s if kind == "decompress" else None)
                for i, (b, s) in enumerate(zip(bufs, streams))]
        torch.cuda.synchronize()
        b = server._launch(reqs, 0.0)
        server.held += b.reserved  # as the loop does
        b.event.synchronize()
        assert 0 < b.reserved <= server._bound(reqs)
        server._retire(b, 0.0)
    # one request alone takes the single-buffer path (decoder, or histogram pass + encoder)
    for r in (SV.Request(9, 0.0, "decompress", stream=streams[0]), SV.Request(10, 0.0, "compress", data=bufs[1])):
        torch.cuda.synchronize()
        b = server._launch([r], 0.0)
        server.held += b.reserved
        b.event.synchronize()
        assert 0 < b.reserved <= server._bound([r])
        server._retire(b, 0.0)
        if r.kind == "decompress":
            assert torch.equal(r.result, bufs[0])
        else:
            assert r.result.to_container() == H.compress(bufs[1]).to_container()
    assert server.held == 0


def test_light_load_single_requests():
    """At a light load most batches hold one request (a lone request goes
    through the single-buffer path); every result is still exact."""
    server = SV.Server(keep_results=True)
    stats, reqs = _run(server, 24, 1.0, seed=15, hi=2 << 20)
    assert stats["batches"] >= 12
    assert {r.kind for r in reqs} == {"compress", "decompress"}


def test_learned_tuner_policy_and_fixed_shape_agree():
    pool = _pool()
    bufs, streams = _streams(pool)
    originals = {id(s): b for s, b in zip(streams, bufs)}

    class Fixed:  # a stand-in tuner that always answers one shape
        def choose(self, f):
            return B.LaunchConfig(region_chunks=2, enc_ctas_per_sm=1, dec_ctas_per_sm=2)

    for srv in (SV.Server(keep_results=True, tuner=Fixed(), tuner_min_bytes=0), SV.Server(keep_results=True)):
        reqs = SV.poisson_requests(30, 100.0, pool, streams, seed=13)
        srv.run(reqs)
        _check(reqs, originals)


def test_plain_policy():
    server = SV.Server(policy="plain", keep_results=True)
    stats, _ = _run(server, 12, 20.0, seed=14, hi=2 << 20)
    assert stats["batches"] == 0 and stats["requests"] == 12
