#!/usr/bin/env python
"""Throughput of the Huffman-with-gap-arrays path on B200.

Default workload (`batch4096`): 4096 independent buffers, sizes log-uniform
in [4 KiB, 4 MiB] (~2.46 GB), each Zipf(s ~ U[0.8,1.6]) or quantised
Gaussian (sigma ~ U[0.5,4]) by its seed, each with its own codebook.  One
step = compress every buffer (histograms -> codebooks on the device ->
encode) then decompress every buffer, as two captured CUDA graphs of the
batched path, with the launch configuration picked by the autotuner.  The
plain single-buffer path, run buffer by buffer through the public API on the
same buffers, is timed beside it (`plain`, `speedup_vs_plain`).

Single-buffer workloads (`--workload mixed_1g | zipf_16m | mixed_256m | zipf_256m`): one
step = histogram (GPU) -> codebook (host, from the 1 KiB histogram) -> fused
encode (GPU) -> decode (GPU), i.e. the reference's bin/encoder followed by
bin/decoder minus file I/O.  Inputs above the 126 MB L2 run back to back; a
smaller one (zipf_16m) has L2 flushed before every step, outside its timing.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
    torchrun --nproc-per-node N bench.py --gpus N ...   (N > 1: one rank per GPU)

Prints one JSON line.  `value` = uncompressed bytes of all ranks / (max over
ranks of the device time of K steps); `e2e` = the same through the public API
with pinned host buffers and the H2D/D2H copies inside the timed region.
The path partitions by buffer, with no collective on the data path: with
N > 1 every rank compresses and decompresses its own 4096-buffer batch (drawn
with its own seeds: a job of N x 4096 buffers, weak scaling); `--shard` splits
the one 4096-buffer batch across the ranks by bytes instead (strong scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "enc/dec GB/s of raw bytes, % HBM roofline; batched+tuned vs plain on 1 B200"
WORKLOADS = {
    "batch4096": ("4096 uint8 buffers, sizes log-uniform in [4 KiB, 4 MiB] (seed 4), each Zipf(s~U[0.8,1.6]) "
                  "or clamp(round(128 + sigma z)) with sigma~U[0.5,4] by its seed, own codebook each", 0),
    "mixed_1g": ("1 GiB uint8, 1 MiB blocks of Zipf(1.05) or 8-bit quantised N(0,1) "
                 "(+-3 sigma -> 0..255), block kind by hash(seed, block), seed 2", 1 << 30),
    "zipf_16m": ("16 MiB uint8 i.i.d. Zipf(s=1.2) over 256 symbols, seed 1", 16 << 20),
    "mixed_256m": ("256 MiB prefix-sized version of the mixed workload (profiling case)", 256 << 20),
    "zipf_256m": ("256 MiB uint8 i.i.d. Zipf(s=1.2), seed 1 (profiling case: the 2-bit shortest code's "
                  "decoder, above L2 size)", 256 << 20),
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="hgap", choices=["hgap", "reference"])
    p.add_argument("--workload", default="batch4096", choices=sorted(WORKLOADS))
    p.add_argument("--batch-count", type=int, default=4096,
                   help="buffers of the batched workload (fewer only for profiling captures)")
    p.add_argument("--plain-buffers", type=int, default=4096,
                   help="buffers of the batch timed through the plain per-buffer path")
    p.add_argument("--no-tune", action="store_true", help="skip tuning: fixed default launch shape")
    p.add_argument("--shard", action="store_true",
                   help="N > 1: split one batch across the ranks by bytes (strong scaling) instead of "
                        "giving every rank its own batch (weak scaling)")
    p.add_argument("--serve-requests", type=int, default=100000,
                   help="requests of the serving run (0: none)")
    p.add_argument("--serve-payloads", type=int, default=1024,
                   help="distinct pre-encoded decompress payloads the serving requests draw from")
    p.add_argument("--serve-overload-requests", type=int, default=5000,
                   help="requests of the overload run (offered load above capacity, small budget)")
    p.add_argument("--serve-gbs", type=float, default=20.0, help="offered load of the serving run")
    p.add_argument("--cpu-sample-mib", type=int, default=256)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--e2e-groups", type=int, default=32, help="batched e2e: groups of consecutive buffers")
    p.add_argument("--e2e-streams", type=int, default=4, help="batched e2e: streams the groups take in turn")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-kernels", action="store_true",
                   help="skip the single-buffer kernel timings on the plain-method inputs (C1, C2)")
    return p.parse_args()


def peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_ratios():
    """DRAM bytes per uncompressed byte per kernel, from the committed ncu summary."""
    out = {}
    for name in ("dram_traffic_mixed_1g.txt", "dram_traffic_batch1024.txt"):
        path = os.path.join(ROOT, "profiles", name)
        if not os.path.exists(path):
            continue
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and parts[0] == "traffic_per_input_byte":
                out[parts[1]] = float(parts[2])
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        import torch
        self.proc = None
        try:
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            ident = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", ident, "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for name, val in zip(names, f[3:7]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.out.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_roundtrip(x_np, threads: int):
    """The oracle (CPU restatement of the reference path) over one sample:
    histogram -> codebook -> encode -> decode, all host threads."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    h = O.histogram_mt(x_np, threads)
    cb = O.codebook(h)
    bits, gaps = O.encode_mt(x_np, cb, cb.total_bits, threads)
    y = O.decode_mt(bits, gaps, (cb.total_bits + 127) // 128, cb, x_np.size, threads)
    dt = time.perf_counter() - t0
    return dt, y


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def make_workload(name: str, device, rank: int = 0):
    from huffman_coding_gap_arrays_b200 import workloads as WL
    if name in ("mixed_1g", "mixed_256m"):
        return WL.mixed_buffer(WORKLOADS[name][1], seed=2 + 1000 * rank, device=device)
    return WL.zipf_buffer(WORKLOADS[name][1], 1.2, seed=1 + 1000 * rank, device=device)


def batch_workload(device, rank: int = 0, count: int = 4096, indices=None):
    """The buffers of the batched workload (4096; fewer for profiling), packed
    back to back in one device allocation (so the end-to-end copies are one
    H2D and one D2H).  `indices`: only those buffers of the batch (a rank's
    share); otherwise the whole batch, drawn with the rank's own seeds."""
    import torch
    from huffman_coding_gap_arrays_b200 import workloads as WL
    if indices is not None:
        all_sizes = WL.batch_sizes(count, seed=4)
        pick = [(all_sizes[i], 1000 + i) for i in indices]
    else:
        pick = [(n, 1000 + i + 1000003 * rank) for i, n in enumerate(WL.batch_sizes(count, seed=4 + 1000 * rank))]
    sizes = [n for n, _ in pick]
    total = sum(sizes)
    flat = torch.empty(max(total, 1), dtype=torch.uint8, device=device)
    views, p = [], 0
    for n, seed in pick:
        v = flat[p:p + n]
        v.copy_(WL.batch_buffer(n, seed, device=device))
        views.append(v)
        p += n
    return sizes, flat[:total], views


def cpu_batch_sample(sizes, flat_host, threads: int, budget: int):
    """Oracle round trips of the batch's first buffers up to `budget` bytes."""
    from oracle import oracle as O
    import numpy as np
    t, done, p = 0.0, 0, 0
    for n in sizes:
        if done >= budget:
            break
        xs = np.ascontiguousarray(flat_host[p:p + n])
        t0 = time.perf_counter()
        h = O.histogram_mt(xs, threads)
        cb = O.codebook(h)
        bits, gaps = O.encode_mt(xs, cb, cb.total_bits, threads)
        y = O.decode_mt(bits, gaps, (cb.total_bits + 127) // 128, cb, n, threads)
        t += time.perf_counter() - t0
        assert np.array_equal(y, xs)
        done += n
        p += n
    return done, t


# ---------------------------------------------------- plain kernels, C1 / C2 --
PLAIN_CONFIGS = (("zipf_16m", "C1: 16 MiB i.i.d. Zipf(1.2), seed 1"),
                 ("mixed_1g", "C2: 1 GiB of 1 MiB Zipf(1.05) / quantised N(0,1) blocks, seed 2"))
FLUSH_BYTES = 256 << 20  # > the 126 MB L2: written before every timed repetition
SERIAL_SAMPLE_MIB = 32   # the single-thread CPU baseline's sample


def _median(v):
    return round(statistics.median(v), 4)


def _entry(ms, n, alg=None):
    d = {"ms": _median(ms), "raw_gbs": round(n / statistics.median(ms) / 1e6, 1)}
    if alg is not None:
        d["alg_gbs"] = round(alg / statistics.median(ms) / 1e6, 1)
    return d


def time_plain_kernels(dev, reps: int = 5):
    """This library's single-buffer entry points on the plain-method inputs
    (C1, C2), each call bracketed by CUDA events on the launching stream, L2
    flushed before every repetition; median of `reps`.  The operations match
    the reference's own kernels timed by `--impl reference` (reference_gpu):
    histogram = hgap_histogram; encode = hgap_encode given the codebook
    (memsets, region histograms, encoder); decode = hgap_decode (workspace
    memset, decoder); pipeline = hgap_encode_histogram + hgap_encode_prepared
    (the histogram pass feeding the codebook, then the encoder alone)."""
    import torch
    import huffman_coding_gap_arrays_b200 as H
    stream = torch.cuda.current_stream()
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    out = {}
    for name, desc in PLAIN_CONFIGS:
        x = make_workload(name, dev)
        n = x.numel()
        hist = H.histogram(x)
        book, sizes = H.Codebook.from_histogram(hist.cpu())
        enc = H.Encoder(n, dev)
        dec = H.Decoder(sizes.segments, dev)
        bits = torch.empty(sizes.words + 4, dtype=torch.int32, device=dev)
        gaps = torch.empty(sizes.gap_words + 4, dtype=torch.int32, device=dev)
        y = torch.empty(n, dtype=torch.uint8, device=dev)
        C = 4 * (sizes.words + sizes.gap_words)
        t = {k: [] for k in ("histogram", "encode", "decode", "pass1", "encode_kernel")}

        def timed(key, fn):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            t[key].append(a.elapsed_time(b))

        for r in range(reps + 1):
            timed("histogram", lambda: H.histogram(x, out=hist))
            timed("encode", lambda: enc.encode(x, book, sizes, bits=bits, gaps=gaps, check_status=False))
            timed("decode", lambda: dec.decode(bits[:sizes.words], gaps[:sizes.gap_words], sizes, book, n,
                                               out=y, check_status=False))
            timed("pass1", lambda: enc.histogram(x, out=hist))
            timed("encode_kernel", lambda: enc.encode(x, book, sizes, bits=bits, gaps=gaps, check_status=False,
                                                      prepared=True))
            if r == 0:
                for v in t.values():
                    v.clear()  # the first round is a warm-up
        enc.check()
        dec.decode(bits[:sizes.words], gaps[:sizes.gap_words], sizes, book, n, out=y)
        if not torch.equal(y, x):
            raise SystemExit(f"{name}: decode(encode(x)) != x")
        out[name] = {
            "config": desc, "bytes": n, "compressed_bytes": C,
            "histogram": _entry(t["histogram"], n, n),
            "encode": _entry(t["encode"], n, 2 * n + C),
            "decode": _entry(t["decode"], n, C + n),
            "pipeline_pass1": _entry(t["pass1"], n, n),
            "pipeline_encode_kernel": _entry(t["encode_kernel"], n, n + C),
        }
        del x, bits, gaps, y, enc, dec
        torch.cuda.empty_cache()
    return out


def time_reference_kernels(dev, reps: int = 5):
    """The reference's OWN GPU kernels (encoder/src/encoder.cu,
    decoder/src/decoder.cu, built unmodified for sm_100a into oracle/_ref) on
    the same plain-method inputs and with the same timing rules as
    time_plain_kernels: cu_histgram + mergeHistogram; encode() on the device
    (its memsets, cuencoder, cu_get_gaparray) given the reference's own
    codebook; decoder_l1_l2() on the device (its memsets, gpu_dec_l1_l2) on the
    longest prefix whose stream fills whole 128-segment blocks (its partial
    last block is unreliable, oracle/ref_gpu.whole_block_prefix; a few KiB
    short of the input).  The reference decoder's output is checked against
    the input."""
    import numpy as np
    import torch
    from oracle import oracle as O
    from oracle import ref_gpu as RG
    stream = torch.cuda.current_stream()
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    out = {}
    for name, desc in PLAIN_CONFIGS:
        x = make_workload(name, dev)
        n = x.numel()
        buf = RG.padded_input(x, dev)
        h, _, _ = RG.histogram(buf, n)
        cb = O.ref_codebook(h)
        _, W, S, G = cb.sizes()
        C = 4 * (W + G)
        t = {k: [] for k in ("hist", "merge", "enc_memset", "cuencoder", "gaparray", "dec_memset", "gpu_dec")}
        # the reference decoder runs on the longest prefix whose stream fills whole 128-segment
        # blocks (its partial last block is unreliable: oracle/ref_gpu.whole_block_prefix)
        m = RG.whole_block_prefix(x, cb)
        xm = x[:m]
        bits_m = int(torch.from_numpy(cb.length.astype(np.int64)).to(dev)[xm.long()].sum().item())
        cbm = RG.with_total_bits(cb, bits_m)
        _, Wm, Sm, Gm = cbm.sizes()
        rb, rg, _, _, _ = RG.encode(RG.padded_input(xm, dev), m, cbm)
        dbufs = RG.DecodeBuffers(rb, rg, m)
        decoded = None
        for r in range(reps + 1):
            flush.zero_()
            _, a, b = RG.histogram(buf, n)
            t["hist"].append(a)
            t["merge"].append(b)
            flush.zero_()
            bits, gaps, em, e, g = RG.encode(buf, n, cb)
            t["enc_memset"].append(em)
            t["cuencoder"].append(e)
            t["gaparray"].append(g)
            flush.zero_()
            res = RG.decode(dbufs, Sm, cbm)
            if res is not None:
                decoded, dm, dk = res
                t["dec_memset"].append(dm)
                t["gpu_dec"].append(dk)
            if r == 0:
                for v in t.values():
                    v.clear()
        torch.cuda.synchronize()
        entry = {"config": desc, "bytes": n, "compressed_bytes": C,
                 "histogram": _entry([a + b for a, b in zip(t["hist"], t["merge"])], n, n),
                 "histogram_kernels_ms": {"cu_histgram": _median(t["hist"]), "mergeHistogram": _median(t["merge"])},
                 "encode": _entry([a + b + c for a, b, c in zip(t["enc_memset"], t["cuencoder"], t["gaparray"])],
                                  n, n + C),
                 "encode_kernels_ms": {"memsets": _median(t["enc_memset"]), "cuencoder": _median(t["cuencoder"]),
                                       "cu_get_gaparray": _median(t["gaparray"])}}
        if t["gpu_dec"]:
            Cm = 4 * (Wm + Gm)
            entry["decode"] = _entry([a + b for a, b in zip(t["dec_memset"], t["gpu_dec"])], m, Cm + m)
            entry["decode_kernels_ms"] = {"memsets": _median(t["dec_memset"]), "gpu_dec_l1_l2": _median(t["gpu_dec"])}
            entry["decode_bytes"] = m
            entry["decode_round_trip_exact"] = bool(torch.equal(decoded, xm))
        else:
            entry["decode"] = None
            entry["decode_skipped"] = "the reference's level-1 table boundary is wrong for this codebook"
        ref_bits = np.asarray(bits.cpu().numpy()).view(np.uint32)
        entry["stream_words"] = int(ref_bits.size)
        out[name] = entry
        del x, xm, buf, bits, gaps, rb, rg, dbufs, decoded
        torch.cuda.empty_cache()
    return out


def run_reference(args, rank: int, world: int):
    """`--impl reference`: the reference path's CPU implementation (the oracle
    port -- the reference itself has no CPU encoder/decoder) on the box's host
    cores, on a bounded sample of the same workload."""
    if rank != 0:
        return
    import numpy as np
    import torch
    threads = host_threads()
    if args.workload == "batch4096":
        desc = WORKLOADS["batch4096"][0]
        sizes, flat, _ = batch_workload("cpu", 0, args.batch_count)
        fh = flat.numpy()
        budget = args.cpu_sample_mib << 20
        for _ in range(args.warmup):
            cpu_batch_sample(sizes, fh, threads, budget // 8)
        done, t = 0, 0.0
        for _ in range(args.steps):
            d, dt = cpu_batch_sample(sizes, fh, threads, budget)
            done += d
            t += dt
        value = done / t / 1e9
        n_full, sample = sum(sizes), done // max(args.steps, 1)
        what = (f"the batch's first buffers up to {budget >> 20} MiB ({sample} bytes), per buffer "
                f"histogram+codebook+encode+decode (oracle/hgap_oracle.c, pthreads)")
    else:
        desc, n_full = WORKLOADS[args.workload]
        x = make_workload(args.workload, "cpu")
        sample = min(n_full, args.cpu_sample_mib << 20)
        xs = np.ascontiguousarray(x[:sample].numpy())
        for _ in range(args.warmup):
            cpu_roundtrip(xs, threads)
        times = []
        for _ in range(args.steps):
            dt, y = cpu_roundtrip(xs, threads)
            times.append(dt)
        assert np.array_equal(y, xs)
        t = sum(times)
        value = sample * args.steps / t / 1e9
        what = (f"first {sample >> 20} MiB of the workload, histogram+codebook+encode+decode per step "
                f"(oracle/hgap_oracle.c, pthreads)")
    ref_gpu = None
    if not args.no_kernels:
        from oracle import ref_gpu as RG
        if not torch.cuda.is_available():
            ref_gpu = {"unavailable": "no CUDA device"}
        elif not RG.available():
            ref_gpu = {"unavailable": "oracle/_ref/libref_gpu_time.so not built (reference sources absent)"}
        else:
            clk = ClockSampler(0)
            ref_gpu = time_reference_kernels(torch.device("cuda", 0))
            ref_gpu["clocks"] = clk.stop()
            ref_gpu["how"] = ("the reference's own kernels (encoder/src/encoder.cu, decoder/src/decoder.cu, "
                              "unmodified, sm_100a) launched as its histgram()/encode()/decoder_l1_l2() do, "
                              "CUDA events around each, L2 flushed before each repetition, median of 5")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * t / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": desc, "bytes": n_full, "sample_bytes": sample},
        "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": what},
        "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_gpu": ref_gpu,
    }
    print(json.dumps(line), flush=True)
    del torch


def train_learned_tuner(dev):
    """The learned tuner, trained on the autotuner's records of batches drawn
    from the same distributions as the workload but with other seeds, counts
    and size ranges (it never sees the timed batch)."""
    import torch
    from huffman_coding_gap_arrays_b200 import mlp as ML
    from huffman_coding_gap_arrays_b200 import tuner as T
    from huffman_coding_gap_arrays_b200 import workloads as WL
    shapes = [(64, 64 << 10), (256, 256 << 10), (512, 1 << 20), (128, 4 << 20), (1024, 4 << 20),
              (2048, 1 << 20), (32, 16 << 20), (384, 2 << 20), (1536, 512 << 10), (768, 4 << 20),
              (96, 8 << 20), (2048, 4 << 20), (128, 128 << 10), (1024, 2 << 20), (3000, 4 << 20),
              (48, 32 << 20), (640, 1 << 20), (2600, 2 << 20), (200, 16 << 20), (4096, 4 << 20),
              # the few-request batches of serving (64 KiB .. 64 MiB requests)
              (1, 64 << 20), (2, 64 << 20), (3, 64 << 20), (1, 8 << 20), (2, 16 << 20), (4, 64 << 20),
              (1, 1 << 20), (8, 64 << 20)]
    hold = [(200, 2 << 20), (1200, 4 << 20), (2, 32 << 20)]

    def records(sh, seed):
        recs = []
        for k, (count, hi) in enumerate(sh):
            sz = WL.batch_sizes(count, lo=4096, hi=hi, seed=seed + k)
            bufs = [WL.batch_buffer(n, (seed + k) * 7919 + i, device=dev) for i, n in enumerate(sz)]
            outs = [torch.empty_like(b) for b in bufs]
            recs.extend(T.Autotuner(reps=5, warmup=2).tune(bufs, outs, T.batch_features(bufs)).records)
            del bufs, outs
        return recs

    lt = ML.LearnedTuner.train(records(shapes, 9500), holdout=records(hold, 9600), steps=3000)
    torch.cuda.empty_cache()
    return lt


def picks_cfg(tuning):
    from huffman_coding_gap_arrays_b200 import batch as B
    m = tuning.get("measured", {})
    if "autotuner" in m:
        return B.LaunchConfig(**m["autotuner"]["config"])
    return B.LaunchConfig(**tuning["config"])


def run_serving(args, pool, learned, fixed_cfg, dev):
    """Serving at `--serve-gbs` offered load: the learned tuner, the one shape
    the exhaustive search chose for the batched workload, and the plain
    per-request path, each on the same request stream; then one run at an
    offered load far above capacity with a small HBM budget, so that the
    admission control binds.  Decompress requests draw from a pool of
    `--serve-payloads` streams, each a buffer of the batched workload's
    distributions (Zipf or quantised Gaussian by its seed) with a size
    log-uniform in [64 KiB, 64 MiB], encoded by the batched path."""
    import numpy as np
    import torch
    from huffman_coding_gap_arrays_b200 import serve as SV
    from huffman_coding_gap_arrays_b200 import workloads as WL
    rng = np.random.default_rng(17)
    streams = []
    for k0 in range(0, args.serve_payloads, 128):  # encoded 128 at a time: the raw buffers go after
        bufs = [WL.batch_buffer(int(np.exp(rng.uniform(np.log(64 << 10), np.log(64 << 20)))), 500_000 + k, dev)
                for k in range(k0, min(args.serve_payloads, k0 + 128))]
        streams += SV.encode_streams(bufs)
        del bufs
    torch.cuda.synchronize()
    traffic = np.mean([st.features for st in streams], axis=0)
    out = {"requests": args.serve_requests, "offered_gbs": args.serve_gbs, "hbm_budget_gb": 40,
           "sizes": "log-uniform 64 KiB .. 64 MiB, 50/50 compress/decompress, Poisson arrivals",
           "payloads": f"compress: slices of the batched workload; decompress: one of {len(streams)} "
                       f"pre-encoded streams of its distributions, drawn per request",
           "warmup": "an untimed stream of min(5000, a fifth) as many requests first, per policy",
           "where": "payloads and results resident in HBM; latency = queueing + GPU service; "
                    "service = launch to completion"}
    policies = [("autotuner_fixed", dict(config=fixed_cfg))]
    if learned is not None and learned.usable:
        # the network departs from the shape the search found for the workload only where
        # it predicts a batch gains more than its margin from another one
        learned.set_default(fixed_cfg)
        policies.insert(0, ("mlp", dict(tuner=learned)))
    policies.append(("plain", dict(policy="plain")))
    warm = min(5000, max(100, args.serve_requests // 5))
    for name, kw in policies:
        srv = SV.Server(hbm_budget=40e9, traffic_features=traffic, device=dev, **kw)
        # untimed warm-up stream: the allocator's pools and the launch attributes settle first
        srv.run(SV.poisson_requests(warm, args.serve_gbs, pool, streams, seed=29))
        srv.reset_counters()
        reqs = SV.poisson_requests(args.serve_requests, args.serve_gbs, pool, streams, seed=23)
        out[name] = srv.run(reqs)
        del reqs
        torch.cuda.synchronize()
    if args.serve_overload_requests:
        gbs, budget = 400.0, 2e9
        srv = SV.Server(hbm_budget=budget, traffic_features=traffic, device=dev, config=fixed_cfg)
        srv.run(SV.poisson_requests(min(1000, args.serve_overload_requests), gbs, pool, streams, seed=31))
        srv.reset_counters()
        reqs = SV.poisson_requests(args.serve_overload_requests, gbs, pool, streams, seed=37)
        st = srv.run(reqs)
        st["offered_gbs"] = gbs
        out["overload_autotuner_fixed"] = st
        del reqs
        torch.cuda.synchronize()
    return out


def run_e2e_batch(args, sizes, flat, flat_out, ins, outs, cfg, total, job_bytes, dev, pg, stream):
    """The batched round trip through host memory (see `e2e` in the module
    docstring); everything it allocates is released when it returns."""
    import numpy as np
    import torch
    from huffman_coding_gap_arrays_b200 import batch as B
    # The batch in groups of consecutive buffers, each with its own plan and graphs, spread
    # over a few streams: one group's uploads run while another's downloads and kernels do
    # (PCIe is full duplex), where a single plan would copy in, compute and copy out in turn.
    # Measured per step (groups x streams): 1 plan 150 ms, 4x2 104 ms, 8x3 95 ms, 16x4 90 ms,
    # 32x4 89 ms -- 3.8 GB each way, ~43 GB/s per direction at once: the link, not the GPU.
    ngroups = max(1, min(args.e2e_groups, len(sizes)))
    offs = [0]
    for n in sizes:
        offs.append(offs[-1] + n)
    cuts = [0]
    for g in range(1, ngroups):  # group ends where the running bytes pass g/ngroups of the batch
        j = int(np.searchsorted(np.asarray(offs), total * g / ngroups))
        cuts.append(min(max(j, cuts[-1] + 1), len(sizes)))
    cuts.append(len(sizes))
    groups = []
    for i0, i1 in zip(cuts[:-1], cuts[1:]):
        if i1 <= i0:
            continue
        gp = B.BatchCodec(sizes[i0:i1], cfg, device=dev)
        gp.bind(ins[i0:i1], outs[i0:i1])
        gp.compress()
        gp.decompress()
        gp.check()
        ge = gp.entries_host()
        ub = max(e.bits_offset + e.words for e in ge)
        ug = max(e.gaps_offset + e.gap_words for e in ge)
        groups.append({
            "plan": gp, "a": offs[i0], "b": offs[i1], "ub": ub, "ug": ug,
            "gc": gp.capture(compress=True, decompress=False),
            "gd": gp.capture(compress=False, decompress=True),
            "ent": torch.empty(gp.entries.numel(), dtype=torch.uint8, pin_memory=True),
            "bits": torch.empty(max(ub, 1), dtype=torch.int32, pin_memory=True),
            "gaps": torch.empty(max(ug, 1), dtype=torch.int32, pin_memory=True)})
    in_host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    in_host.copy_(flat)
    out_host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    streams = [torch.cuda.Stream(device=dev) for _ in range(max(1, args.e2e_streams))]

    def e2e_step():
        cur = torch.cuda.current_stream(dev)
        for k, G in enumerate(groups):
            s = streams[k % len(streams)]
            s.wait_stream(cur)
            gp, a_, b2, ub, ug = G["plan"], G["a"], G["b"], G["ub"], G["ug"]
            with torch.cuda.stream(s):
                flat[a_:b2].copy_(in_host[a_:b2], non_blocking=True)      # H2D inputs
                G["gc"].replay()                                         # compress
                G["ent"].copy_(gp.entries, non_blocking=True)            # D2H entries + streams
                G["bits"][:ub].copy_(gp.bits[:ub], non_blocking=True)
                G["gaps"][:ug].copy_(gp.gaps[:ug], non_blocking=True)
                gp.entries.copy_(G["ent"], non_blocking=True)            # H2D for decompress
                gp.bits[:ub].copy_(G["bits"][:ub], non_blocking=True)
                gp.gaps[:ug].copy_(G["gaps"][:ug], non_blocking=True)
                G["gd"].replay()                                         # decompress
                out_host[a_:b2].copy_(flat_out[a_:b2], non_blocking=True)  # D2H outputs
        for s in streams:
            cur.wait_stream(s)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    e2e_steps = max(2, args.steps // 2)
    a = torch.cuda.Event(enable_timing=True)
    b_ = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    b_.record(stream)
    torch.cuda.synchronize()
    e_ms = a.elapsed_time(b_)
    for G in groups:
        G["plan"].check()
    if not torch.equal(out_host, in_host):
        raise SystemExit("e2e round trip mismatch")
    if pg:
        tm = torch.tensor([e_ms], device=dev)
        pg.all_reduce(tm, op=pg.ReduceOp.MAX)
        e_ms = float(tm.item())
    cont = sum(G["plan"].entries.numel() + 4 * (G["ub"] + G["ug"]) for G in groups)
    e2e = {"value": round(job_bytes * e2e_steps / e_ms / 1e6, 3), "unit": "GB/s",
           "h2d_bytes_per_step": total + cont, "d2h_bytes_per_step": cont + total,
           "ms_per_step": round(e_ms / e2e_steps, 3),
           "how": f"{len(groups)} groups of consecutive buffers on {len(streams)} streams: upload, compress, "
                  "container down and up again, decompress, download; each group's copies and "
                  "kernels in order, groups overlapping"}
    return e2e


def run_batch(args, rank, world, dev, pg):
    """The batched path on the 4096-buffer workload (see the module docstring)."""
    import numpy as np
    import torch
    import huffman_coding_gap_arrays_b200 as H
    from huffman_coding_gap_arrays_b200 import batch as B
    from huffman_coding_gap_arrays_b200 import tuner as T

    from huffman_coding_gap_arrays_b200 import parallel as PL
    from huffman_coding_gap_arrays_b200 import workloads as WL
    desc = WORKLOADS["batch4096"][0]
    if args.batch_count != 4096:
        desc = desc.replace("4096 uint8 buffers", f"{args.batch_count} uint8 buffers (profiling size)")
    shard = world > 1 and args.shard
    if shard:  # one batch, each rank its byte-balanced share: no collective on the data path
        all_sizes = WL.batch_sizes(args.batch_count, seed=4)
        mine = PL.shard_by_bytes(all_sizes, world)[rank]
        sizes, flat, ins = batch_workload(dev, rank, args.batch_count, indices=mine)
        job_bytes = sum(all_sizes)
    else:
        sizes, flat, ins = batch_workload(dev, rank, args.batch_count)
        job_bytes = sum(sizes)
        if pg:  # every rank's own batch (its own sizes): the job is all of them, summed once, untimed
            t = torch.tensor([job_bytes], dtype=torch.int64, device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.SUM)
            job_bytes = int(t.item())
    total = sum(sizes)
    flat_out = torch.empty(total, dtype=torch.uint8, device=dev)
    outs, p = [], 0
    for n in sizes:
        outs.append(flat_out[p:p + n])
        p += n

    # ---- tuning (untimed): learned tuner, checked against the exhaustive search
    plan = B.BatchCodec(sizes, B.LaunchConfig(region_chunks=1), device=dev)  # workspace fits every shape
    plan.bind(ins, outs)
    tuning = {}
    learned = None
    if args.no_tune:
        cfg = B.LaunchConfig()
        tuning["method"] = "fixed default"
    else:
        t0 = time.time()
        learned = train_learned_tuner(dev)
        tuning["learned_train_seconds"] = round(time.time() - t0, 2)
        tuning["learned_holdout_rmse"] = round(learned.holdout_rmse, 4)
        feats = T.batch_features(ins)
        t0 = time.time()
        res = T.Autotuner(reps=2, warmup=1).tune(ins, outs, feats, plan=plan)
        tuning["autotuner_seconds"] = round(time.time() - t0, 2)
        picks = {"default": B.LaunchConfig(), "autotuner": res.config}
        if learned.usable:
            picks["mlp"] = learned.choose(feats)
        measured = {}
        for name, c in picks.items():
            plan.config = c
            cm = T._time(plan.compress, 3, 1)
            dm = T._time(plan.decompress, 3, 1)
            plan.check()
            measured[name] = {"config": vars(c), "compress_ms": round(cm, 4), "decompress_ms": round(dm, 4)}
        tuning["measured"] = measured
        cfg = picks["mlp"] if "mlp" in picks else picks["autotuner"]
        tuning["method"] = ("learned tuner (MLP ensemble trained on autotuner records of other batches)"
                            if "mlp" in picks else "autotuner (exhaustive; learned tuner not usable)")
    tuning["config"] = vars(cfg)
    plan.config = cfg
    plan.compress()
    plan.decompress()
    plan.check()
    if not torch.equal(flat_out, flat):
        raise SystemExit("batched round trip mismatch")
    ents = plan.entries_host()
    C = sum(4 * (e.words + e.gap_words) for e in ents)
    used_bits = max(e.bits_offset + e.words for e in ents)
    used_gaps = max(e.gaps_offset + e.gap_words for e in ents)
    g_c = plan.capture(compress=True, decompress=False)
    g_d = plan.capture(compress=False, decompress=True)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        g_c.replay()
        g_d.replay()
    torch.cuda.synchronize()

    clocks = ClockSampler(dev.index or 0) if rank == 0 else None
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        evs[k][0].record(stream)
        g_c.replay()
        evs[k][1].record(stream)
        g_d.replay()
        evs[k][2].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clock_info = clocks.stop() if clocks else None
    ms = t0.elapsed_time(t1)
    plan.check()
    if not torch.equal(flat_out, flat):
        raise SystemExit("batched round trip mismatch after the timed steps")
    if pg:
        tm = torch.tensor([ms], device=dev)
        pg.all_reduce(tm, op=pg.ReduceOp.MAX)
        ms = float(tm.item())
    c_ms = sum(e[0].elapsed_time(e[1]) for e in evs) / args.steps
    d_ms = sum(e[1].elapsed_time(e[2]) for e in evs) / args.steps
    peak, peak_src = peak_hbm()
    alg = {"compress": 2 * total + C, "decompress": C + total}
    ph_ms = {"compress": c_ms, "decompress": d_ms}
    kernels = {k: {"ms": round(ph_ms[k], 4), "raw_gbs": round(total / ph_ms[k] / 1e6, 1),
                   "alg_gbs": round(alg[k] / ph_ms[k] / 1e6, 1),
                   "frac_of_" + peak_src: round(alg[k] / ph_ms[k] / 1e6 / peak, 4)} for k in ph_ms}
    dom = max(ph_ms, key=ph_ms.get)
    achieved = alg[dom] / ph_ms[dom] / 1e6
    tr = traffic_ratios()
    roofline = {"bound": "hbm", "kernel": "batched " + dom, "achieved": round(achieved, 1), "peak": peak,
                "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": (round(tr["batch_" + dom] * total) if ("batch_" + dom) in tr else None),
                "algorithmic_bytes": alg[dom]}

    # ---- the plain single-buffer path, buffer by buffer, same buffers --------
    plain = None
    kp = min(args.plain_buffers, len(sizes))
    if kp:
        # one untimed pass first: the allocator's pools see every size once, as the batched
        # path's workspaces were allocated before its clock started
        warm = [H.compress(x) for x in ins[:kp]]
        warm = [H.decompress(c) for c in warm]
        del warm
        torch.cuda.synchronize()
        a = time.perf_counter()
        comp = [H.compress(x) for x in ins[:kp]]
        torch.cuda.synchronize()
        b_ = time.perf_counter()
        dec_out = [H.decompress(c) for c in comp]
        torch.cuda.synchronize()
        c_ = time.perf_counter()
        sub = sum(sizes[:kp])
        if not all(torch.equal(y, x) for y, x in zip(dec_out, ins[:kp])):
            raise SystemExit("plain round trip mismatch")
        plain = {"buffers": kp, "bytes": sub, "compress_gbs": round(sub / (b_ - a) / 1e9, 3),
                 "decompress_gbs": round(sub / (c_ - b_) / 1e9, 3),
                 "roundtrip_gbs": round(sub / (c_ - a) / 1e9, 3),
                 "how": "codec.compress / codec.decompress per buffer (histogram -> host codebook -> "
                        "encode; decode), wall clock with device syncs, after one untimed pass"}
        del comp, dec_out

    # ---- end to end through the public API, host buffers ---------------------
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e_batch(args, sizes, flat, flat_out, ins, outs, cfg, total, job_bytes, dev, pg, stream)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()  # the serving legs start from the allocator state they had before

    # ---- serving: a Poisson stream of mixed requests (64 KiB .. 64 MiB) -------
    serving = None
    if args.serve_requests and rank == 0 and world == 1:
        serving = run_serving(args, flat, learned, picks_cfg(tuning), dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_threads()
        fh = flat.cpu().numpy()
        budget = args.cpu_sample_mib << 20
        cpu_batch_sample(sizes, fh, threads, budget // 16)
        done, dt = cpu_batch_sample(sizes, fh, threads, budget)
        cpu = {"value": round(done / dt / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"the batch's first buffers up to {budget >> 20} MiB ({done} bytes), one "
                         f"histogram+codebook+encode+decode round trip per buffer (oracle/hgap_oracle.c, pthreads)"}
        sb = SERIAL_SAMPLE_MIB << 20
        done1, dt1 = cpu_batch_sample(sizes, fh, 1, sb)
        cpu["serial"] = {"value": round(done1 / dt1 / 1e9, 4), "unit": "GB/s", "cores": 1,
                         "sample": f"the batch's first buffers up to {SERIAL_SAMPLE_MIB} MiB ({done1} bytes), "
                                   f"the same round trip on one thread"}

    plain_kernels = None
    if rank == 0 and world == 1 and not args.no_kernels:
        clk = ClockSampler(dev.index or 0)
        plain_kernels = time_plain_kernels(dev)
        plain_kernels["clocks"] = clk.stop()
        plain_kernels["how"] = ("hgap_histogram / hgap_encode / hgap_decode and the two-call pipeline, CUDA "
                                "events around each call, L2 flushed before each repetition, median of 5")

    if rank == 0:
        value = job_bytes * args.steps / ms / 1e6
        line = {
            "metric": METRIC,
            "value": round(value, 3),
            "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "strong" if shard else "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": desc, "buffers": len(sizes), "bytes_per_gpu": total,
                       "parallelism": (f"batch sharded by bytes over {world} ranks, no data-path collective"
                                       if shard else f"{world} rank(s), each its own batch (own seeds), "
                                                     "no data-path collective"),
                       "step": "batched compress (device histograms, codebooks, encode) then batched "
                               "decompress, two captured CUDA graphs",
                       "l2": (f"inputs ({total / 1e9:.2f} GB per GPU) larger than the 126 MB L2; no flush"
                              if total > 126e6 else "inputs smaller than the 126 MB L2 (profiling size)"),
                       "compressed_bytes": C, "compressed_over_raw": round(C / total, 4),
                       "tuning": tuning},
            "encode_gbs": round(total / c_ms / 1e6, 1),
            "decode_gbs": round(total / d_ms / 1e6, 1),
            "plain": plain,
            "serving": serving,
            "speedup_vs_plain": (round(value / world / plain["roundtrip_gbs"], 2)
                                 if plain else None),
            "kernels": kernels,
            "plain_kernels": plain_kernels,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": (B.COMPRESS_KERNELS + B.DECOMPRESS_KERNELS) * args.steps,
            "clocks": clock_info,
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import huffman_coding_gap_arrays_b200 as H

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
        pg = dist

    if args.workload == "batch4096":
        run_batch(args, rank, world, dev, pg)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    desc, n = WORKLOADS[args.workload]
    x = make_workload(args.workload, dev, rank)
    stream = torch.cuda.current_stream()
    hist = torch.empty(256, dtype=torch.int32, device=dev)
    hist_host = torch.empty(256, dtype=torch.int32, pin_memory=True)

    # size the outputs once from the histogram (W for this buffer is fixed)
    enc = H.Encoder(n, dev)
    enc.histogram(x, out=hist)
    book0, sizes0 = H.Codebook.from_histogram(hist.cpu())
    bits = torch.empty(sizes0.words + 16, dtype=torch.int32, device=dev)
    gaps = torch.empty(sizes0.gap_words + 16, dtype=torch.int32, device=dev)
    out = torch.empty(n + 16, dtype=torch.uint8, device=dev)
    dec = H.Decoder(sizes0.segments, dev)

    ev = {k: [] for k in ("hist", "encode", "decode")}

    def step(record: bool):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(6)] if record else None
        if record:
            e[0].record(stream)
        enc.histogram(x, out=hist)  # hgap_encode_histogram: global + per-super-tile histograms
        if record:
            e[1].record(stream)
        hist_host.copy_(hist, non_blocking=True)
        stream.synchronize()
        book, sizes = H.Codebook.from_histogram(hist_host)
        if record:
            e[2].record(stream)
        enc.encode(x, book, sizes, bits=bits, gaps=gaps, check_status=False, prepared=True)
        if record:
            e[3].record(stream)
            e[4].record(stream)
        dec.decode(bits, gaps, sizes, book, n, out=out, check_status=False)
        if record:
            e[5].record(stream)
            ev["hist"].append((e[0], e[1]))
            ev["encode"].append((e[2], e[3]))
            ev["decode"].append((e[4], e[5]))
        return book, sizes

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    enc.check()
    dec.check()
    if not torch.equal(out[:n], x):
        raise SystemExit("decode(encode(x)) != x")

    clocks = ClockSampler(local) if rank == 0 else None
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    # an input that fits the 126 MB L2 gets L2 flushed (a 256 MiB write) before every
    # step, outside the step's own events; larger inputs run back to back
    small = n < (128 << 20)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev) if small else None
    spans = []
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        if small:
            flush.zero_()
            a_ = torch.cuda.Event(enable_timing=True)
            b_ = torch.cuda.Event(enable_timing=True)
            a_.record(stream)
            book, sizes = step(True)
            b_.record(stream)
            spans.append((a_, b_))
        else:
            book, sizes = step(True)
    t1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clock_info = clocks.stop() if clocks else None
    ms = sum(a_.elapsed_time(b_) for a_, b_ in spans) if small else t0.elapsed_time(t1)
    enc.check()
    dec.check()
    if not torch.equal(out[:n], x):
        raise SystemExit("decode(encode(x)) != x after the timed steps")
    if pg:
        tm = torch.tensor([ms], device=dev)
        pg.all_reduce(tm, op=pg.ReduceOp.MAX)
        ms = float(tm.item())

    kern_ms = {k: sum(a.elapsed_time(b) for a, b in v) / len(v) for k, v in ev.items()}
    C = 4 * (sizes.words + sizes.gap_words)
    alg = {"hist": n, "encode": n + C, "decode": C + n}
    peak, peak_src = peak_hbm()
    kernels = {k: {"ms": round(kern_ms[k], 4),
                   "raw_gbs": round(n / kern_ms[k] / 1e6, 1),
                   "alg_gbs": round(alg[k] / kern_ms[k] / 1e6, 1),
                   "frac_of_" + peak_src: round(alg[k] / kern_ms[k] / 1e6 / peak, 4)}
               for k in kern_ms}
    dom = max(kern_ms, key=kern_ms.get)
    achieved = alg[dom] / kern_ms[dom] / 1e6
    tr = traffic_ratios()
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": (round(tr[dom] * n) if dom in tr else None),
                "algorithmic_bytes": alg[dom]}

    # ---- end to end through the public API, host buffers -------------------
    e2e = None
    if not args.no_e2e:
        x_host = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        x_host.copy_(x)
        bits_host = torch.empty(sizes.words, dtype=torch.int32, pin_memory=True)
        gaps_host = torch.empty(sizes.gap_words, dtype=torch.int32, pin_memory=True)
        y_host = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        x_dev = torch.empty_like(x)
        bits_in = torch.empty_like(bits)
        gaps_in = torch.empty_like(gaps)

        def e2e_step():
            x_dev.copy_(x_host, non_blocking=True)                      # H2D input
            enc.histogram(x_dev, out=hist)
            hist_host.copy_(hist, non_blocking=True)
            stream.synchronize()
            book, sz = H.Codebook.from_histogram(hist_host)
            b, g = enc.encode(x_dev, book, sz, bits=bits, gaps=gaps, check_status=False, prepared=True)
            bits_host[:sz.words].copy_(b, non_blocking=True)            # D2H container payload
            gaps_host[:sz.gap_words].copy_(g, non_blocking=True)
            bits_in[:sz.words].copy_(bits_host[:sz.words], non_blocking=True)   # H2D for decode
            gaps_in[:sz.gap_words].copy_(gaps_host[:sz.gap_words], non_blocking=True)
            dec.decode(bits_in, gaps_in, sz, book, n, out=out, check_status=False)
            y_host.copy_(out[:n], non_blocking=True)                   # D2H output
            return sz

        e2e_steps = max(2, args.steps // 2)
        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        a = torch.cuda.Event(enable_timing=True)
        b_ = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(e2e_steps):
            sz = e2e_step()
        b_.record(stream)
        torch.cuda.synchronize()
        e_ms = a.elapsed_time(b_)
        enc.check()
        dec.check()
        if not torch.equal(y_host, x_host):
            raise SystemExit("e2e round trip mismatch")
        if pg:
            tm = torch.tensor([e_ms], device=dev)
            pg.all_reduce(tm, op=pg.ReduceOp.MAX)
            e_ms = float(tm.item())
        cbytes = 4 * (sz.words + sz.gap_words)
        e2e = {"value": round(world * n * e2e_steps / e_ms / 1e6, 3), "unit": "GB/s",
               "h2d_bytes_per_step": n + cbytes, "d2h_bytes_per_step": cbytes + n,
               "ms_per_step": round(e_ms / e2e_steps, 3)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_threads()
        sample = min(n, args.cpu_sample_mib << 20)
        xs = np.ascontiguousarray(x[:sample].cpu().numpy())
        cpu_roundtrip(xs, threads)
        dt, y = cpu_roundtrip(xs, threads)
        assert np.array_equal(y, xs)
        cpu = {"value": round(sample / dt / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"first {sample >> 20} MiB of the workload, one histogram+codebook+encode+"
                         f"decode round trip (oracle/hgap_oracle.c, pthreads)"}
        s1 = min(n, SERIAL_SAMPLE_MIB << 20)
        dt1, y1 = cpu_roundtrip(np.ascontiguousarray(xs[:s1]), 1)
        assert np.array_equal(y1, xs[:s1])
        cpu["serial"] = {"value": round(s1 / dt1 / 1e9, 4), "unit": "GB/s", "cores": 1,
                         "sample": f"first {s1 >> 20} MiB of the workload, the same round trip on one thread"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(world * n * args.steps / ms / 1e6, 3),
            "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": desc, "bytes_per_gpu": n, "parallelism": f"replicas x{world}",
                       "step": "histogram -> codebook (host) -> encode -> decode",
                       "l2": (f"input ({n / 2**20:.0f} MiB) fits the 126 MB L2: L2 flushed before every step, "
                              f"outside its timing" if small else
                              f"input ({n / 2**20:.0f} MiB) larger than the 126 MB L2; no flush"),
                       "compressed_bytes": C, "bits_per_byte": round(sizes.bits / n, 4)},
            "encode_gbs": round(n / (kern_ms["hist"] + kern_ms["encode"]) / 1e6, 1),
            "decode_gbs": round(n / kern_ms["decode"] / 1e6, 1),
            "kernels": kernels,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": 3 * args.steps,
            "clocks": clock_info,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
