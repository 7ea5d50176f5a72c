"""Streaming container I/O: file-to-file compress and decompress in the
reference's container format (writer encoder/src/huff.cpp:111-125, reader
decoder/src/huff.cpp:27-81), with the disk, the copies and the kernels
overlapped.

Files are processed in groups of up to ``group_bytes`` (a larger file is a
group of its own).  Each group is one batched call (``batch.py``), so every
file gets its own codebook built on the device, and every container is the
one ``codec.compress`` would write for that file alone.  Two pinned host
staging buffers and two device buffer sets are used in turn:

    read group k+1 from disk    (I/O thread)      |
    H2D group k, then its batched call (streams)  |  at the same time
    D2H + write group k-1's results (I/O thread)  |

The host waits only for a group's small entry table (to learn its stream
sizes) before copying its streams back, one group behind the GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from ._lib import BatchEntry, CCodebook, check, lib
from .batch import ENTRY_BYTES, BatchCodec, LaunchConfig
from .codec import _stream


def _groups(sizes, group_bytes):
    out, cur, tot = [], [], 0
    for i, n in enumerate(sizes):
        if cur and tot + n > group_bytes:
            out.append(cur)
            cur, tot = [], 0
        cur.append(i)
        tot += n
    if cur:
        out.append(cur)
    return out


def _read_into(paths, pinned: torch.Tensor):
    """Reads files back to back into a pinned uint8 buffer; returns offsets."""
    view = pinned.numpy()
    offs, p = [], 0
    for path in paths:
        with open(path, "rb", buffering=0) as f:
            n = os.fstat(f.fileno()).st_size
            got = f.readinto(memoryview(view[p:p + n]))
            if got != n:
                raise IOError(f"short read of {path}")
        offs.append(p)
        p += n
    return offs


def _container_bytes(e) -> int:
    return int(lib().hgap_container_bytes(e.symbol_count, e.words, e.segments))


def _write_container(path, e, bits_np, gaps_np):
    """Writes one container from a batch entry and its host stream words."""
    cb = CCodebook()
    cb.symbol_count = e.symbol_count
    C.memmove(C.addressof(cb.symbols), C.addressof(e.symbols), 2 * 256)
    size = _container_bytes(e)
    buf = np.empty(max(size, 1), np.uint8)
    written = C.c_size_t(0)
    check(lib().hgap_container_write(buf.ctypes.data, size, C.byref(cb), e.n, e.words, e.segments,
                                     gaps_np.ctypes.data, bits_np.ctypes.data, C.byref(written)),
          "hgap_container_write")
    with open(path, "wb") as f:
        f.write(memoryview(buf[:written.value]))


def _status_after(ws: torch.Tensor, what: str) -> None:
    """Device status of a finished call (its completion event has been
    waited for, so the status word is final): read on the legacy stream,
    which does not wait for the pipeline's other streams."""
    check(lib().hgap_batch_status(ws.data_ptr(), None), what)


class _Slot:
    """One side of the double buffer: pinned staging and device input, with
    events for the last copy in and the last kernel that read it."""

    def __init__(self, nbytes: int, device):
        self.pinned = torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)
        self.dev = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device)
        self.h2d_done = torch.cuda.Event()
        self.h2d_done.record()
        self.used = torch.cuda.Event()
        self.used.record()


def compress_files(in_paths, out_paths, group_bytes: int = 256 << 20, config: LaunchConfig | None = None,
                   device="cuda") -> dict:
    """Compresses each input file to a container file.  Returns byte counts."""
    if len(in_paths) != len(out_paths):
        raise ValueError("one output path per input path")
    dev = torch.device(device)
    sizes = [os.path.getsize(p) for p in in_paths]
    groups = _groups(sizes, group_bytes)
    cap = max(sum(sizes[i] for i in g) for g in groups) if groups else 0
    slots = [_Slot(cap, dev), _Slot(cap, dev)]
    copy_s = torch.cuda.Stream(device=dev)
    comp_s = torch.cuda.Stream(device=dev)
    io = ThreadPoolExecutor(max_workers=2)
    stats = {"files": len(in_paths), "bytes_in": sum(sizes), "bytes_out": 0}

    def read(k):
        slots[k % 2].h2d_done.synchronize()  # the previous H2D from this staging buffer is done
        return _read_into([in_paths[i] for i in groups[k]], slots[k % 2].pinned)

    def finish(g, plan, ent_host, ent_done):
        ent_done.synchronize()
        raw = ent_host.numpy().tobytes()
        ents = [BatchEntry.from_buffer_copy(raw[j * ENTRY_BYTES:(j + 1) * ENTRY_BYTES]) for j in range(len(g))]
        for e in ents:
            if e.status:
                check(int(e.status), "batched compress")
        wb = max((e.bits_offset + e.words for e in ents), default=0)
        gb = max((e.gaps_offset + e.gap_words for e in ents), default=0)
        bits_h = torch.empty(max(wb, 1), dtype=torch.int32, pin_memory=True)
        gaps_h = torch.empty(max(gb, 1), dtype=torch.int32, pin_memory=True)
        with torch.cuda.stream(copy_s):
            copy_s.wait_event(ent_done)  # this group's compress, not the next one's
            if wb:
                bits_h[:wb].copy_(plan.bits[:wb], non_blocking=True)
            if gb:
                gaps_h[:gb].copy_(plan.gaps[:gb], non_blocking=True)
        done = torch.cuda.Event()
        done.record(copy_s)
        done.synchronize()
        _status_after(plan.enc_ws, "batched compress (device)")
        bn = bits_h.numpy().view(np.uint32)
        gn = gaps_h.numpy().view(np.uint32)

        def write():
            out = 0
            for i, e in zip(g, ents):
                _write_container(out_paths[i], e, bn[e.bits_offset:e.bits_offset + e.words],
                                 gn[e.gaps_offset:e.gaps_offset + e.gap_words])
                out += _container_bytes(e)
            return out
        return io.submit(write)

    pending_read = io.submit(read, 0) if groups else None
    writes, prev = [], None
    for k, g in enumerate(groups):
        offs = pending_read.result()
        slot = slots[k % 2]
        n = sum(sizes[i] for i in g)
        with torch.cuda.stream(copy_s):
            copy_s.wait_event(slot.used)  # the compress that read this device buffer is done
            slot.dev[:n].copy_(slot.pinned[:n], non_blocking=True)
            slot.h2d_done.record(copy_s)
        if k + 1 < len(groups):
            pending_read = io.submit(read, k + 1)
        ins = [slot.dev[o:o + sizes[i]] for o, i in zip(offs, g)]
        with torch.cuda.stream(comp_s):
            comp_s.wait_event(slot.h2d_done)
            plan = BatchCodec([sizes[i] for i in g], config, device=dev)
            plan.bind(ins)
            plan.compress(stream=comp_s)
            ent_host = torch.empty(plan.entries.numel(), dtype=torch.uint8, pin_memory=True)
            ent_host.copy_(plan.entries, non_blocking=True)
            ent_done = torch.cuda.Event()
            ent_done.record(comp_s)
            slot.used.record(comp_s)
        if prev is not None:
            writes.append(finish(*prev))
        prev = (g, plan, ent_host, ent_done)
    if prev is not None:
        writes.append(finish(*prev))
    stats["bytes_out"] = sum(w.result() for w in writes)
    io.shutdown()
    return stats


def _parse(path):
    """A container file -> (entry without offsets, bits u32, gaps u32)."""
    raw = np.fromfile(path, np.uint8)
    cb = CCodebook()
    n, W, S = C.c_uint64(), C.c_uint64(), C.c_uint64()
    gp, bp = C.c_void_p(), C.c_void_p()
    check(lib().hgap_container_parse(raw.ctypes.data, raw.size, C.byref(cb), C.byref(n), C.byref(W), C.byref(S),
                                     C.byref(gp), C.byref(bp)), f"hgap_container_parse({path})")
    base = raw.ctypes.data
    G = (S.value + 7) // 8
    g0 = (gp.value or base) - base
    b0 = (bp.value or base) - base
    e = BatchEntry()
    e.n, e.words, e.segments, e.gap_words = n.value, W.value, S.value, G
    e.bits = W.value * 32
    e.symbol_count = cb.symbol_count
    C.memmove(C.addressof(e.symbols), C.addressof(cb.symbols), 2 * 256)
    return e, raw[b0:b0 + 4 * W.value], raw[g0:g0 + 4 * G]


def decompress_files(in_paths, out_paths, group_bytes: int = 256 << 20, config: LaunchConfig | None = None,
                     device="cuda") -> dict:
    """Decodes container files back to the original files."""
    if len(in_paths) != len(out_paths):
        raise ValueError("one output path per input path")
    dev = torch.device(device)
    csizes = [os.path.getsize(p) for p in in_paths]
    groups = _groups(csizes, group_bytes)
    copy_s = torch.cuda.Stream(device=dev)
    comp_s = torch.cuda.Stream(device=dev)
    io = ThreadPoolExecutor(max_workers=2)
    stats = {"files": len(in_paths), "bytes_in": sum(csizes), "bytes_out": 0}

    def load(k):
        """Parses a group's containers into pinned arenas and an entry table."""
        parsed = [_parse(in_paths[i]) for i in groups[k]]
        wsum = sum(((e.words + 3) // 4) * 4 for e, _, _ in parsed)
        gsum = sum(e.gap_words for e, _, _ in parsed)
        bits_h = torch.zeros(max(wsum, 4), dtype=torch.int32, pin_memory=True)
        gaps_h = torch.zeros(max(gsum, 1), dtype=torch.int32, pin_memory=True)
        bv = bits_h.numpy().view(np.uint8)
        gv = gaps_h.numpy().view(np.uint8)
        arr = (BatchEntry * len(parsed))()
        wo = go = 0
        for j, (e, b, g) in enumerate(parsed):
            e.bits_offset, e.gaps_offset = wo, go
            bv[4 * wo:4 * wo + b.size] = b
            gv[4 * go:4 * go + g.size] = g
            C.memmove(C.byref(arr[j]), C.byref(e), ENTRY_BYTES)
            wo += ((e.words + 3) // 4) * 4
            go += e.gap_words
        ent_h = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).pin_memory()
        return parsed, bits_h, gaps_h, ent_h

    def finish(g, parsed, outs, out_h, done, ws):
        done.synchronize()
        _status_after(ws, "batched decompress (device)")

        def write():
            tot = 0
            for i, (e, _, _), o in zip(g, parsed, outs):
                with open(out_paths[i], "wb") as f:
                    f.write(memoryview(out_h.numpy()[o:o + e.n]))
                tot += e.n
            return tot
        return io.submit(write)

    pending = io.submit(load, 0) if groups else None
    writes, prev = [], None
    for k, g in enumerate(groups):
        parsed, bits_h, gaps_h, ent_h = pending.result()
        if k + 1 < len(groups):
            pending = io.submit(load, k + 1)
        nouts = [int(e.n) for e, _, _ in parsed]
        total = sum(nouts)
        with torch.cuda.stream(copy_s):
            d_bits = bits_h.to(dev, non_blocking=True)
            d_gaps = gaps_h.to(dev, non_blocking=True)
            d_ent = ent_h.to(dev, non_blocking=True)
        for t in (d_bits, d_gaps, d_ent):
            t.record_stream(comp_s)  # read by the decompress on the other stream
        h2d = torch.cuda.Event()
        h2d.record(copy_s)
        with torch.cuda.stream(comp_s):
            comp_s.wait_event(h2d)
            out_d = torch.empty(max(total, 1), dtype=torch.uint8, device=dev)
            offs = np.concatenate([[0], np.cumsum(nouts)[:-1]]).astype(np.int64) if nouts else []
            d_out = torch.tensor([out_d.data_ptr() + int(o) for o in offs], dtype=torch.int64).to(dev)
            sz = np.array(nouts, np.uint64)
            nb = lib().hgap_batch_decompress_workspace_bytes(len(g), sz.ctypes.data_as(C.POINTER(C.c_uint64)))
            ws = torch.empty((nb + 7) // 8, dtype=torch.int64, device=dev)
            cfg = (config or LaunchConfig()).cstruct()
            check(lib().hgap_batch_decompress(len(g), d_ent.data_ptr(), d_bits.data_ptr(), d_gaps.data_ptr(),
                                              d_out.data_ptr(), ws.data_ptr(), ws.numel() * 8, C.byref(cfg),
                                              _stream(comp_s)), "hgap_batch_decompress")
            out_h = torch.empty(max(total, 1), dtype=torch.uint8, pin_memory=True)
            out_h.copy_(out_d, non_blocking=True)
            done = torch.cuda.Event()
            done.record(comp_s)
        if prev is not None:
            writes.append(finish(*prev))
        prev = (g, parsed, list(offs), out_h, done, ws)
        del d_bits, d_gaps, d_ent
    if prev is not None:
        writes.append(finish(*prev))
    stats["bytes_out"] = sum(w.result() for w in writes)
    io.shutdown()
    return stats


__all__ = ["compress_files", "decompress_files"]
