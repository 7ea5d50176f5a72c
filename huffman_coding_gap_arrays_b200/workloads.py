"""Seeded synthetic byte streams with the shapes of the benchmark configs.

The reference ships no data; these generators stand in for it:

* ``zipf_buffer``      -- i.i.d. symbols, symbol = rank-1, P(rank) ~ rank^-s over 256 ranks
                          (16 MiB, s = 1.2: the small plain-method case);
* ``mixed_buffer``     -- 1 MiB blocks, each Zipf(1.05) or 8-bit quantised N(0,1)
                          (clamped to +-3 sigma, mapped to 0..255), chosen per block
                          by a hash of (seed, block) (1 GiB: the large single-buffer case);
* ``bf16_planes``      -- BF16 weights N(0, 0.02), split into the exponent byte
                          plane and the sign|mantissa byte plane;
* ``batch_sizes`` / ``batch_buffer`` -- log-uniform buffer sizes in [4 KiB, 4 MiB] with a
                          per-buffer Zipf(s ~ U[0.8,1.6]) or quantised Gaussian
                          (clamp(round(128 + sigma z)), sigma ~ U[0.5,4]) distribution.

All draw from torch generators on the requested device, so a 1 GiB buffer is
generated on the GPU in milliseconds; the CPU oracle receives the same bytes
after a copy.  Parity never depends on the generator.
"""
from __future__ import annotations

import math

import torch

MiB = 1 << 20


def _gen(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def _zipf_cdf(s: float, device) -> torch.Tensor:
    r = torch.arange(1, 257, dtype=torch.float64, device=device)
    p = r.pow(-s)
    c = torch.cumsum(p / p.sum(), 0)
    c[-1] = 1.0
    return c


def _zipf(n: int, s: float, g: torch.Generator, device) -> torch.Tensor:
    u = torch.rand(n, generator=g, device=device, dtype=torch.float64)
    idx = torch.searchsorted(_zipf_cdf(s, device), u, right=True)
    return idx.clamp_(max=255).to(torch.uint8)


def _gauss_q(n: int, g: torch.Generator, device) -> torch.Tensor:
    z = torch.randn(n, generator=g, device=device, dtype=torch.float32).clamp_(-3.0, 3.0)
    return torch.round((z + 3.0) / 6.0 * 255.0).to(torch.uint8)


def zipf_buffer(n: int, s: float = 1.2, seed: int = 1, device="cuda") -> torch.Tensor:
    return _zipf(n, s, _gen(seed, device), device)


def _block_kind(seed: int, block: int) -> int:
    # splitmix64 of (seed, block): 0 -> Zipf(1.05), 1 -> quantised Gaussian
    z = (seed * 0x9E3779B97F4A7C15 + block * 0xBF58476D1CE4E5B9 + 0x94D049BB133111EB) & (2**64 - 1)
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
    return (z ^ (z >> 31)) & 1


def mixed_buffer(n: int = 1 << 30, seed: int = 2, block: int = MiB, device="cuda") -> torch.Tensor:
    g = _gen(seed, device)
    nblk = (n + block - 1) // block
    kinds = torch.tensor([_block_kind(seed, b) for b in range(nblk)], dtype=torch.bool)
    out = torch.empty(n, dtype=torch.uint8, device=device)
    zi = torch.nonzero(~kinds).flatten().tolist()
    gi = torch.nonzero(kinds).flatten().tolist()
    for sel, make in ((zi, lambda m: _zipf(m, 1.05, g, device)), (gi, lambda m: _gauss_q(m, g, device))):
        if not sel:
            continue
        vals = make(len(sel) * block).view(len(sel), block)
        for j, b in enumerate(sel):
            lo = b * block
            hi = min(n, lo + block)
            out[lo:hi] = vals[j, :hi - lo]
    return out


def bf16_planes(count: int = 256 * MiB, seed: int = 3, device="cuda"):
    """(exponent plane, sign|mantissa plane) of `count` BF16 values N(0, 0.02)."""
    g = _gen(seed, device)
    w = torch.randn(count, generator=g, device=device, dtype=torch.float32).mul_(0.02)
    b = w.to(torch.bfloat16).view(torch.int16).to(torch.int32) & 0xFFFF
    exp = ((b >> 7) & 0xFF).to(torch.uint8)
    sm = (((b >> 15) << 7) | (b & 0x7F)).to(torch.uint8)
    return exp, sm


def batch_sizes(count: int = 4096, lo: int = 4096, hi: int = 4 * MiB, seed: int = 4) -> list[int]:
    g = _gen(seed, "cpu")
    u = torch.rand(count, generator=g, dtype=torch.float64)
    return [int(math.floor(math.exp(math.log(lo) + x * (math.log(hi) - math.log(lo))))) for x in u.tolist()]


def batch_buffer(size: int, seed: int, device="cuda") -> torch.Tensor:
    """One batched-workload buffer; its distribution is chosen by its seed."""
    g = _gen(seed, device)
    gc = _gen(seed, "cpu")
    kind, a = torch.rand(2, generator=gc, dtype=torch.float64).tolist()
    if kind < 0.5:
        return _zipf(size, 0.8 + 0.8 * a, g, device)
    sigma = 0.5 + 3.5 * a
    z = torch.randn(size, generator=g, device=device, dtype=torch.float32)
    return torch.round(128.0 + sigma * z).clamp_(0, 255).to(torch.uint8)
