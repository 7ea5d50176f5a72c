"""Generates the golden fixtures in this folder from the REFERENCE's own GPU
encoder (encoder/src/encoder.cu histgram() + encode(), compiled unmodified by
oracle/Makefile into oracle/_ref/libref_encoder.so) -- run once on a GPU host:

    python tests/golden/make_golden.py [outdir]

For every case in CASES the input is regenerated from (dist, n, seed) with
numpy, the codebook comes from the reference's own host code
(store_symbols + qsort(compare) + boundary_PM), and the reference GPU path
encodes it.  Small cases store the whole container (encoder/src/huff.cpp:
111-125 layout) as <name>.bin; every case stores sha256 digests of the
reference histogram, bitstream and gap array in golden.json.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

# (name, dist, n, seed); n >= 1 and at least two distinct symbols (the
# reference is undefined for fewer: histgram underflows at n = 0 and
# boundary_PM reads past one symbol).
CASES = [
    ("tiny_zipf_5", "zipf", 5, 1),
    ("zipf_1000", "zipf", 1000, 2),
    ("uniform_4099", "uniform", 4099, 3),
    ("two_8193", "two", 8193, 4),
    ("deep_20000", "deep", 20000, 5),
    ("zipf_65537", "zipf", 65537, 6),
    ("zipf_1M", "zipf", 1 << 20, 7),
    ("uniform_1M_plus_3", "uniform", (1 << 20) + 3, 8),
    ("deep_3M", "deep", 3 * (1 << 20) + 1, 9),
    ("zipf_16M", "zipf", 16 << 20, 1),
]
FULL_CONTAINER_MAX = 70_000


def make(dist: str, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if dist == "zipf":
        r = np.arange(1, 257); p = r ** -1.2; p /= p.sum()
        return rng.choice(256, size=n, p=p).astype(np.uint8)
    if dist == "uniform":
        return rng.integers(0, 256, size=n, dtype=np.uint8)
    if dist == "two":
        return rng.integers(0, 2, size=n, dtype=np.uint8)
    if dist == "deep":
        p = 1.0 / 1.618 ** np.arange(40); p /= p.sum()
        return (rng.choice(40, size=n, p=p).astype(np.uint8) * 5 + 3).astype(np.uint8)
    raise ValueError(dist)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(outdir: str) -> None:
    os.makedirs(outdir, exist_ok=True)
    manifest = {"generator": "reference GPU encoder (encoder/src/encoder.cu) via oracle/_ref",
                "cases": []}
    for name, dist, n, seed in CASES:
        x = make(dist, n, seed)
        cb = O.ref_codebook(O.histogram(x))
        hist, bits, gaps = O.ref_gpu_encode(x, cb)
        _, W, S, G = cb.sizes()
        entry = {"name": name, "dist": dist, "n": n, "seed": seed, "symbols": int(cb.count),
                 "max_len": int(cb.lengths.max()), "bits": cb.total_bits, "words": W,
                 "segments": S, "sha_hist": sha(hist), "sha_bits": sha(bits), "sha_gaps": sha(gaps)}
        if n <= FULL_CONTAINER_MAX:
            blob = O.container(cb, n, bits, gaps, S)
            with open(os.path.join(outdir, name + ".bin"), "wb") as f:
                f.write(blob)
            entry["container"] = name + ".bin"
            entry["sha_container"] = hashlib.sha256(blob).hexdigest()
        manifest["cases"].append(entry)
        print(name, W, S, entry["sha_bits"][:16], flush=True)
    with open(os.path.join(outdir, "golden.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
