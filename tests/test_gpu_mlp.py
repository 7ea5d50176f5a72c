"""The learned tuner on the GPU: its CUDA forward, gradient and Adam kernels
against the float64 oracle, and what the trained network gains over the
fixed default launch shape (compared with the exhaustive autotuner)."""
import numpy as np
import pytest
import torch

from huffman_coding_gap_arrays_b200 import batch as B
from huffman_coding_gap_arrays_b200 import mlp as ML
from huffman_coding_gap_arrays_b200 import tuner as TU
from huffman_coding_gap_arrays_b200 import workloads as WL
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _problem(seed, n):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, M.PARAMS).astype(np.float32)
    X = rng.normal(0, 1, (n, M.IN)).astype(np.float32)
    T = rng.normal(0, 1, (n, M.OUT)).astype(np.float32)
    T[rng.random(T.shape) < 0.2] = np.nan
    return p, X, T


@pytest.mark.parametrize("n", [1, 31, 300, 5000])
def test_forward_and_gradient_match_oracle(n):
    p, X, T = _problem(n, n)
    net = ML.LaunchMLP()
    net.params.copy_(torch.from_numpy(p))
    Xd = torch.from_numpy(X).cuda()
    Td = torch.from_numpy(T).cuda()
    y = net.forward_normalized(Xd).cpu().numpy()
    y_ref, _ = M.forward(p.astype(np.float64), X.astype(np.float64))
    assert np.allclose(y, y_ref, rtol=1e-4, atol=1e-4)
    scale = 1.0 / n
    loss, g = net.loss_grad_normalized(Xd, Td, scale)
    l_ref, g_ref = M.loss_grad(p.astype(np.float64), X.astype(np.float64), T.astype(np.float64), scale)
    assert abs(float(loss.item()) - l_ref) <= 1e-4 * max(1.0, abs(l_ref))
    g = g.cpu().numpy()
    assert np.allclose(g, g_ref, rtol=2e-3, atol=2e-5), float(np.abs(g - g_ref).max())


def test_adam_matches_oracle():
    p, X, T = _problem(7, 200)
    net = ML.LaunchMLP()
    net.params.copy_(torch.from_numpy(p))
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    pr, m, v = p.astype(np.float64), np.zeros(M.PARAMS), np.zeros(M.PARAMS)
    for k in range(1, 6):
        net.loss_grad_normalized(Xd, Td, 1 / 200)
        net.adam_step(1e-2, weight_decay=1e-3)
        _, g = M.loss_grad(pr, X.astype(np.float64), T.astype(np.float64), 1 / 200)
        pr, m, v = M.adam(pr, g, m, v, k, 1e-2, wd=1e-3)
    assert np.allclose(net.params.cpu().numpy(), pr, rtol=1e-3, atol=1e-4)


def test_training_fits_a_known_function():
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (2000, M.IN)).astype(np.float32)
    T = np.stack([np.sin(2 * X[:, 0]) + X[:, 4] ** 2, np.abs(X[:, 1]) - X[:, 5]], 1).astype(np.float32)
    net = ML.LaunchMLP(seed=1)
    losses = net.fit(X, T, steps=1500, lr=5e-3, weight_decay=0.0, log_every=100)
    assert losses[-1] < 0.05 * losses[0]
    P = net.predict(X)
    assert np.sqrt(np.mean((P - T) ** 2)) < 0.1


def _batch(count, hi, seed):
    sizes = WL.batch_sizes(count, lo=4096, hi=hi, seed=seed)
    return [WL.batch_buffer(n, seed * 7919 + i) for i, n in enumerate(sizes)]


# (count, largest buffer) of the batches: small requests up to the 4096-buffer mix
TRAIN = [(64, 64 << 10), (256, 256 << 10), (512, 1 << 20), (128, 4 << 20), (1024, 4 << 20), (2048, 1 << 20),
         (32, 16 << 20), (384, 2 << 20), (1536, 512 << 10), (768, 4 << 20), (96, 8 << 20), (2048, 4 << 20),
         (128, 128 << 10), (1024, 2 << 20), (3000, 4 << 20), (48, 32 << 20), (640, 1 << 20), (2600, 2 << 20),
         (200, 16 << 20), (4096, 4 << 20)]
HOLD = [(200, 2 << 20), (1200, 4 << 20)]
TEST = [(300, 1 << 20), (900, 4 << 20), (2500, 4 << 20), (150, 8 << 20), (1800, 2 << 20), (60, 16 << 20),
        (3500, 4 << 20), (500, 512 << 10)]


def _records(shapes, seed, reps=5):
    recs = []
    for k, (count, hi) in enumerate(shapes):
        bufs = _batch(count, hi, seed + k)
        outs = [torch.empty_like(b) for b in bufs]
        res = TU.Autotuner(reps=reps, warmup=2).tune(bufs, outs, TU.batch_features(bufs))
        assert all(torch.equal(o, b) for o, b in zip(outs, bufs))
        recs.extend(res.records)
        del bufs, outs
    return recs


def _measure(bufs, cfg, reps=5):
    outs = [torch.empty_like(b) for b in bufs]
    plan = B.BatchCodec([b.numel() for b in bufs], cfg)
    plan.bind(bufs, outs)
    c = TU._time(plan.compress, reps, 2)
    d = TU._time(plan.decompress, reps, 2)
    plan.check()
    assert all(torch.equal(o, b) for o, b in zip(outs, bufs))
    return c, d


def test_learned_tuner_gains_over_default():
    """Trained on the autotuner's records of one set of batches, the ensemble
    picks launch shapes for unseen batches that beat the fixed default shape
    and come close to the exhaustive autotuner's own measured best, without
    measuring anything."""
    recs = _records(TRAIN, 500)
    hold = _records(HOLD, 600)
    lt = ML.LearnedTuner.train(recs, holdout=hold, steps=3000)
    assert lt.usable, lt.holdout_rmse
    tot = {"mlp": 0.0, "default": 0.0, "best": 0.0}
    comp = {"mlp": 0.0, "default": 0.0, "best": 0.0}
    for k, (count, hi) in enumerate(TEST):
        bufs = _batch(count, hi, 700 + k)
        f = TU.batch_features(bufs)
        best = TU.Autotuner(reps=3, warmup=1).tune(bufs, [torch.empty_like(b) for b in bufs], f)
        pick = lt.choose(f)
        row = {}
        for key, cfg in (("mlp", pick), ("default", B.LaunchConfig()), ("best", best.config)):
            c, d = _measure(bufs, cfg)
            tot[key] += c + d
            comp[key] += c
            row[key] = (vars(cfg), round(c, 3), round(d, 3))
        print(count, hi, row)
        del bufs
    print("learned tuner totals (ms):", {k: round(v, 4) for k, v in tot.items()}, "compress",
          {k: round(v, 4) for k, v in comp.items()}, "holdout rmse", round(lt.holdout_rmse, 4))
    assert comp["mlp"] < 0.97 * comp["default"], comp       # the shape choice that matters: compress
    assert tot["mlp"] < tot["default"], tot                 # and nothing lost on the whole round trip
    assert tot["mlp"] <= 1.05 * tot["best"], tot
