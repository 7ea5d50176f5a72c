"""Learned launch tuner: a small MLP, trained and run on the GPU by the
project's own CUDA kernels (csrc/mlp.cu), that predicts how the batched
compress and decompress times of an input (a batch of buffers, or one buffer)
move with the launch shape.

    X = [log2 size, entropy, longest code, level-2 byte fraction,
         log2 buffer count,                                              (input)
         log2 region chunks, histogram / encoder / decoder CTAs per SM,
         decoder tile (-1: 256 segments, 0: by the book, 1: 512)]          (shape)
    y = [log compress ms, log decompress ms], each relative to the mean over
        the shapes measured on the same input: only the ranking of shapes for
        one input matters, and the size effect would otherwise swamp it.

It is trained on the autotuner's own records (``tuner.Autotuner``).
``LearnedTuner.choose`` scores every candidate shape with a forward pass of an
ensemble of networks (one per seed) and keeps the default shape unless a
candidate that every network predicts faster has a mean predicted gain above
a margin -- the exhaustive autotuner's pick without its measurements.  It only chooses launch shapes, which leave the
output format unchanged.  Untrained, or with a held-out error above its
limit, it falls back to running the autotuner.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from ._lib import MLP_IN, MLP_OUT, MLP_PARAMS, check, lib
from .batch import LaunchConfig
from .codec import _stream
from .tuner import DEC_SPACE, Autotuner, compress_space, with_dec

SHAPES = [(32, 10), (32,), (32, 32), (32,), (2, 32), (2,)]
# CTAs per SM that "0" (the occupancy maximum) means for each grid on B200
MAX_CTAS = {"hist": 4, "enc": 2, "dec": 5}  # what 0 (the occupancy maximum) stands for in the features


TILE_CODE = {0: 0.0, 256: -1.0, 512: 1.0}


def config_vector(cfg: LaunchConfig) -> np.ndarray:
    return np.array([math.log2(max(cfg.region_chunks, 1)),
                     cfg.hist_ctas_per_sm or MAX_CTAS["hist"],
                     cfg.enc_ctas_per_sm or MAX_CTAS["enc"],
                     cfg.dec_ctas_per_sm or MAX_CTAS["dec"],
                     TILE_CODE.get(cfg.dec_tile_segs, 0.0)], np.float32)


def records_to_xy(records, relative: bool = True):
    """Autotuner records -> (X n x 10, T n x 2 log-ms targets, NaN = not
    measured).  With `relative`, each target is taken relative to the mean
    log time of the records with the same features (one tuned input)."""
    X = np.stack([np.concatenate([r.features, config_vector(r.config)]) for r in records]).astype(np.float32)
    T = np.stack([[math.log(r.compress_ms) if r.compress_ms == r.compress_ms else np.nan,
                   math.log(r.decompress_ms) if r.decompress_ms == r.decompress_ms else np.nan]
                  for r in records]).astype(np.float64)
    if relative:
        keys = [tuple(np.round(r.features, 5).tolist()) for r in records]
        for k in set(keys):
            idx = np.array([i for i, kk in enumerate(keys) if kk == k])
            for o in range(T.shape[1]):
                col = T[idx, o]
                ok = np.isfinite(col)
                if ok.any():
                    T[idx[ok], o] = col[ok] - col[ok].mean()
    return X, T.astype(np.float32)


class LaunchMLP:
    """Parameters, Adam state and input normalisation on the device; every
    forward, gradient and update is a libhgap.so kernel."""

    def __init__(self, seed: int = 0, device="cuda"):
        self.device = torch.device(device)
        rng = np.random.default_rng(seed)
        parts = []
        for shape in SHAPES:
            if len(shape) == 2:
                parts.append(rng.normal(0, math.sqrt(2.0 / shape[1]), shape).reshape(-1))
            else:
                parts.append(np.zeros(shape))
        p = np.concatenate(parts).astype(np.float32)
        assert p.size == MLP_PARAMS
        self.params = torch.from_numpy(p).to(self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.step = 0
        self.mean = np.zeros(MLP_IN, np.float32)
        self.std = np.ones(MLP_IN, np.float32)

    def _upload(self, X) -> torch.Tensor:
        Xn = ((np.asarray(X, np.float32) - self.mean) / self.std).astype(np.float32)
        return torch.from_numpy(np.ascontiguousarray(Xn)).to(self.device)

    def forward_normalized(self, Xn: torch.Tensor, stream=None) -> torch.Tensor:
        Y = torch.empty(Xn.shape[0], MLP_OUT, dtype=torch.float32, device=self.device)
        check(lib().hgap_mlp_forward(self.params.data_ptr(), Xn.data_ptr(), Xn.shape[0], Y.data_ptr(),
                                     _stream(stream)), "hgap_mlp_forward")
        return Y

    def predict(self, X) -> np.ndarray:
        """Predicted [log compress ms, log decompress ms] per row of raw inputs."""
        return self.forward_normalized(self._upload(X)).cpu().numpy()

    def loss_grad_normalized(self, Xn: torch.Tensor, T: torch.Tensor, scale: float, stream=None):
        check(lib().hgap_mlp_loss_grad(self.params.data_ptr(), Xn.data_ptr(), T.data_ptr(), Xn.shape[0],
                                       float(scale), self.grad.data_ptr(), self.loss.data_ptr(),
                                       _stream(stream)), "hgap_mlp_loss_grad")
        return self.loss, self.grad

    def adam_step(self, lr: float, b1=0.9, b2=0.999, eps=1e-8, weight_decay=0.0, stream=None) -> None:
        self.step += 1
        check(lib().hgap_mlp_adam(self.params.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                                  self.v.data_ptr(), self.step, lr, b1, b2, eps, weight_decay, _stream(stream)),
              "hgap_mlp_adam")

    def fit(self, X, T, steps: int = 3000, lr: float = 3e-3, weight_decay: float = 1e-3,
            log_every: int = 0) -> list:
        """Full-batch Adam on the mean squared error of the targets plus a small
        L2 term (timings are noisy; cross-validation over recorded batches
        picked 1e-3), with the learning rate decaying tenfold over the run."""
        X = np.asarray(X, np.float32)
        T = np.asarray(T, np.float32)
        self.mean = X.mean(0).astype(np.float32)
        self.std = (X.std(0) + 1e-3).astype(np.float32)
        Xn = self._upload(X)
        Td = torch.from_numpy(np.ascontiguousarray(T)).to(self.device)
        scale = 1.0 / max(1, int(np.isfinite(T).sum()))
        losses = []
        for k in range(steps):
            self.loss_grad_normalized(Xn, Td, scale)
            self.adam_step(lr * (0.1 ** (k / max(steps, 1))), weight_decay=weight_decay)
            if log_every and (k % log_every == 0 or k == steps - 1):
                losses.append(float(self.loss.item()))
        if not losses:
            losses.append(float(self.loss.item()))
        return losses


class LearnedTuner:
    """Chooses a launch shape per input from the predictions of an ensemble of
    MLPs, with the exhaustive autotuner as the fallback."""

    def __init__(self, mlps=None, space=None, dec_space=DEC_SPACE, max_rmse: float = 0.3,
                 margin: float = 0.03, dec_margin: float = 0.05, default: LaunchConfig | None = None):
        self.mlps = list(mlps) if mlps else []
        self.space = list(space) if space is not None else compress_space()
        self.dec_space = tuple(dec_space)
        self.max_rmse = max_rmse
        self.margin = margin
        self.dec_margin = dec_margin  # the decoder grid moves decompress time little: be stricter
        self.default = default or LaunchConfig()
        self.holdout_rmse = float("inf")
        self._memo = {}  # choices by features rounded to 1/8: a serving loop asks about the same sizes

    @classmethod
    def train(cls, records, holdout=None, seeds=(0, 1, 2), steps: int = 3000, **kw) -> "LearnedTuner":
        X, T = records_to_xy(records)
        mlps = []
        for sd in seeds:
            m = LaunchMLP(sd)
            m.fit(X, T, steps=steps)
            mlps.append(m)
        t = cls(mlps, **kw)
        Xh, Th = records_to_xy(holdout) if holdout else (X, T)
        P = t.predict(Xh)
        ok = np.isfinite(Th)
        t.holdout_rmse = float(np.sqrt(np.mean((P[ok] - Th[ok]) ** 2))) if ok.any() else float("inf")
        return t

    def set_default(self, cfg: LaunchConfig) -> None:
        """The shape kept unless a candidate is predicted faster by the margin
        (e.g. the exhaustive search's pick for the workload); forgets the memo."""
        self.default = cfg
        self._memo.clear()

    def predict(self, X) -> np.ndarray:
        return np.mean([m.predict(X) for m in self.mlps], axis=0)

    @property
    def usable(self) -> bool:
        return bool(self.mlps) and self.holdout_rmse <= self.max_rmse

    def _pick(self, f, cands, default, out: int, margin: float):
        """Among the candidates that every member of the ensemble predicts
        faster than the default, the one with the best mean prediction --
        taken only if that mean gain exceeds the margin."""
        X = np.stack([np.concatenate([f, config_vector(c)]) for c in list(cands) + [default]])
        P = np.stack([m.predict(X)[:, out] for m in self.mlps])  # members x (candidates + default)
        rel = P[:, :-1] - P[:, -1:]                               # log time relative to the default
        mean = np.where((rel < 0).all(axis=0), rel.mean(axis=0), np.inf)
        i = int(np.argmin(mean))
        return cands[i] if mean[i] < math.log(1.0 - margin) else default

    def choose(self, features) -> LaunchConfig:
        """The compress shape with the least predicted compress time, then the
        decoder grid with the least predicted decompress time."""
        f = np.round(np.asarray(features, np.float32) * 8) / 8
        key = tuple(f.tolist())
        if key in self._memo:
            return self._memo[key]
        d0 = self.default
        d0dec = (d0.dec_ctas_per_sm, d0.dec_tile_segs)
        c = self._pick(f, self.space, with_dec(d0, d0dec), 0, self.margin)
        dec = [with_dec(c, d) for d in self.dec_space]
        dd = with_dec(c, d0dec)
        pick = self._pick(f, dec, dd, 1, self.dec_margin)
        self._memo[key] = pick
        return pick

    def precompute(self, traffic, log2_lo: float, log2_hi: float, log2_count: float = 0.0) -> None:
        """Fills the memo for every input size from 2^log2_lo to 2^log2_hi (in
        the memo's 1/8 steps) for fixed byte statistics and buffer count, with
        one forward pass per network -- so that a serving loop never waits for one."""
        keys = np.arange(np.floor(log2_lo * 8) / 8, np.ceil(log2_hi * 8) / 8 + 1e-9, 0.125)
        if not len(keys) or not self.mlps:
            return
        d0 = self.default
        comp = list(self.space)
        d0dec = (d0.dec_ctas_per_sm, d0.dec_tile_segs)
        base = with_dec(d0, d0dec)
        rest = np.round(np.concatenate([np.asarray(traffic, np.float32), [log2_count]]) * 8) / 8
        feats = np.concatenate([keys[:, None], np.tile(rest, (len(keys), 1))], axis=1).astype(np.float32)
        nf = len(feats)

        def rows(cfg_vecs):  # every feature row against every config row (per feature, in order)
            k = cfg_vecs.shape[-2]
            F = np.repeat(feats, k, axis=0)
            Cv = cfg_vecs.reshape(-1, cfg_vecs.shape[-1]) if cfg_vecs.ndim == 3 else np.tile(cfg_vecs, (nf, 1))
            return np.concatenate([F, Cv], axis=1)

        def best(P, k, margin):  # per feature row: the candidate index, or k (the default)
            rel = P[:, :, :k] - P[:, :, k:k + 1]
            mean = np.where((rel < 0).all(axis=0), rel.mean(axis=0), np.inf)
            i = np.argmin(mean, axis=1)
            return np.where(mean[np.arange(nf), i] < math.log(1.0 - margin), i, k)

        # stage 1: the compress shape for every size at once
        cands = comp + [base]
        V = np.stack([config_vector(c) for c in cands])
        P = np.stack([m.predict(rows(V))[:, 0] for m in self.mlps]).reshape(len(self.mlps), nf, len(cands))
        picks = [cands[i] for i in best(P, len(comp), self.margin)]
        # stage 2: the decoder grid for each size's compress shape
        dec = [[with_dec(c, d) for d in self.dec_space] + [with_dec(c, d0dec)] for c in picks]
        V = np.stack([np.stack([config_vector(c) for c in row]) for row in dec])
        nd = len(self.dec_space) + 1
        P = np.stack([m.predict(rows(V))[:, 1] for m in self.mlps]).reshape(len(self.mlps), nf, nd)
        for j, i in enumerate(best(P, nd - 1, self.dec_margin)):
            self._memo[tuple(feats[j].tolist())] = dec[j][i]

    def choose_or_search(self, features, inputs, outputs) -> LaunchConfig:
        """The ensemble's pick when it is trained and accurate enough on
        held-out records; otherwise the exhaustive autotuner on these buffers."""
        if self.usable:
            return self.choose(features)
        return Autotuner(space=self.space, dec_space=self.dec_space).tune(inputs, outputs, features).config


__all__ = ["LaunchMLP", "LearnedTuner", "config_vector", "records_to_xy"]
