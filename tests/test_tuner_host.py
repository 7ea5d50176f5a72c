"""Host logic of the learned tuner (no GPU): the memo that serving fills
before its clock starts must hold exactly the shapes `choose` picks."""
import numpy as np

from huffman_coding_gap_arrays_b200 import mlp as M


class _LinearNet:
    """A stand-in for one trained network: a fixed linear map of the inputs."""

    def __init__(self, seed):
        rng = np.random.default_rng(seed)
        self.w = rng.normal(size=(10, 2))

    def predict(self, X):
        X = np.asarray(X, np.float64)
        return np.stack([np.sin(X @ self.w[:, 0]), np.cos(X @ self.w[:, 1]) * X[:, 0] / 30], axis=1)


def test_precompute_equals_choose():
    t = M.LearnedTuner([_LinearNet(s) for s in (1, 2, 3)], margin=0.0, dec_margin=0.0)
    traffic = np.array([5.0, 13.0, 0.125], np.float32)
    for count in (0.0, 2.0, 5.0):
        t._memo.clear()
        t.precompute(traffic, 16.0, 26.0, count)
        memo = dict(t._memo)
        assert len(memo) == 81
        for key, cfg in memo.items():
            t._memo.clear()
            assert t.choose(np.array(key, np.float32)) == cfg, key


def test_set_default_forgets_the_memo():
    from huffman_coding_gap_arrays_b200.batch import LaunchConfig
    t = M.LearnedTuner([_LinearNet(s) for s in (1, 2)], margin=0.99, dec_margin=0.99)
    t.precompute(np.array([5.0, 13.0, 0.0], np.float32), 20.0, 21.0, 0.0)
    assert t._memo
    fixed = LaunchConfig(region_chunks=32, hist_ctas_per_sm=4, enc_ctas_per_sm=2)
    t.set_default(fixed)
    assert not t._memo
    # no candidate can beat a 99 % margin: the new default is kept
    assert t.choose(np.array([20.0, 5.0, 13.0, 0.0, 0.0], np.float32)) == fixed


def test_serving_batches_hit_the_precomputed_memo():
    """Every batch a serving run can form -- any 1..max_batch of its requests,
    any byte statistics -- quantizes to a memo entry the run filled before its
    clock started, so no batch waits for a forward pass."""
    from huffman_coding_gap_arrays_b200 import serve as S
    t = M.LearnedTuner([_LinearNet(s) for s in (4, 5)], margin=0.0, dec_margin=0.0)
    rng = np.random.default_rng(9)
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(64 << 10), np.log(64 << 20), 400))]
    max_batch = 48
    S.precompute_grid(t, sizes, max_batch)
    filled = dict(t._memo)
    assert filled
    for _ in range(2000):
        k = int(rng.integers(1, max_batch + 1))
        pick = rng.choice(len(sizes), size=k, replace=False)
        nb = np.array([sizes[i] for i in pick], np.float64)
        stats = np.stack([rng.uniform(0, 8.5, k), rng.uniform(1, 16, k), rng.uniform(0, 1, k) ** 3], axis=1)
        f = S.quantize_features(np.concatenate([[np.log2(nb.sum())], (nb[:, None] * stats).sum(0) / nb.sum(),
                                                [np.log2(k)]]))
        key = tuple((np.round(np.asarray(f, np.float32) * 8) / 8).tolist())
        assert key in filled, key
        assert t.choose(f) == filled[key]
    assert len(t._memo) == len(filled)  # nothing was added: every choice came from the memo
