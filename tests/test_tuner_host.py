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
