"""The denoiser autotuner's host logic on the CPU, against a scripted stand-in for the denoiser: it picks the
fastest convolution kernels on inference and the fastest weight-gradient kernel on training steps (with the chosen
convolution kernels in force), leaves the denoiser in them, and puts the weights back after timing training.  The
calls it makes (set_tcgen05, set_wgrad, denoise, train, params, set_params) are each covered on the GPU by the
denoiser tests."""
import numpy as np

from bluetruthengine_b200.autotune import autotune_denoiser


class ScriptedDenoiser:
    """Device times per kernel choice; training moves the weights as a real step would."""

    def __init__(self, infer_ms, train_ms):
        self.infer_ms, self.train_ms = infer_ms, train_ms
        self.mode, self.kind, self.last = 2, 1, 0.0
        self.w = np.linspace(0, 1, 7).astype(np.float32)
        self.restored = 0
        self.train_modes = set()

    def set_tcgen05(self, mode):
        self.mode = mode

    def set_wgrad(self, kind):
        self.kind = kind

    def denoise(self, rad, feat):
        assert rad.shape[2] == 3 and feat.shape[2] == 6
        self.last = self.infer_ms[self.mode]

    def train(self, steps, batch, crop, lr, seed):
        self.train_modes.add(self.mode)
        self.last = self.train_ms[self.kind] * steps
        self.w = self.w + 0.5

    def last_ms(self):
        return self.last

    def params(self):
        return self.w.copy()

    def set_params(self, p):
        self.w = p.copy()
        self.restored += 1


def test_inference_only_picks_fastest_kernels():
    dn = ScriptedDenoiser({1: 3.0, 2: 1.2, 3: 1.3}, {})
    mode, kind, results = autotune_denoiser(dn, 64, 48, kernels=(2, 3, 1), iters=2)
    assert (mode, kind) == (2, None) and dn.mode == 2
    assert [(r.kernels, r.wgrad, r.ms) for r in results] == [(2, -1, 1.2), (3, -1, 1.3), (1, -1, 3.0)]
    assert dn.restored == 0


def test_training_kernels_timed_under_the_chosen_convolutions_and_weights_restored():
    dn = ScriptedDenoiser({1: 3.0, 2: 1.4, 3: 1.1}, {0: 5.6, 1: 4.02, 2: 4.03, 5: 4.01, 7: 4.05})
    w0 = dn.params()
    mode, kind, results = autotune_denoiser(dn, 32, 32, kernels=(2, 3, 1), wgrad=(1, 2, 5, 7, 0), train_steps=4)
    assert mode == 3 and kind == 5
    assert dn.mode == 3 and dn.kind == 5
    assert dn.train_modes == {3}
    assert np.array_equal(dn.params(), w0) and dn.restored == 1
    train = [r for r in results if r.wgrad >= 0]
    assert [r.wgrad for r in train] == [1, 2, 5, 7, 0]
    assert all(r.kernels == 3 for r in train)
    assert train[2].ms == 4.01
