"""The denoiser trainer's chunk loop on the host (no GPU): the weights of the best chunk are kept, and a chunk whose
loss blows up returns to them with half the learning rate."""
import numpy as np

from bluetruthengine_b200.train_denoiser import train_chunks


class FakeNet:
    """Stands in for Denoiser: its 'weights' are one number, each chunk's loss is a scripted value, and a
    blow-up is planted in the script (the losses a diverged Adam run produces)."""

    def __init__(self, chunk_losses):
        self.script = list(chunk_losses)
        self.w = np.zeros(1, np.float32)
        self.lrs, self.restored = [], []

    def train(self, steps, batch, crop, lr, seed):
        self.lrs.append(lr)
        self.w = self.w + 1.0          # every chunk moves the weights
        return np.full(steps, self.script.pop(0), np.float32)

    def params(self):
        return self.w.copy()

    def set_params(self, p):
        self.restored.append(float(p[0]))
        self.w = np.array(p, np.float32)

    def last_ms(self):
        return 1.0


def test_best_weights_kept_and_blowup_rolled_back():
    # chunks 1-4 improve, chunk 5 blows up (0.050 > 1.5 x 0.020), chunks 6-8 recover
    net = FakeNet([0.040, 0.030, 0.025, 0.020, 0.050, 0.019, 0.018, 0.0185])
    p, losses, best, best_step, rollbacks = train_chunks(net, 8 * 250, 8, 128, 1e-3, 1)
    assert rollbacks == 1
    assert net.restored == [4.0]                 # the weights after chunk 4 (the best before the blow-up)
    assert net.lrs[5] == 5e-4 and net.lrs[4] == 1e-3   # half the rate after the rollback
    assert best == np.float32(0.018) and best_step == 7 * 250
    assert float(p[0]) == 6.0                    # chunk 7's weights: restored 4, then chunks 6 and 7
    assert len(losses) == 8 * 250


def test_last_fifth_runs_at_a_tenth():
    net = FakeNet([0.05 - 0.001 * i for i in range(10)])
    train_chunks(net, 10 * 250, 8, 128, 1e-3, 1)
    assert net.lrs[:8] == [1e-3] * 8 and all(abs(x - 1e-4) < 1e-12 for x in net.lrs[8:])
