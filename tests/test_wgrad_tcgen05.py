"""The denoiser's weight gradient on the tcgen05 tensor cores against a plain PyTorch FP32 reference of the same op,
and a short training run with it.

The kernel reduces over pixels (M = output channels, N = input channels, K = pixels) from channel-major copies of
dY and of the column-shifted X; inputs are rounded to bf16 before the reference runs, so the remaining differences
are FP32 summation order, bounded as a fraction of the gradient's largest magnitude as for the other kernels."""
import numpy as np
import pytest

from test_denoiser import _bf16, _torch_conv

pytestmark = pytest.mark.gpu

# (N, H, W, Cin, Cout): image widths multiples of 8 and pixel counts multiples of 64, as the kernel needs
SHAPES = [(2, 16, 64, 32, 48), (1, 32, 32, 80, 16), (4, 8, 8, 224, 96), (8, 16, 16, 128, 128), (2, 24, 40, 16, 32)]


@pytest.fixture(scope="module")
def dn():
    from bluetruthengine_b200.denoiser import Denoiser
    return Denoiser()


@pytest.mark.parametrize("shape", SHAPES)
def test_weight_gradient_tcgen05_matches_torch(dn, shape):
    n, h, w, cin, cout = shape
    rng = np.random.default_rng(cin * 5 + cout)
    x = _bf16(rng.normal(size=(n, h, w, cin)))
    wt = _bf16(rng.normal(size=(9, cout, cin)) / np.sqrt(9 * cin))
    dy = _bf16(rng.normal(size=(n, h, w, cout)))
    got = dn.debug_conv(7, x=x, dy=dy, shape=shape)
    import torch
    _, wt_t, y = _torch_conv(x, wt, np.zeros(cout, np.float32))
    y.backward(torch.from_numpy(dy).permute(0, 3, 1, 2))
    ref_w = wt_t.grad.permute(2, 3, 0, 1).reshape(9, cout, cin).numpy()
    gw = got[:9 * cout * cin].reshape(9, cout, cin)
    ew = np.abs(gw - ref_w).max() / np.abs(ref_w).max()
    print("tcgen05 weight gradient", shape, ew)
    assert ew < 1e-3
    warp_level = dn.debug_conv(2, x=x, dy=dy, shape=shape)[:9 * cout * cin].reshape(9, cout, cin)
    assert np.abs(gw - warp_level).max() / np.abs(ref_w).max() < 1e-3


@pytest.mark.parametrize("kind", [2, 3, 4, 5, 6, 7])
def test_weight_gradient_tcgen05_pipeline_shapes(dn, kind):
    """Every pipeline shape of the tcgen05 weight gradient (stages, copy lag, pixels per stage, copy form) gives the
    same sums, on every test shape, two calls in a row."""
    try:
        dn.set_wgrad(kind)
        for shape in SHAPES:
            n, h, w, cin, cout = shape
            rng = np.random.default_rng(cin * 7 + cout + kind)
            x = _bf16(rng.normal(size=(n, h, w, cin)))
            dy = _bf16(rng.normal(size=(n, h, w, cout)))
            import torch
            wt = np.zeros((9, cout, cin), np.float32)
            _, wt_t, y = _torch_conv(x, wt, np.zeros(cout, np.float32))
            y.backward(torch.from_numpy(dy).permute(0, 3, 1, 2))
            ref_w = wt_t.grad.permute(2, 3, 0, 1).reshape(9, cout, cin).numpy()
            ref_b = dy.reshape(-1, cout).sum(0)
            for _ in range(2):
                got = dn.debug_conv(7, x=x, dy=dy, shape=shape)
                gw = got[:9 * cout * cin].reshape(9, cout, cin)
                gb = got[9 * cout * cin:]
                assert np.abs(gw - ref_w).max() / np.abs(ref_w).max() < 1e-3, (kind, shape)
                assert np.abs(gb - ref_b).max() / max(np.abs(ref_b).max(), 1e-6) < 1e-3, (kind, shape)
    finally:
        dn.set_wgrad(1)   # the default


def test_training_with_tcgen05_weight_gradient(dn):
    """The training loop with the tcgen05 weight gradient (the 48x48 crops and their 24x24 level take it; the
    smaller levels fall back) lowers the L1 loss as the warp-level kernel's run does."""
    rng = np.random.default_rng(3)
    S, H, W = 6, 64, 64
    yy, xx = np.mgrid[0:H, 0:W] / 64.0
    target = np.stack([np.stack([0.5 + 0.4 * np.sin(6 * xx + k), 0.3 + 0.2 * yy, 0.2 + 0.1 * np.cos(4 * yy + k)], -1)
                       for k in range(S)]).astype(np.float32)
    noisy = (target * rng.exponential(1.0, size=target.shape)).astype(np.float32)
    feat = np.concatenate([target / target.max(), np.broadcast_to([0, 1, 0], target.shape)], -1).astype(np.float32)
    losses = {}
    try:
        for kind in (0, 1):
            dn.set_wgrad(kind)
            dn.init(7)
            dn.set_dataset(noisy, feat, target)
            losses[kind] = dn.train(steps=60, batch=4, crop=48, lr=2e-3, seed=1)
    finally:
        dn.set_wgrad(1)   # the default
    for kind, loss in losses.items():
        print("wgrad kind", kind, "loss first/last", loss[:5].mean(), loss[-5:].mean())
        assert np.isfinite(loss).all() and loss[-5:].mean() < 0.7 * loss[:5].mean()
    assert abs(losses[1][-5:].mean() - losses[0][-5:].mean()) < 0.2 * losses[0][-5:].mean()
