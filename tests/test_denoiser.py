"""The denoiser's tensor-core kernels against a plain PyTorch FP32 reference of the same op, and its
training / inference path end to end.

Inputs are rounded to bf16 before the FP32 reference runs, so the reference sees exactly the operands
the kernels see; the remaining differences are FP32 summation order and the bf16 rounding of the
kernels' outputs, bounded below as a fraction of the output's largest magnitude."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# small shapes run the tap-split kernel, the last (3 x 300 x 4 = 3600 CTAs of 64 pixels) the unsplit one
SHAPES = [(2, 20, 37, 32, 48), (1, 16, 64, 16, 32), (1, 9, 70, 224, 96), (2, 8, 24, 80, 16), (4, 300, 130, 32, 48),
          (1, 12, 150, 112, 48), (1, 10, 140, 96, 128), (1, 10, 140, 32, 16)]


def _bf16(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).to(torch.float32).numpy()


def _torch_conv(x, w, bias=None):
    """x [N,H,W,Cin], w [9][Cout][Cin] -> y [N,H,W,Cout] in FP32 (cross-correlation, zero padding)."""
    import torch
    cout, cin = w.shape[1], w.shape[2]
    wt = torch.from_numpy(w).reshape(3, 3, cout, cin).permute(2, 3, 0, 1).contiguous()
    xt = torch.from_numpy(x).permute(0, 3, 1, 2).contiguous().requires_grad_(True)
    wt.requires_grad_(True)
    y = torch.nn.functional.conv2d(xt, wt, None if bias is None else torch.from_numpy(bias), padding=1)
    return xt, wt, y


@pytest.fixture(scope="module")
def dn():
    from bluetruthengine_b200.denoiser import Denoiser
    return Denoiser()


KERNEL_OPS = {"mma": (0, 1), "tcgen05": (3, 4), "tcgen05_row": (5, 6)}


def _row_ok(cin, cout):
    """Shapes the row-tile kernel takes: Cout 16..64 in steps of 16, 96 or 128, Cin in 16-channel steps (a layer whose
    weights and slabs do not fit shared memory at once runs in passes, e.g. Cin 112 -> Cout 48)."""
    return cout in (16, 32, 48, 64, 96, 128) and cin % 16 == 0


@pytest.mark.parametrize("kernel", ["mma", "tcgen05", "tcgen05_row"])
@pytest.mark.parametrize("shape", SHAPES)
def test_conv_forward_matches_torch(dn, shape, kernel):
    """Forward 3x3 conv + bias + ReLU: warp-level MMA kernel, tcgen05 pixel-tile and row-tile kernels."""
    n, h, w, cin, cout = shape
    if kernel == "tcgen05_row" and not _row_ok(cin, cout):
        pytest.skip("layer outside the row-tile kernel's shapes")
    rng = np.random.default_rng(cin * 7 + cout)
    x = _bf16(rng.normal(size=(n, h, w, cin)))
    wt = _bf16(rng.normal(size=(9, cout, cin)) / np.sqrt(9 * cin))
    b = rng.normal(size=cout).astype(np.float32)
    got = dn.debug_conv(KERNEL_OPS[kernel][0], x=x, w=wt, bias=b, shape=shape, relu=True)
    _, _, y = _torch_conv(x, wt, b)
    ref = np.maximum(y.detach().permute(0, 2, 3, 1).numpy(), 0.0)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print("forward", kernel, shape, "max error / max |y|", err)
    assert err < 1e-2


@pytest.mark.parametrize("kernel", ["mma", "tcgen05", "tcgen05_row"])
@pytest.mark.parametrize("shape", SHAPES)
def test_conv_data_gradient_matches_torch(dn, shape, kernel):
    n, h, w, cin, cout = shape
    if kernel == "tcgen05_row" and not _row_ok(cout, cin):
        pytest.skip("layer outside the row-tile kernel's shapes")
    rng = np.random.default_rng(cin * 5 + cout)
    x = _bf16(rng.normal(size=(n, h, w, cin)))
    wt = _bf16(rng.normal(size=(9, cout, cin)) / np.sqrt(9 * cin))
    dy = _bf16(rng.normal(size=(n, h, w, cout)))
    got = dn.debug_conv(KERNEL_OPS[kernel][1], w=wt, dy=dy, shape=shape)
    import torch
    xt, wt_t, y = _torch_conv(x, wt)
    y.backward(torch.from_numpy(dy).permute(0, 3, 1, 2))
    ref = xt.grad.permute(0, 2, 3, 1).numpy()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print("data gradient", kernel, shape, err)
    assert err < 1e-2


@pytest.mark.parametrize("shape", SHAPES)
def test_conv_weight_gradient_matches_torch(dn, shape):
    n, h, w, cin, cout = shape
    rng = np.random.default_rng(cin * 3 + cout)
    x = _bf16(rng.normal(size=(n, h, w, cin)))
    wt = _bf16(rng.normal(size=(9, cout, cin)) / np.sqrt(9 * cin))
    dy = _bf16(rng.normal(size=(n, h, w, cout)))
    got = dn.debug_conv(2, x=x, dy=dy, shape=shape)
    import torch
    xt, wt_t, y = _torch_conv(x, wt, np.zeros(cout, np.float32))
    y.backward(torch.from_numpy(dy).permute(0, 3, 1, 2))
    ref_w = wt_t.grad.permute(2, 3, 0, 1).reshape(9, cout, cin).numpy()
    ref_b = dy.reshape(-1, cout).sum(0)
    gw = got[:9 * cout * cin].reshape(9, cout, cin)
    gb = got[9 * cout * cin:]
    ew = np.abs(gw - ref_w).max() / np.abs(ref_w).max()
    eb = np.abs(gb - ref_b).max() / max(np.abs(ref_b).max(), 1e-6)
    print("weight gradient", shape, ew, eb)
    assert ew < 1e-3 and eb < 1e-3


def test_training_reduces_loss_and_denoise_runs(dn):
    """A short training run on synthetic pairs (smooth targets, noisy inputs) lowers the L1 loss; the
    trained network then denoises an image of a size that is not a multiple of 16."""
    rng = np.random.default_rng(3)
    S, H, W = 6, 64, 64
    yy, xx = np.mgrid[0:H, 0:W] / 64.0
    target = np.stack([np.stack([0.5 + 0.4 * np.sin(6 * xx + k), 0.3 + 0.2 * yy, 0.2 + 0.1 * np.cos(4 * yy + k)], -1)
                       for k in range(S)]).astype(np.float32)
    noisy = (target * rng.exponential(1.0, size=target.shape)).astype(np.float32)
    feat = np.concatenate([target / target.max(), np.broadcast_to([0, 1, 0], target.shape)], -1).astype(np.float32)
    dn.init(7)
    dn.set_dataset(noisy, feat, target)
    loss = dn.train(steps=60, batch=4, crop=48, lr=2e-3, seed=1)
    print("loss first/last", loss[:5].mean(), loss[-5:].mean())
    assert np.isfinite(loss).all() and loss[-5:].mean() < 0.7 * loss[:5].mean()
    out = dn.denoise(noisy[0, :50, :61], feat[0, :50, :61])
    assert out.shape == (50, 61, 3) and np.isfinite(out).all() and (out >= 0).all()
    from bluetruthengine_b200.denoiser import rel_mse
    assert rel_mse(out, target[0, :50, :61]) < rel_mse(noisy[0, :50, :61], target[0, :50, :61])
    p = dn.params()
    dn.set_params(p)
    assert np.array_equal(dn.params(), p)


def test_renderer_denoiser_toggle(dn, bte, cornell_scene):
    """cudaToggleDenoiser path: with weights loaded, each frame presents the denoised accumulation
    (read back as floats and as the packed framebuffer); plain accumulation is unchanged by it."""
    from conftest import bits
    r = bte.Renderer()
    sc = cornell_scene
    W, H = sc.width, sc.height
    r.cleanup()
    r.upload(sc)
    r.set_config(samples_per_frame=2, max_depth=6, rr_start=3, env_sampling=0)
    r.reset_accumulation(W, H)
    r.render(W, H)
    plain = r.read_accum(W, H).copy()
    dn.init(5)
    assert r.toggle_denoiser() is True
    r.reset_accumulation(W, H)
    r.render(W, H)
    acc = r.read_accum(W, H)
    den = r.read_denoised(W, H)
    fb = r.read_framebuffer(W, H)
    feat = np.concatenate(r.read_aov(W, H), -1)
    assert r.toggle_denoiser() is False
    assert np.array_equal(bits(plain), bits(acc))
    assert den.shape == (H, W, 3) and np.isfinite(den).all()
    assert np.array_equal(den, dn.denoise(acc.reshape(H, W, 3), feat))
    assert fb.size == W * H


CONVS = [(16, 32), (32, 32), (32, 48), (48, 48), (48, 64), (64, 64), (64, 96), (96, 96), (96, 128), (128, 128),
         (224, 96), (96, 96), (160, 64), (64, 64), (112, 48), (48, 48), (80, 32), (32, 32), (32, 16)]


def _torch_unet(params, rad, feat):
    """The denoiser's network in PyTorch FP32, rounding activations to bf16 where the kernels store them."""
    import torch
    import torch.nn.functional as F
    bf = lambda t: t.to(torch.bfloat16).to(torch.float32)
    H, W = rad.shape[:2]
    Hp, Wp = (H + 15) // 16 * 16, (W + 15) // 16 * 16
    pad = lambda a: np.pad(a, ((0, Hp - H), (0, Wp - W), (0, 0)), mode="edge")
    x = np.concatenate([np.log1p(np.maximum(pad(rad), 0)), pad(feat), np.zeros((Hp, Wp, 7), np.float32)], -1)
    x = bf(torch.from_numpy(x.astype(np.float32)).permute(2, 0, 1)[None])
    ws, off = [], 0
    for cin, cout in CONVS:
        w = torch.from_numpy(params[off:off + 9 * cout * cin].reshape(3, 3, cout, cin)).permute(2, 3, 0, 1)
        off += 9 * cout * cin
        b = torch.from_numpy(params[off:off + cout])
        off += cout
        ws.append((bf(w), b))
    conv = lambda t, i, relu=True: bf(F.relu(F.conv2d(t, *ws[i], padding=1)) if relu else F.conv2d(t, *ws[i], padding=1))
    pool = lambda t: bf(F.avg_pool2d(t, 2))
    up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")
    e0 = conv(conv(x, 0), 1)
    e1 = conv(conv(pool(e0), 2), 3)
    e2 = conv(conv(pool(e1), 4), 5)
    e3 = conv(conv(pool(e2), 6), 7)
    e4 = conv(conv(pool(e3), 8), 9)
    d3 = conv(conv(torch.cat([up(e4), e3], 1), 10), 11)
    d2 = conv(conv(torch.cat([up(d3), e2], 1), 12), 13)
    d1 = conv(conv(torch.cat([up(d2), e1], 1), 14), 15)
    d0 = conv(conv(torch.cat([up(d1), e0], 1), 16), 17)
    out = conv(d0, 18, relu=False)
    pred = out[0, :3] + x[0, :3]
    return np.maximum(np.expm1(pred.permute(1, 2, 0).numpy()), 0)[:H, :W]


@pytest.mark.parametrize("tc", [0, 2, 3])
@pytest.mark.parametrize("size", [(72, 100), (470, 640)])
def test_network_inference_matches_torch(dn, size, tc):
    """The whole inference path (feature assembly, edge padding, encoder, in-place upsample+concat decoder,
    residual output) against the same network written in PyTorch, on a random network; the larger size
    runs the full-resolution layers on the unsplit warp-level kernel (tc 0) or on the tcgen05 row-tile
    kernel, the upsample + concat layers included, upsampled beforehand (tc 2) or inside the kernel (tc 3)."""
    dn.init(11)
    p = dn.params()
    rng = np.random.default_rng(5)
    H, W = size
    rad = rng.exponential(0.4, size=(H, W, 3)).astype(np.float32)
    feat = np.concatenate([rng.uniform(0, 1, (H, W, 3)), rng.normal(size=(H, W, 3))], -1).astype(np.float32)
    dn.set_tcgen05(tc)
    try:
        got = dn.denoise(rad, feat)
    finally:
        dn.set_tcgen05(2)   # the default
    ref = _torch_unet(p, rad, feat)
    lg, lr = np.log1p(got), np.log1p(ref)
    err = np.abs(lg - lr)
    print("log-space error max", err.max(), "mean", err.mean())
    assert err.mean() < 5e-3 and err.max() < 0.1


@pytest.mark.parametrize("tc", [2, 3])
@pytest.mark.parametrize("size", [(560, 720), (976, 1280)])
def test_network_inference_row_passes_match_torch(dn, size, tc):
    """The row-tile kernel on layers that run in passes over their input channels with FP32 partial sums:
    at these sizes the level-1 decoder layer (upsampled 64 + 48 channels -> 48) and, at the larger one,
    the level-2 decoder layer (upsampled 96 + 64 -> 64) are large enough for the tensor-core path."""
    dn.init(13)
    p = dn.params()
    rng = np.random.default_rng(9)
    H, W = size
    rad = rng.exponential(0.4, size=(H, W, 3)).astype(np.float32)
    feat = np.concatenate([rng.uniform(0, 1, (H, W, 3)), rng.normal(size=(H, W, 3))], -1).astype(np.float32)
    dn.set_tcgen05(tc)
    try:
        got = dn.denoise(rad, feat)
    finally:
        dn.set_tcgen05(2)   # the default
    ref = _torch_unet(p, rad, feat)
    err = np.abs(np.log1p(got) - np.log1p(ref))
    print("log-space error max", err.max(), "mean", err.mean())
    assert err.mean() < 5e-3 and err.max() < 0.1


def test_inference_replay_across_sizes(dn):
    """The inference sequence is replayed from a CUDA graph per image size and buffer set: after a larger image
    has reallocated the activations and scratch buffers, the first size must give the same bits as before."""
    dn.init(17)
    rng = np.random.default_rng(3)
    def pair(H, W):
        rad = rng.exponential(0.4, size=(H, W, 3)).astype(np.float32)
        feat = np.concatenate([rng.uniform(0, 1, (H, W, 3)), rng.normal(size=(H, W, 3))], -1).astype(np.float32)
        return rad, feat
    a = pair(200, 300)
    b = pair(560, 720)
    first = dn.denoise(*a)
    again = dn.denoise(*a)          # replayed
    dn.denoise(*b)                  # new size: buffers grow
    back = dn.denoise(*a)           # first size again
    back2 = dn.denoise(*a)          # and replayed
    assert np.array_equal(first, again) and np.array_equal(first, back) and np.array_equal(first, back2)


def test_pipeline_wait_gives_up_and_context_survives(dn):
    """The failure path of the tensor-core kernels' pipeline waits, without a fault: a bounded wait on an mbarrier
    that nothing completes gives up (status 2) after about two seconds instead of hanging, and the device is
    still usable afterwards: the row-tile convolution then matches its result from before the probe bit for bit."""
    rng = np.random.default_rng(9)
    shape = (1, 16, 64, 16, 32)
    n, h, w, cin, cout = shape
    x = rng.normal(size=(n, h, w, cin)).astype(np.float32)
    wt = (rng.normal(size=(9, cout, cin)) * 0.1).astype(np.float32)
    b = rng.normal(size=cout).astype(np.float32)
    before = dn.debug_conv(5, x=x, w=wt, bias=b, shape=shape)
    status, seconds = dn.debug_wait_timeout()
    print("wait gave up after", seconds, "s, status", status)
    assert status == 2
    assert 1.0 <= seconds < 30.0
    after = dn.debug_conv(5, x=x, w=wt, bias=b, shape=shape)
    assert np.array_equal(before.view(np.uint32), after.view(np.uint32))
