"""Python side of the learned denoiser (C-ABI: bte_denoiser_* in include/bte/render_api.h).

The network replaces the reference's vendor denoiser stage (src/host/denoiser.cu:72-109,
cudaToggleDenoiser in include/render_kernel.h:187).  It is trained only on image pairs this
renderer produces: low-spp radiance plus the albedo/normal features (bte_read_aov) as input, long-run
FP64-accumulated radiance as target.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, load_library


def rel_mse(x: np.ndarray, ref: np.ndarray, eps: float = 1e-2) -> float:
    """Mean over pixels and channels of (x - r)^2 / (r^2 + eps)."""
    x = np.asarray(x, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    return float(np.mean((x - r) ** 2 / (r * r + eps)))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class Denoiser:
    """The learned denoiser of one build of the library (default: the process default, see load_library);
    the renderer of the same build presents its output when toggled on."""

    def __init__(self, variant: str | None = None):
        self.lib = load_library(variant=variant)

    def _ck(self, rc: int) -> int:
        return _check(rc, self.lib)

    def init(self, seed: int = 1):
        self._ck(self.lib.bte_denoiser_init(C.c_uint64(seed)))

    def param_count(self) -> int:
        n = C.c_longlong()
        self._ck(self.lib.bte_denoiser_param_count(C.byref(n)))
        return n.value

    def params(self) -> np.ndarray:
        out = np.empty(self.param_count(), dtype=np.float32)
        self._ck(self.lib.bte_denoiser_get_params(out.ctypes.data_as(C.c_void_p), C.c_longlong(out.size)))
        return out

    def set_params(self, p: np.ndarray):
        p = _f32(p)
        self._ck(self.lib.bte_denoiser_set_params(p.ctypes.data_as(C.c_void_p), C.c_longlong(p.size)))

    def save(self, path: str):
        np.savez_compressed(path, params=self.params().astype(np.float16))

    def load(self, path: str):
        """Weights saved by `save` or by train_denoiser (float16 on disk, float32 masters on the device)."""
        with np.load(path) as z:
            self.set_params(z["params"].astype(np.float32))

    def set_dataset(self, noisy: np.ndarray, features: np.ndarray, target: np.ndarray):
        """noisy [S, H, W, 3], features [S, H, W, 6], target [S, H, W, 3]."""
        noisy, features, target = _f32(noisy), _f32(features), _f32(target)
        S, H, W, _ = noisy.shape
        assert features.shape == (S, H, W, 6) and target.shape == (S, H, W, 3)
        self._keep = (noisy, features, target)
        self._ck(self.lib.bte_denoiser_set_dataset(noisy.ctypes.data_as(C.c_void_p), features.ctypes.data_as(C.c_void_p),
                                                 target.ctypes.data_as(C.c_void_p), S, W, H))

    def train(self, steps: int, batch: int = 8, crop: int = 128, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        loss = np.empty(steps, dtype=np.float32)
        self._ck(self.lib.bte_denoiser_train(int(steps), int(batch), int(crop), C.c_float(lr), C.c_uint64(seed),
                                           loss.ctypes.data_as(C.c_void_p)))
        return loss

    def denoise(self, radiance: np.ndarray, features: np.ndarray | None) -> np.ndarray:
        radiance = _f32(radiance)
        H, W, _ = radiance.shape
        out = np.empty((H, W, 3), dtype=np.float32)
        fp = None
        if features is not None:
            features = _f32(features)
            assert features.shape == (H, W, 6)
            fp = features.ctypes.data_as(C.c_void_p)
        self._ck(self.lib.bte_denoiser_denoise(radiance.ctypes.data_as(C.c_void_p), fp, W, H, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_tcgen05(self, mode):
        """Convolution kernels: 0 (or False) the warp-level MMA kernel only, 1 (or True) the tcgen05 pixel-tile
        kernel for the full-resolution layers, 2 (the default) the tcgen05 row-tile kernel for every layer with
        enough 128-pixel row tiles (layers it does not take stay on the warp-level kernel), decoder inputs
        upsampled beforehand; 3 the same with the upsampling done inside the row-tile kernel."""
        self._ck(self.lib.bte_denoiser_set_tcgen05(int(mode)))

    def debug_wait_timeout(self):
        """Run the tensor-core kernels' bounded wait on a barrier nothing completes: (status, seconds), status 2
        when the wait gave up as designed."""
        st = C.c_uint()
        sec = C.c_double()
        self._ck(self.lib.bte_denoiser_debug_wait_timeout(C.byref(st), C.byref(sec)))
        return st.value, sec.value

    def set_wgrad(self, kind: int):
        """Weight-gradient kernel of training: 1 tcgen05 where the layer's shape allows (default), 0 warp-level mma.sync,
        2-7 tcgen05 with one of its pipeline shapes (a tuning choice with the same sums)."""
        self._ck(self.lib.bte_denoiser_set_wgrad(int(kind)))

    def last_ms(self) -> float:
        ms = C.c_float()
        self._ck(self.lib.bte_denoiser_last_ms(C.byref(ms)))
        return ms.value

    def debug_conv(self, op: int, x=None, w=None, bias=None, dy=None, shape=(1, 16, 16, 16, 16), relu=True):
        """op 0: forward, 1: data gradient, 2: weight gradient (+ bias gradient) of one 3x3 conv layer;
        ops 3 and 4: ops 0 and 1 on the tcgen05 pixel-tile kernel; ops 5 and 6 on the row-tile kernel;
        op 7: op 2 on the tcgen05 weight-gradient kernel.
        shape = (N, H, W, Cin, Cout); x [N,H,W,Cin], w [9][Cout][Cin], dy [N,H,W,Cout]."""
        n, h, wd, cin, cout = shape
        keep = [None if a is None else _f32(a) for a in (x, w, bias, dy)]
        if op in (0, 3, 5):
            out = np.empty((n, h, wd, cout), dtype=np.float32)
        elif op in (1, 4, 6):
            out = np.empty((n, h, wd, cin), dtype=np.float32)
        else:
            out = np.empty(9 * cout * cin + cout, dtype=np.float32)
        ptrs = [None if a is None else a.ctypes.data_as(C.c_void_p) for a in keep]
        self._ck(self.lib.bte_denoiser_debug_conv(op, ptrs[0], ptrs[1], ptrs[2], ptrs[3], n, h, wd, cin, cout,
                                                1 if relu else 0, out.ctypes.data_as(C.c_void_p)))
        return out


def _main(argv=None):
    """Time inference: python -m bluetruthengine_b200.denoiser --width 1920 --height 1080 --iters 5 [--kernels 0|1|2]
    Time training steps instead: python -m bluetruthengine_b200.denoiser --train-steps 10 [--wgrad 0|1] (batch 8 of
    256x256 crops from 16 seeded synthetic images, after one untimed step)."""
    import argparse
    import json
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--iters", type=int, default=5)
    ap.add_argument("--kernels", type=int, default=2,
                    help="0 warp-level MMA only, 1 tcgen05 pixel tiles, 2 tcgen05 row tiles, 3 row tiles upsampling in-kernel")
    ap.add_argument("--weights", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights",
                                                      "denoiser_mixed.npz"))
    ap.add_argument("--train-steps", type=int, default=0, help="time this many training steps instead of inference")
    ap.add_argument("--wgrad", type=int, default=1, help="training weight gradients: 1 tcgen05, 0 warp-level, 2-7 tcgen05 pipeline shapes")
    args = ap.parse_args(argv)
    dn = Denoiser()
    if args.train_steps > 0:
        dn.init(7)
        rng = np.random.default_rng(0)
        dn.set_dataset(rng.exponential(0.5, size=(16, 256, 256, 3)).astype(np.float32),
                       rng.uniform(0, 1, size=(16, 256, 256, 6)).astype(np.float32),
                       rng.exponential(0.5, size=(16, 256, 256, 3)).astype(np.float32))
        dn.set_wgrad(args.wgrad)
        dn.train(1, batch=8, crop=256, lr=1e-4, seed=1)
        dn.train(args.train_steps, batch=8, crop=256, lr=1e-4, seed=2)
        print(json.dumps({"train_steps": args.train_steps, "batch": 8, "crop": 256, "wgrad": args.wgrad,
                          "ms_per_step": dn.last_ms() / args.train_steps}), flush=True)
        return
    dn.load(args.weights)
    dn.set_tcgen05(args.kernels)
    rng = np.random.default_rng(0)
    rad = rng.exponential(0.5, size=(args.height, args.width, 3)).astype(np.float32)
    feat = rng.uniform(0, 1, size=(args.height, args.width, 6)).astype(np.float32)
    ms = []
    for _ in range(args.iters):
        dn.denoise(rad, feat)
        ms.append(dn.last_ms())
    print(json.dumps({"width": args.width, "height": args.height, "ms": ms}), flush=True)


if __name__ == "__main__":
    _main()
