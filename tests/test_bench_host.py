"""Host-side arithmetic of bench.py, on the CPU.

* The denoiser FLOP table the bench scores against (DENOISER_CONVS) is the network the library builds: the
  convolutions of bte_denoise.cu's step table, in order, with their channel counts and pyramid levels.
* The algorithmic bytes per unit of work add up from the reference's SoA record sizes
  (include/wavefront/wavefront_buffers.h:40-90: path state 69 B, hit 36 B, queue entry 4 B, shadow record 44 B).
* The layer-by-layer denoiser roofline is at least each bound it takes the larger of, and scales with the pixels.
* Without a measured-peaks file the bench falls back to the stated fallback peaks and says so.
* The kernel count it claims per frame follows the renderer's launch sequence for the tuning in force, and the
  host<->device bytes it claims per end-to-end step are the copies the renderer's frame makes.
* The clock record read from nvidia-smi's CSV: median SM clock, max clock and the throttle reasons seen.
"""
import importlib.util
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _network_convs():
    """(Cin, Cout, level) of every convolution in the order the library's step table runs them."""
    src = open(os.path.join(ROOT, "bluetruthengine_b200", "csrc", "bte_denoise.cu")).read()
    tensors = re.search(r"const TensorSpec kTensors\[\] = \{(.*?)\};", src, re.S).group(1)
    tensors = [(int(c), int(lv)) for c, lv in re.findall(r"\{(\d+),\s*(\d+)\}", tensors)]
    convs = re.search(r"const Conv kConvs\[\] = \{(.*?)\};", src, re.S).group(1)
    convs = [(int(a), int(b)) for a, b, _, _ in re.findall(r"\{(\d+),\s*(\d+),\s*(\d+),\s*(true|false)\}", convs)]
    steps = re.search(r"const Step kSteps\[\] = \{(.*?)\};", src, re.S).group(1)
    steps = re.findall(r"\{(kConvOp|kPoolOp|kUpCatOp),\s*(-?\d+),\s*(-?\d+),\s*(-?\d+),\s*(-?\d+)\}", steps)
    assert len(tensors) == 28 and len(convs) == 19 and len(steps) == 27
    out = []
    for op, s, _, d, c in steps:
        if op != "kConvOp":
            continue
        cin, cout = convs[int(c)]
        src_c, src_lv = tensors[int(s)]
        dst_c, dst_lv = tensors[int(d)]
        assert (cin, cout) == (src_c, dst_c) and src_lv == dst_lv, (op, s, d, c)
        out.append((cin, cout, src_lv))
    return out


def test_denoiser_flop_table_is_the_built_network(bench):
    assert [tuple(c) for c in bench.DENOISER_CONVS] == _network_convs()
    expect = sum(2 * 9 * ci * co / 4 ** lv for ci, co, lv in _network_convs())
    assert bench.DENOISER_FLOP_PER_PIXEL == pytest.approx(expect, rel=1e-12)


def test_algorithmic_bytes_from_reference_record_sizes(bench):
    state, hit, queue, shadow, ray, radiance_rmw = 69, 36, 4, 44, 24, 24
    assert bench.BYTES_PER_EXTEND_RAY == queue + ray + hit
    assert bench.BYTES_PER_SHADE_SEGMENT == queue + state + hit + state + queue
    assert bench.BYTES_PER_SEGMENT == bench.BYTES_PER_EXTEND_RAY + bench.BYTES_PER_SHADE_SEGMENT + 5
    assert bench.BYTES_PER_SAMPLE_FIXED == (state + queue) + (12 + 4 + radiance_rmw)
    assert bench.BYTES_PER_SHADOW == shadow + shadow + radiance_rmw
    assert bench.BYTES_PER_CONNECT_RAY == shadow + radiance_rmw


def test_denoiser_layer_roofline(bench):
    tflops, gbs = 1648.4, 6550.7
    t = bench.denoiser_layer_bound_ms(1920, 1080, tflops, gbs)
    px = 1920 * 1088   # image heights are padded to a multiple of 16
    flop_ms = bench.DENOISER_FLOP_PER_PIXEL * px / (tflops * 1e12) * 1e3
    assert t >= flop_ms * (1 - 1e-9)
    bytes_ms = sum(2 * (ci + co) * px / 4 ** lv for ci, co, lv in bench.DENOISER_CONVS) / (gbs * 1e9) * 1e3
    assert t >= bytes_ms * (1 - 1e-9)
    assert t <= flop_ms + bytes_ms
    t4k = bench.denoiser_layer_bound_ms(3840, 2160, tflops, gbs)
    assert t4k == pytest.approx(4 * t, rel=0.02)
    assert bench.denoiser_layer_bound_ms(1920, 1080, tflops * 2, gbs * 2) == pytest.approx(t / 2, rel=1e-9)


def test_peaks_fall_back_without_measurements(bench, tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.measured_peaks() == (6650.0, "fallback")
    assert bench.measured_bf16_tflops() == (1590.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 6550.7, "bf16_tflops": 1648.4}')
    assert bench.measured_peaks() == (6550.7, "measured")
    assert bench.measured_bf16_tflops()[0] == 1648.4


def test_frame_launch_count(bench):
    default = {"tailPaths": 4096, "sortShading": 1, "raySortBits": 0, "raySortBounces": 4, "orderBounces": 3}
    # generate + present, 16 x (extend, shade, connect), tail, compactions: buckets of 0, 1, 2 and queues of 1, 2
    assert bench.frame_launches(16, default) == 2 + 48 + 1 + 3 + 2
    assert bench.frame_launches(16, dict(default, tailPaths=0)) == 55
    assert bench.frame_launches(16, dict(default, sortShading=0)) == 51           # no path order without sorting
    assert bench.frame_launches(16, dict(default, raySortBits=3)) == 51 + 2 * 4   # reordering replaces path order
    assert bench.frame_launches(2, default) == 2 + 6 + 1 + 2 + 1                  # order capped at the depth
    assert bench.frame_launches(1, dict(default, raySortBits=3)) == 2 + 3 + 1     # no bounce 1 to reorder


def test_e2e_copy_bytes_are_the_frames_copies(bench):
    """The copies renderFrame makes (the frame-index upload, the counter and error-word readbacks) and the
    framebuffer readback, counted from the renderer's source."""
    src = open(os.path.join(ROOT, "bluetruthengine_b200", "csrc", "bte_renderer.cu")).read()
    body = src[src.index("void renderFrame(int w, int h)"):]
    body = body[:body.index("\n}\n")]
    h2d = re.findall(r"cudaMemcpyAsync\(([^;]*?)cudaMemcpyHostToDevice", body)
    d2h = re.findall(r"cudaMemcpyAsync\(([^;]*?)cudaMemcpyDeviceToHost", body)
    assert len(h2d) == 1 and "sizeof(uint32_t)" in h2d[0]
    assert len(d2h) == 3 and sum("(depth + 1)" in c for c in d2h) == 2 and sum(", 4," in c for c in d2h) == 1
    W, H, depth = 1920, 1080, 16
    assert bench.e2e_copy_bytes(W, H, depth) == (4, W * H * 4 + 2 * 17 * 4 + 4)


def test_clock_lines(bench):
    lines = ["0, 1965, 1965, 640.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n",
             "0, 1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n",
             "0, 1800, 1965, 999.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n",
             "0, [N/A], 1965, 10.0, 0x0, Not Active, Not Active, Not Active, Not Active\n",   # unreadable: skipped
             "garbage\n"]
    got = bench.parse_clock_lines(lines)
    assert got == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    hot = ["0, 1200, 1965, 700, 0x48, Not Active, Active, Not Active, Not Active\n"]
    assert bench.parse_clock_lines(hot)["reasons"] == ["hw_thermal_slowdown"]
    assert bench.parse_clock_lines([]) is None
