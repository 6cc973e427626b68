"""Seeded scene generators: deterministic bytes, outward windings, sizes."""
import hashlib
import os

import numpy as np


def _digest(path):
    h = hashlib.sha256()
    d = os.path.dirname(path)
    for f in sorted(os.listdir(d)):
        if f.startswith("."):
            continue
        h.update(f.encode())
        h.update(open(os.path.join(d, f), "rb").read())
    return h.hexdigest()


def test_generators_are_deterministic(tmp_path, monkeypatch):
    from bluetruthengine_b200 import scenes
    a = _digest(scenes.random_scene(5))
    monkeypatch.setattr(scenes, "CACHE_ROOT", str(tmp_path))
    b = _digest(scenes.random_scene(5))
    assert a == b


def test_icosphere_and_cube_windings():
    from bluetruthengine_b200 import scenes
    for lvl in range(4):
        v, f = scenes.icosphere(lvl)
        assert len(f) == 20 * 4 ** lvl
        n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
        assert np.all((n * v[f].mean(1)).sum(1) > 0)
    v, f = scenes.unit_cube()
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    assert np.all((n * v[f].mean(1)).sum(1) > 0)
    v, f = scenes.grid_plane(4, 1.0)
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    assert np.all(n[:, 1] > 0) and len(f) == 32


def test_bench_scene_size(bte):
    from bluetruthengine_b200 import scenes
    sc = bte.load_scene(scenes.disney_spheres())
    assert 1_000_000 <= sc.triangle_count <= 1_100_000
    assert sc.width == 1920 and sc.height == 1080
    assert sc.env_rgba.shape == (1024, 2048, 4)
    assert np.isclose(sc.env_rgba[..., :3].max(), 1e4, rtol=0.01)
    b = sc.bsdfs
    assert np.all(b["type"] == 5) and len(b) == 65
    metal = b["p1"][1:, 0]
    assert set(np.unique(metal)) <= {0.0, 1.0}
