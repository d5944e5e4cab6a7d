"""Preview passes and region render (PathTracer.h:89-92, 134-140).

* A preview level matches the oracle's preview pass (pixel centres, one
  sample, depth 4, global seed level + 1) on the same random numbers: the
  tape comes from a renderer of the preview's size whose preview count equals
  the level, which makes its wave 0 draw with exactly those seeds.
* With previews, full-resolution wave w draws with global seed n + w + 1, and
  until the first wave pt_tonemap shows the finest preview upsampled.
* A region render samples only the rectangle, every region pixel equals the
  same pixel of a full render, and resetting the region keeps the rest.
"""
import numpy as np
import pytest

from lsystemeditor_b200.pathtracer import PathTracer
from lsystemeditor_b200.records import default_params
from tests.helpers import rel_rmse, zoo_camera, zoo_scene

pytestmark = pytest.mark.gpu


def _setup(tracer, w, h, waves=4, depth=6):
    mesh = zoo_scene(n_per_mat=120, seed=5)
    params = default_params(background_r=0.2, background_g=0.22, background_b=0.3, max_path_depth=depth,
                            min_samples=waves, max_samples_per_pixel=waves)
    tracer.configure(w, h, mesh)
    tracer.set_camera(zoo_camera(w, h))
    tracer.set_params(params)
    return mesh, params


def test_preview_levels_match_oracle(tracer, oracle):
    w, h, n = 96, 80, 3
    mesh, params = _setup(tracer, w, h)
    tracer.set_preview_steps_per_level(n)
    tracer.render(1)
    sc = oracle.scene(mesh)
    pprev = params.copy()
    pprev["max_path_depth"] = 4
    for lv in range(n):
        img = tracer.preview(lv)
        ds = 2 ** (n - lv)
        assert img.shape == (h // ds, w // ds, 4)
        ph, pw = img.shape[:2]
        with PathTracer(0) as t2:
            t2.configure(pw, ph, mesh)
            t2.set_preview_steps_per_level(lv)
            tape = t2.rng_tape(0, 1, 80)[0]
        ref, err = sc.render_preview(zoo_camera(w, h), pprev, pw, ph, tape, 80)
        assert err == 0
        e = rel_rmse(img[..., :3], ref[..., :3])
        assert np.all(e <= 1e-3), (lv, e)
    tracer.set_preview_steps_per_level(0)


def test_preview_shifts_full_resolution_seeds(tracer, oracle):
    w, h, n, waves = 48, 40, 2, 3
    mesh, params = _setup(tracer, w, h, waves=waves)
    tracer.set_preview_steps_per_level(n)
    tape = tracer.rng_tape(0, waves, 160)   # drawn with global seeds n + w + 1
    tracer.render(0)
    rgba, counts, _ = tracer.readback()
    assert np.all(counts == waves)
    st = oracle.scene(mesh).render(zoo_camera(w, h), params, w, h, waves, tape=tape, tape_stride=160)
    assert st["tape_errors"] == 0
    e = rel_rmse(rgba.reshape(-1, 4)[:, :3], st["acc"][:, :3])
    assert np.all(e <= 1e-3), e
    tracer.set_preview_steps_per_level(0)


def test_tonemap_shows_upsampled_preview_before_first_wave(tracer):
    w, h, n = 64, 48, 2
    mesh, params = _setup(tracer, w, h, waves=2)
    tracer.set_preview_steps_per_level(n)
    bg = np.array([0.2, 0.22, 0.3], np.float32)
    q = (np.clip(bg / (np.float32(1) + bg), 0, 1) * np.float32(255)).astype(np.uint8)
    assert np.all(tracer.tonemap(0, 1.0)[..., :3] == q), "nothing rendered yet: background everywhere"
    tracer.render_previews()
    prev = tracer.preview(n - 1)
    ph, pw = prev.shape[:2]
    yy, xx = np.mgrid[0:h, 0:w]
    up = prev[np.minimum(yy // 2, ph - 1), np.minimum(xx // 2, pw - 1), :3].astype(np.float32)
    want = (np.clip(up / (np.float32(1) + up), 0, 1) * np.float32(255)).astype(np.uint8)
    assert np.array_equal(tracer.tonemap(0, 1.0)[..., :3], want)
    tracer.render(1)   # after a full-resolution wave the accumulator is shown
    rgba, _, _ = tracer.readback()
    acc = rgba[..., :3].astype(np.float32)
    want = (np.clip(acc / (np.float32(1) + acc), 0, 1) * np.float32(255)).astype(np.uint8)
    assert np.array_equal(tracer.tonemap(0, 1.0)[..., :3], want)
    tracer.set_preview_steps_per_level(0)


def test_region_render(tracer):
    w, h, waves = 48, 40, 3
    mesh, params = _setup(tracer, w, h, waves=waves)
    tracer.render(0)
    full, fcounts, _ = tracer.readback()
    x0, y0, x1, y1 = 30, 25, 9, 7   # unordered corners are ordered
    tracer.set_render_region(x0, y0, x1, y1)
    # enabling clears the region only
    rgba, counts, _ = tracer.readback()
    inside = np.zeros((h, w), bool)
    inside[7:26, 9:31] = True
    assert np.all(counts[inside] == 0) and np.array_equal(counts[~inside], fcounts[~inside])
    assert np.array_equal(rgba[~inside], full[~inside])
    tracer.render(0)
    rgba, counts, _ = tracer.readback()
    assert np.all(counts[inside] == waves)
    assert np.array_equal(rgba[inside], full[inside]), "region pixels differ from the full render"
    assert np.array_equal(rgba[~inside], full[~inside])
    # a full reset (parameter change) clears everything and samples only the region
    tracer.set_params(params)
    tracer.render(0)
    rgba, counts, _ = tracer.readback()
    assert np.all(counts[~inside] == 0) and np.all(counts[inside] == waves)
    assert np.array_equal(rgba[inside], full[inside])
    tracer.set_render_region(0, 0, 0, 0, enabled=False)
    tracer.render(0)
    rgba, counts, _ = tracer.readback()
    assert np.all(counts == waves) and np.array_equal(rgba, full)
