"""Frame-loop graphs and the autotuner (GPU).

* The bounce loop replayed from CUDA graphs (the default) renders exactly what
  the same loop launched kernel by kernel renders (stage profiling turns the
  graphs off), for a plain scene, a spectral render and a batch of views.
* pt_autotune returns knobs from its candidate sets, never a slower probe
  than the configuration it started from, and the image rendered with the
  chosen knobs is bit-identical to the one rendered with the defaults.
* pt_readback fills caller-owned (e.g. pinned) arrays exactly like fresh ones.
* The closest-hit stage renders the same image, sample counts and convergence
  flags in both its forms: one warp per 32 queued rays with pushes into the
  miss/hit and next-bounce queues, and per-lane ray replacement with
  queue-order routing and a slot-ordered next-bounce queue -- graphed and
  launched kernel by kernel, with few path slots (many recycled paths), for
  RGB and spectral paths and for a batch of scenes.
"""
import numpy as np
import pytest

from lsystemeditor_b200.pathtracer import PROFILE_STAGE_TIMES, PathTracer
from lsystemeditor_b200.records import default_params, look_at_camera
from tests.helpers import sky, spectral_zoo_scene, zoo_camera, zoo_scene

pytestmark = pytest.mark.gpu


def _render(t, profile):
    t.set_profiling(PROFILE_STAGE_TIMES if profile else 0)
    t.reset_accumulation()
    t.render(0)
    out = t.readback()[0].copy()
    t.set_profiling(0)
    return out


@pytest.mark.parametrize("nw", [0, 8])
def test_graphs_match_direct_launches(nw):
    mesh = spectral_zoo_scene(n_per_mat=150, seed=8)
    w, h = 64, 48
    params = default_params(background_r=0.1, background_g=0.12, background_b=0.2, max_path_depth=8,
                            min_samples=8, max_samples_per_pixel=24, relative_error_threshold=0.3,
                            spectral_wavelengths=nw)
    with PathTracer(0) as t:
        t.configure(w, h, mesh)
        t.set_camera(zoo_camera(w, h))
        t.set_params(params)
        graphed = _render(t, False)
        direct = _render(t, True)
        assert np.array_equal(graphed, direct)


def test_autotune_keeps_the_image():
    mesh = spectral_zoo_scene(n_per_mat=150, seed=9)
    w, h = 96, 64
    params = default_params(background_r=0.1, background_g=0.12, background_b=0.2, max_path_depth=8,
                            min_samples=16, max_samples_per_pixel=16)
    with PathTracer(0) as t:
        t.configure(w, h, mesh)
        t.set_camera(zoo_camera(w, h))
        t.set_params(params)
        t.render(0)
        before = t.readback()[0].copy()
        tune = t.autotune(waves=4)
        assert tune["path_capacity"] in (1 << 21, 1 << 22, 1 << 23, 1 << 24)
        assert tune["blocks_per_sm"] in (0, 2, 3, 4)
        assert tune["samples_per_launch"] in (0, 4, 16, 64)
        assert tune["trials"] >= 2 and tune["ms_best"] <= tune["ms_default"]
        t.render(0)
        after = t.readback()[0]
        assert np.array_equal(before, after), "the tuned knobs changed the image"


def _render_all(t):
    t.reset_accumulation()
    t.render(0)
    rgba, counts, conv = t.readback()
    return rgba.copy(), counts.copy(), conv.copy()


@pytest.mark.parametrize("nw, mis", [(0, 0), (8, 0), (0, 1)])
def test_extend_modes_render_the_same_image(nw, mis):
    """Closest-hit and shadow stages in the warp-fetch and per-lane forms; with
    emitter MIS the emissive shadow rays end short of the light (tMax)."""
    mesh = spectral_zoo_scene(n_per_mat=150, seed=11)
    w, h = 64, 48
    params = default_params(background_r=0.1, background_g=0.12, background_b=0.2, max_path_depth=8,
                            min_samples=8, max_samples_per_pixel=32, relative_error_threshold=0.3,
                            spectral_wavelengths=nw, emitter_mis=mis)
    with PathTracer(0) as t:
        t.configure(w, h, mesh)
        t.set_camera(zoo_camera(w, h))
        t.set_params(params)
        t.set_extend_mode(1)
        warp = _render_all(t)
        runs = {}
        t.set_extend_mode(2)
        runs["lane"] = _render_all(t)
        t.set_profiling(PROFILE_STAGE_TIMES)
        runs["lane, kernel by kernel"] = _render_all(t)
        t.set_profiling(0)
        t.set_tuning(path_capacity=1 << 12)
        runs["lane, 4096 path slots"] = _render_all(t)
        t.set_extend_mode(1)
        runs["warp, 4096 path slots"] = _render_all(t)
        t.set_tuning()
        t.set_extend_mode(0)
        runs["auto"] = _render_all(t)
        for name, got in runs.items():
            for a, b, what in zip(warp, got, ("image", "sample counts", "convergence flags")):
                assert np.array_equal(a, b), f"{name}: {what} differ from the warp form"
        assert warp[0][..., :3].max() > 0 and len(np.unique(warp[1])) > 1
        with pytest.raises(RuntimeError):
            t.set_extend_mode(3)


def test_extend_modes_batch():
    views = [(zoo_scene(n_per_mat=n, seed=30 + k), w, h, eye)
             for k, (n, w, h, eye) in enumerate([(120, 40, 32, (0.5, 1.0, 9.0)), (40, 24, 24, (4.0, 2.0, 7.0)),
                                                 (200, 56, 30, (-3.0, 0.5, 8.0))])]
    params = default_params(max_path_depth=6, min_samples=6, max_samples_per_pixel=6, environment_intensity=1.2)
    out = {}
    with PathTracer(0) as t:
        for mode in (1, 2):
            t.set_extend_mode(mode)
            t.batch_configure([(w, h) for _, w, h, _ in views])
            for k, (mesh, w, h, eye) in enumerate(views):
                t.batch_set_mesh(k, mesh)
                t.batch_set_camera(k, look_at_camera(eye, (0.0, 0.0, 0.0), fov_y_deg=45.0, aspect=w / h))
            t.set_params(params)
            t.set_environment(sky())
            t.reset_accumulation()
            t.render(0)
            out[mode] = [t.batch_readback(k) for k in range(len(views))]
    for k, (a, b) in enumerate(zip(out[1], out[2])):
        for x, y, what in zip(a, b, ("image", "sample counts", "convergence flags")):
            assert np.array_equal(x, y), f"scene {k}: {what} differ between the warp and lane forms"
        assert a[0][..., :3].max() > 0


def test_readback_into_caller_buffers():
    mesh = spectral_zoo_scene(n_per_mat=60, seed=12)
    w, h = 40, 24
    with PathTracer(0) as t:
        t.configure(w, h, mesh)
        t.set_camera(zoo_camera(w, h))
        t.set_params(default_params(max_path_depth=4, min_samples=4, max_samples_per_pixel=4))
        t.render(0)
        fresh = t.readback()
        out = (np.full((h, w, 4), -1.0, np.float32), np.zeros((h, w), np.uint32), np.full((h, w), 7, np.uint8))
        got = t.readback(out)
        assert all(g is o for g, o in zip(got, out))
        for a, b in zip(fresh, out):
            assert np.array_equal(a, b)
        with pytest.raises(ValueError):
            t.readback((np.zeros((h, w, 3), np.float32), out[1], out[2]))
