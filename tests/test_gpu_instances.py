"""Instanced scenes and the distant light on the GPU.

* Two-level traversal (object-space rays through each instance's object BVH
  under a top-level BVH) finds the hits of the flattened mesh, which is what
  the reference builds from its instances: the same hit/miss on all but a few
  rays grazing an edge, t within 1e-4 relative, the same shading normal.
* An instanced render matches the oracle's render of the flattened mesh on the
  same random numbers (relative RMSE per channel <= 5e-3; object-space
  rounding can flip a grazing ray's hit, which changes that one path).
* With the distant light (RGB radiance or a 5800 K blackbody, over a lit or a
  black sky), RGB and spectral renders match the oracle's restatement on the
  same random numbers (relative RMSE <= 1e-3).
* Batch views sharing one instanced scene render each view exactly as a plain
  render of that view.
"""

import numpy as np
import pytest

from lsystemeditor_b200.pathtracer import PathTracer
from lsystemeditor_b200.records import default_params
from lsystemeditor_b200.scene import forest_scene
from tests.helpers import rel_rmse, spectral_inputs, spectral_zoo_scene, zoo_camera

pytestmark = pytest.mark.gpu


def _small_forest(views=2, w=48, h=32, seed=7):
    return forest_scene(width=w, height=h, trees=3, instances=18, seed=seed, extent=14.0, sides=8, rings=2,
                        views=views, max_depth=6, min_spp=4, max_spp=4, iterations=(2, 3))


def _rays(lo, hi, n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    o[:, 1] = hi[1] + 2.0
    tgt = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o, d.astype(np.float32)


def test_instanced_trace_matches_flattened(tracer):
    scene, cams, params, sun = _small_forest()
    flat = scene.flatten()
    lo, hi = flat.bounds()
    o, d = _rays(lo, hi, 20000, 3)
    tmin = np.zeros(len(o), np.float32)
    tracer.configure(16, 16)
    tracer.set_instances(scene.objects, scene.instances)
    a = tracer.trace_rays(o, d, tmin)
    tracer.set_mesh(flat)
    b = tracer.trace_rays(o, d, tmin)
    hit_a, hit_b = a["hit"].astype(bool), b["hit"].astype(bool)
    assert hit_b.sum() > 2000
    agree = np.mean(hit_a == hit_b)
    assert agree >= 0.999, agree
    both = hit_a & hit_b
    assert np.all(np.abs(a["t"][both] - b["t"][both]) <= 1e-4 * np.abs(b["t"][both]) + 1e-5)
    same = np.abs(a["t"][both] - b["t"][both]) <= 1e-6 * np.abs(b["t"][both]) + 1e-6
    dots = np.sum(a["normal"][both] * b["normal"][both], axis=1)
    assert np.mean(dots[same] > 0.999) > 0.999


@pytest.mark.parametrize("mode", [0, 2])
def test_instanced_render_matches_oracle(tracer, oracle, mode):
    """Instanced render (warp-fetch form in the automatic mode on this small
    forest, and the two-level per-lane form) against the oracle's render of
    the flattened scene, replaying the GPU's random numbers."""
    scene, cams, params, sun = _small_forest()
    w, h, waves, stride = 48, 32, 4, 160
    params = params.copy()
    tracer.set_extend_mode(mode)
    tracer.configure(w, h)
    tracer.set_instances(scene.objects, scene.instances)
    tracer.set_camera(cams[0])
    tracer.set_params(params)
    tracer.set_environment(None)
    tape = tracer.rng_tape(0, waves, stride)
    tracer.reset_accumulation()
    tracer.render(waves)
    rgba = tracer.readback()[0].reshape(-1, 4)
    tracer.set_extend_mode(0)
    st = oracle.scene(scene.flatten()).render(cams[0], params, w, h, waves, tape=tape, tape_stride=stride)
    assert st["tape_errors"] == 0
    err = rel_rmse(rgba[:, :3], st["acc"][:, :3])
    assert np.all(err <= 5e-3), err


def _sun_pair(tracer, oracle, params, light, nw=0, env=None):
    mesh = spectral_zoo_scene(n_per_mat=120, seed=6)
    w, h, waves, stride = 40, 32, 6, 200
    params = params.copy()
    params["spectral_wavelengths"] = nw
    tracer.configure(w, h, mesh)
    tracer.set_camera(zoo_camera(w, h))
    tracer.set_params(params)
    tracer.set_environment(env)
    tracer.set_distant_light(**light)
    tape = tracer.rng_tape(0, waves, stride)
    tracer.reset_accumulation()
    tracer.render(waves)
    rgba = tracer.readback()[0].reshape(-1, 4)
    tracer.set_distant_light(None)
    sc = oracle.scene(mesh)
    resp = PathTracer.spectral_response()
    coef = None if light.get("temperature_k", 0.0) > 0 else PathTracer.spectral_uplift(light["radiance"])[0]
    sc.set_sun(light["direction"], light["half_angle"], radiance=light.get("radiance", (0.0, 0.0, 0.0)),
               temperature_k=light.get("temperature_k", 0.0), luminance=light.get("luminance", 1.0), resp=resp,
               coef=coef)
    oenv = oracle.env(env) if env is not None else None
    if nw == 0:
        st = sc.render(zoo_camera(w, h), params, w, h, waves, tape=tape, tape_stride=stride, env=oenv)
    else:
        sp = spectral_inputs(mesh, params, nw, env)
        st = sc.render_spectral(zoo_camera(w, h), params, w, h, waves, sp, tape=tape, tape_stride=stride, env=oenv)
    assert st["tape_errors"] == 0
    return rgba, st


@pytest.mark.parametrize("nw", [0, 8])
@pytest.mark.parametrize("sky", ["black", "lit"])
def test_sun_parity(tracer, oracle, nw, sky):
    bg = (0.0, 0.0, 0.0) if sky == "black" else (0.3, 0.35, 0.5)
    params = default_params(background_r=bg[0], background_g=bg[1], background_b=bg[2], max_path_depth=6,
                            min_samples=6, max_samples_per_pixel=6)
    light = dict(direction=(0.3, 1.0, 0.4), half_angle=0.02, temperature_k=5800.0, luminance=400.0)
    rgba, st = _sun_pair(tracer, oracle, params, light, nw=nw)
    err = rel_rmse(rgba[:, :3], st["acc"][:, :3])
    assert np.all(err <= 1e-3), err


def test_sun_rgb_radiance_parity(tracer, oracle):
    params = default_params(background_r=0.2, background_g=0.25, background_b=0.3, max_path_depth=6,
                            min_samples=6, max_samples_per_pixel=6)
    light = dict(direction=(-0.5, 1.0, 0.2), half_angle=0.05, radiance=(60.0, 50.0, 30.0))
    for nw in (0, 4):
        rgba, st = _sun_pair(tracer, oracle, params, light, nw=nw)
        err = rel_rmse(rgba[:, :3], st["acc"][:, :3])
        assert np.all(err <= 1e-3), (nw, err)


def test_shared_views_match_plain_renders():
    scene, cams, params, sun = _small_forest(views=2)
    sizes = [(40, 24), (32, 32)]
    params = params.copy()
    params["spectral_wavelengths"] = 8
    plain = []
    with PathTracer(0) as t:
        for k, (w, h) in enumerate(sizes):
            t.configure(w, h)
            t.set_instances(scene.objects, scene.instances)
            cam = cams[k].copy()
            cam["aspect"] = w / h
            t.set_camera(cam)
            t.set_params(params)
            t.set_distant_light(**sun)
            t.render(0)
            plain.append(t.readback()[0])
    with PathTracer(0) as t:
        t.batch_configure(sizes)
        t.set_instances(scene.objects, scene.instances, scene=0)
        t.batch_share_scene(1, 0)
        for k, (w, h) in enumerate(sizes):
            cam = cams[k].copy()
            cam["aspect"] = w / h
            t.batch_set_camera(k, cam)
        t.set_params(params)
        t.set_distant_light(**sun)
        t.render(0)
        for k in range(2):
            assert np.array_equal(t.batch_readback(k)[0], plain[k]), f"view {k} differs from its plain render"


@pytest.mark.parametrize("nw", [0, 8])
def test_instanced_extend_modes_render_the_same_image(nw):
    """Closest-hit and shadow stages of an instanced scene (two-level BVH, sun
    light) in the warp-fetch and the per-lane forms, with many recycled path
    slots: identical images, sample counts and trace results."""
    scene, cams, params, sun = _small_forest(views=1, w=64, h=48)
    params = params.copy()
    params["spectral_wavelengths"] = nw
    params["min_samples"] = 4
    params["max_samples_per_pixel"] = 12
    params["relative_error_threshold"] = 0.3
    out = {}
    with PathTracer(0) as t:
        t.configure(64, 48)
        t.set_instances(scene.objects, scene.instances)
        t.set_camera(cams[0])
        t.set_params(params)
        if sun is not None:
            t.set_distant_light(**sun)
        for mode, cap in ((1, 0), (2, 0), (2, 4096)):
            t.set_extend_mode(mode)
            t.set_tuning(cap, 0)
            t.reset_accumulation()
            t.render(0)
            rgba, counts, conv = t.readback()
            out[(mode, cap)] = (rgba.copy(), counts.copy(), conv.copy())
        t.set_tuning(0, 0)
        t.set_extend_mode(0)
    ref = out[(1, 0)]
    assert ref[0][..., :3].max() > 0
    for key, got in out.items():
        for a, b, what in zip(ref, got, ("image", "sample counts", "convergence flags")):
            assert np.array_equal(a, b), f"mode {key}: {what} differ from the warp form"
