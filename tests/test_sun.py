"""Distant light (extension), oracle side (no GPU): a rough plane lit only by
the light reaches the radiance f(wo, n) * L * pi * sin^2(half-angle) of a
narrow cone around its normal, with the light's next-event samples and the
BSDF samples that escape into the cone combined by MIS; a light with a
temperature has the requested luminance; without a light the oracle's
estimator is the reference's (the golden and pin tests cover that)."""
import math

import numpy as np

from lsystemeditor_b200.pathtracer import PathTracer
from lsystemeditor_b200.records import default_material, default_params, look_at_camera
from lsystemeditor_b200.scene import quad_mesh


def test_plane_under_the_light(oracle):
    mat = default_material(r=0.6, g=0.5, b=0.4, roughness=1.0, specular=0.5)
    mesh = quad_mesh((0, 0, 0), (50, 0, 0), (0, 0, -50), mat, normal=(0, 1, 0))
    w = h = 16
    cam = look_at_camera((0.0, 5.0, 0.001), (0.0, 0.0, 0.0), fov_y_deg=2.0, aspect=1.0)
    cam["focus_valid"] = 0
    params = default_params(background_r=0.0, background_g=0.0, background_b=0.0, max_path_depth=1,
                            min_samples=256, max_samples_per_pixel=256)
    half = 0.05
    L = np.array([2.0, 3.0, 4.0], np.float32)
    sc = oracle.scene(mesh)
    sc.set_sun((0.0, 1.0, 0.0), half, radiance=L)
    st = sc.render(cam, params, w, h, 256, fp64=True)
    img = st["acc"][:, :3].mean(0)
    f = np.asarray(oracle.brdf_eval([0, 1, 0], [0, 1, 0], mat, 1.0, [0, 1, 0]), np.float64)
    want = f * L * math.pi * math.sin(half) ** 2
    assert np.allclose(img, want, rtol=0.02), (img, want)


def test_blackbody_luminance(oracle):
    """RGB of a 5800 K light = its luminance (Rec. 709 weights) through the response table, seen directly."""
    mesh = quad_mesh((0, -100, 0), (1, 0, 0), (0, 0, -1), default_material(), normal=(0, 1, 0))
    w = h = 4
    cam = look_at_camera((0.0, 0.0, 0.0), (0.0, 1.0, 0.0001), fov_y_deg=0.01, aspect=1.0)
    cam["focus_valid"] = 0
    params = default_params(background_r=0.0, background_g=0.0, background_b=0.0, max_path_depth=1,
                            min_samples=1, max_samples_per_pixel=1)
    sc = oracle.scene(mesh)
    sc.set_sun((0.0, 1.0, 0.0), 0.01, temperature_k=5800.0, luminance=7.0, resp=PathTracer.spectral_response())
    rgb = sc.render(cam, params, w, h, 1, fp64=True)["acc"][:, :3].mean(0)
    assert abs(0.2126 * rgb[0] + 0.7152 * rgb[1] + 0.0722 * rgb[2] - 7.0) < 1e-4
    assert rgb[0] > rgb[2] * 0.9 and rgb.min() > 0  # a warm white
