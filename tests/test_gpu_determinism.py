"""Renders and hits do not depend on the BVH's layout (GPU).

The compressed wide BVH is collapsed top-down in parallel, and the order in
which nodes and leaf ranges are allocated differs from build to build.  Every
closest-hit traversal therefore breaks exact-t ties by the original triangle
index (instanced scenes: by the (instance, triangle) pair), never by a leaf's
position.  Scenes built from duplicated triangles make every hit such a tie:

* each ray's hit is the higher-indexed copy, with the t of the single mesh;
* two renderers built from the same flat or instanced scene (the copies of a
  triangle carrying different materials and normals) render bit-identical
  images, RGB and spectral, with and without a distant light.
"""
import numpy as np
import pytest

from lsystemeditor_b200.pathtracer import PathTracer
from lsystemeditor_b200.records import default_params, look_at_camera
from lsystemeditor_b200.scene import HostMesh
from tests.helpers import random_soup, rays_through_bounds

pytestmark = pytest.mark.gpu


def _doubled(n=3000, seed=4):
    """Every triangle twice: copy k + n has the vertices of k, another material and other normals."""
    a = random_soup(n, seed=seed, materials=3)
    b = random_soup(n, seed=seed + 1, materials=3)
    b.positions = a.positions.copy()
    return a, HostMesh.concat([a, b])


def test_exact_ties_go_to_the_higher_index():
    single, doubled = _doubled()
    n = single.triangle_count
    o, d = rays_through_bounds(single, 20000, seed=5)
    with PathTracer(0) as t:
        t.configure(16, 16)
        t.set_mesh(single)
        a = t.trace_rays(o, d)
        t.set_mesh(doubled)
        b = t.trace_rays(o, d)
    assert a["hit"].sum() > 5000
    assert np.array_equal(a["hit"], b["hit"])
    hit = a["hit"]
    assert np.array_equal(a["t"][hit], b["t"][hit])
    assert np.array_equal(b["tri"][hit], a["tri"][hit] + n), "a tie did not go to the higher triangle index"


def _render(mesh_or_objects, instances, nw, sun):
    w, h = 64, 48
    params = default_params(background_r=0.3, background_g=0.35, background_b=0.4, max_path_depth=6,
                            min_samples=8, max_samples_per_pixel=8, spectral_wavelengths=nw)
    with PathTracer(0) as t:
        t.configure(w, h)
        if instances is None:
            t.set_mesh(mesh_or_objects)
        else:
            t.set_instances(mesh_or_objects, instances)
        t.set_camera(look_at_camera((0.0, 3.0, 14.0), (0.0, 0.0, 0.0), fov_y_deg=45.0, aspect=w / h))
        t.set_params(params)
        if sun:
            t.set_distant_light((0.4, 0.8, 0.45), half_angle=0.01, temperature_k=5800.0, luminance=20.0)
        t.reset_accumulation()
        t.render(0)
        rgba, counts, _ = t.readback()
        return rgba.copy(), counts.copy()


@pytest.mark.parametrize("nw,sun", [(0, False), (0, True), (8, True)])
def test_two_builds_render_the_same_image(nw, sun):
    _, doubled = _doubled()
    xf0 = np.array([[1, 0, 0, -2.5], [0, 1, 0, 0], [0, 0, 1, 0]], np.float32)
    xf1 = np.array([[0, 0, 1, 2.5], [0, 1, 0, 0.5], [-1, 0, 0, 0]], np.float32)
    for scene, inst in ((doubled, None), ([doubled], [(xf0, 0), (xf1, 0)])):
        a = _render(scene, inst, nw, sun)
        b = _render(scene, inst, nw, sun)
        assert a[0][..., :3].max() > 0
        assert np.array_equal(a[1], b[1])
        assert np.array_equal(a[0], b[0]), "two builds of the same scene rendered different images"
