"""Scene construction and display output on the device.

* The device loft (pt_batch_set_tubes) writes the same triangles, bit for bit,
  as the host generator (TubeSet.host_mesh), read back with pt_export_mesh.
* A scene built on the device traces like the same scene uploaded from the
  host (hit ids / t / normal / uv, up to exact-t ties).
* The emissive list and CDF are built on the device; renders of a scene with
  lights are covered against the oracle by test_gpu_parity; here the device
  build of a light-only soup is checked through light sampling statistics.
* pt_tonemap follows the reference display pipeline exactly (restated here in
  numpy single precision); pt_exposure_multiplier the physical-camera formula.
"""
import numpy as np
import pytest

from lsystemeditor_b200.records import default_params
from lsystemeditor_b200.scene import tree_tubes
from tests.helpers import rays_through_bounds, zoo_camera, zoo_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("iterations,sides,rings", [(4, 6, 2), (5, 12, 5), (6, 64, 16)])
def test_device_loft_matches_host_generator(tracer, iterations, sides, rings):
    ts = tree_tubes(iterations=iterations, seed=30 + iterations, sides=sides, rings=rings)
    host = ts.host_mesh()
    tracer.configure(16, 16)
    tracer.batch_set_tubes(0, ts)
    dev = tracer.export_mesh(0)
    assert dev.triangle_count == host.triangle_count == ts.triangle_count
    for f in ("positions", "normals", "uvs", "material_ids"):
        a, b = getattr(dev, f), getattr(host, f)
        bad = np.nonzero(a.reshape(len(a), -1) != b.reshape(len(b), -1))[0]
        assert len(bad) == 0, f"{f}: {len(bad)} triangles differ, first {bad[:5]}"


def test_device_built_scene_traces_like_uploaded_scene(tracer):
    from tests.test_gpu_parity import _compare_hits
    ts = tree_tubes(iterations=6, seed=5, sides=16, rings=6)
    host = ts.host_mesh()
    o, d = rays_through_bounds(host, 100_000, seed=6)
    tracer.configure(16, 16, host)
    a = tracer.trace_rays(o, d)
    tracer.batch_set_tubes(0, ts)
    b = tracer.trace_rays(o, d)
    assert a["hit"].sum() > 5000
    _compare_hits(b, a, "device-built vs uploaded")


def test_device_built_scene_renders_like_uploaded_scene(tracer):
    ts = tree_tubes(iterations=5, seed=8, sides=12, rings=4)
    host = ts.host_mesh()
    w, h = 48, 40
    lo, hi = host.bounds()
    from lsystemeditor_b200.records import look_at_camera
    c = (lo + hi) * 0.5
    cam = look_at_camera((c[0], c[1] + 1.0, c[2] + 9.0), c, fov_y_deg=45.0, aspect=w / h)
    params = default_params(max_path_depth=6, min_samples=8, max_samples_per_pixel=8, background_r=0.1,
                            background_g=0.1, background_b=0.12)
    out = []
    for build in ("host", "device"):
        tracer.configure(w, h)
        if build == "host":
            tracer.set_mesh(host)
        else:
            tracer.batch_set_tubes(0, ts)
        tracer.set_camera(cam)
        tracer.set_params(params)
        tracer.render(0)
        out.append(tracer.readback())
    (ra, ca, _), (rb, cb, _) = out
    assert np.array_equal(ca, cb)
    # identical meshes give identical light lists and, up to exact-t ties in the
    # independently built trees, identical paths
    diff = np.abs(ra - rb).max(axis=-1)
    assert np.mean(diff > 1e-6) < 0.01, f"{np.mean(diff > 1e-6):.4f} of the pixels differ"


def _tonemap_numpy(acc, counts, conv, params, exposure):
    f32 = np.float32
    bg = np.array([params["background_r"], params["background_g"], params["background_b"]], f32)
    rgb = np.where(counts[..., None] > 0, acc[..., :3].astype(f32), bg[None, None, :])
    e = rgb * f32(exposure)
    x = e / (f32(1.0) + e)
    q = (np.minimum(np.maximum(x, f32(0.0)), f32(1.0)) * f32(255.0)).astype(np.uint8)
    out = np.concatenate([q, np.full(q.shape[:2] + (1,), 255, np.uint8)], -1)
    if int(params["debug_overlay_mode"]) == 2:
        out = np.where(conv[..., None] != 0, np.array([0, int(f32(0.35) * f32(255.0)), 0, 255], np.uint8),
                       np.array([255, 0, 0, 255], np.uint8)).astype(np.uint8)
    return out


@pytest.mark.parametrize("overlay", [0, 2])
def test_tonemap_follows_display_pipeline(tracer, overlay):
    mesh = zoo_scene(n_per_mat=60, seed=2)
    w, h = 40, 30
    params = default_params(max_path_depth=5, min_samples=2, max_samples_per_pixel=12, relative_error_threshold=0.5,
                            background_r=0.3, background_g=0.2, background_b=0.1, debug_overlay_mode=overlay)
    tracer.configure(w, h, mesh)
    tracer.set_camera(zoo_camera(w, h))
    tracer.set_params(params)
    tracer.render(3)  # leave some pixels active
    acc, counts, conv = tracer.readback()
    for exposure in (1.0, 0.37, 4.0):
        got = tracer.tonemap(0, exposure)
        want = _tonemap_numpy(acc, counts, conv, params, exposure)
        assert np.array_equal(got, want), exposure
    tracer.reset_accumulation()  # no samples yet: background everywhere
    acc, counts, conv = tracer.readback()
    assert np.array_equal(tracer.tonemap(0, 1.0), _tonemap_numpy(acc, counts, conv, params, 1.0))


def test_exposure_multiplier():
    from lsystemeditor_b200.pathtracer import PathTracer
    f32 = np.float32
    for fs, sh, iso in [(2.8, 1 / 60, 100), (0.01, 0.5, 0.2), (16, 2.0, 3200)]:
        f = max(f32(fs), f32(0.1))
        i = max(f32(iso), f32(1.0))
        want = f32(sh) * (i / f32(100.0)) / (f * f)
        assert PathTracer.exposure_multiplier(fs, sh, iso) == float(want)


def test_device_loft_of_config0_is_the_reference_generator_mesh(tracer):
    """Config 0 built on the device from its tube set (pt_batch_set_tubes with the
    spline frames): bit for bit the host generator's mesh, and -- where the
    reference's own generator is available -- its triangles in its order
    (positions within 1e-5, normals within 1e-4, uvs exactly)."""
    from lsystemeditor_b200.scene import config0_scene
    spec = config0_scene()
    tracer.configure(16, 16)
    tracer.batch_set_tubes(0, spec.tubes)
    dev = tracer.export_mesh(0)
    for f in ("positions", "normals", "uvs", "material_ids"):
        assert np.array_equal(getattr(dev, f), getattr(spec.mesh, f)), f
    from oracle.bindings import ReferenceGenerator, reference_generator_available
    if not reference_generator_available():
        pytest.skip("reference generator build unavailable")
    ref = ReferenceGenerator().build("F(0.1,0.02)\nF(h,r) -> F(h,r)[Yaw(25.7)F(h,r)]F(h,r)[Yaw(0-25.7)F(h,r)]F(h,r)",
                                     4, rotation_deg=(0.0, 90.0, 0.0), sides=8)
    n = ref["positions"].shape[0]
    assert n == 20000
    assert np.abs(dev.positions[:n] - ref["positions"]).max() < 1e-5
    assert np.abs(dev.normals[:n] - ref["normals"]).max() < 1e-4
    assert np.array_equal(dev.uvs[:n], ref["uvs"])
