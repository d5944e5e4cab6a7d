"""Batched form: several scenes rendered together by one renderer.

Every scene of a batch must come out bit-identical to the same scene rendered
alone (same seeds from the pixel's index within its own image, same kernels,
samples folded in the same order), for fixed and adaptive sample counts; the
single-scene parity tests then carry over to every scene of a batch.
"""
import numpy as np
import pytest

from lsystemeditor_b200.records import default_params, look_at_camera
from tests.helpers import sky, zoo_scene

pytestmark = pytest.mark.gpu


def _scenes():
    out = []
    for k, (n, w, h, eye) in enumerate([(120, 40, 32, (0.5, 1.0, 9.0)), (40, 24, 24, (4.0, 2.0, 7.0)),
                                        (200, 56, 30, (-3.0, 0.5, 8.0)), (10, 8, 12, (0.0, 6.0, 2.0))]):
        mesh = zoo_scene(n_per_mat=n, seed=20 + k)
        cam = look_at_camera(eye, (0.0, 0.0, 0.0), fov_y_deg=45.0, aspect=w / h)
        out.append((mesh, cam, w, h))
    return out


def _plain(tracer, scenes, params, env):
    res = []
    for mesh, cam, w, h in scenes:
        tracer.configure(w, h, mesh)
        tracer.set_camera(cam)
        tracer.set_params(params)
        tracer.set_environment(env)
        tracer.reset_accumulation()
        tracer.render(0)
        res.append(tracer.readback())
    return res


def _batched(tracer, scenes, params, env):
    tracer.batch_configure([(w, h) for _, _, w, h in scenes])
    for k, (mesh, cam, w, h) in enumerate(scenes):
        tracer.batch_set_mesh(k, mesh)
        tracer.batch_set_camera(k, cam)
    tracer.set_params(params)
    tracer.set_environment(env)
    tracer.reset_accumulation()
    tracer.render(0)
    return [tracer.batch_readback(k) for k in range(len(scenes))]


@pytest.mark.parametrize("adaptive", [False, True])
def test_batch_equals_scenes_rendered_alone(tracer, adaptive):
    scenes = _scenes()
    if adaptive:
        params = default_params(background_r=0.2, background_g=0.2, background_b=0.25, max_path_depth=5,
                                min_samples=4, max_samples_per_pixel=40, relative_error_threshold=0.3)
        env = None
    else:
        params = default_params(max_path_depth=6, min_samples=6, max_samples_per_pixel=6, environment_intensity=1.2)
        env = sky()
    alone = _plain(tracer, scenes, params, env)
    together = _batched(tracer, scenes, params, env)
    for k, ((ra, ca, va), (rb, cb, vb)) in enumerate(zip(alone, together)):
        assert np.array_equal(ca, cb), f"scene {k}: sample counts differ"
        assert np.array_equal(va, vb), f"scene {k}: convergence flags differ"
        assert np.array_equal(ra, rb), f"scene {k}: image differs"
        assert ra[..., :3].max() > 0
    if adaptive:
        counts = np.concatenate([c.ravel() for _, c, _ in together])
        assert len(np.unique(counts)) > 2, "adaptive sampling did not stop pixels at different counts"
    # the single-scene calls address scene 0 of the batch
    rgba0, counts0, _ = tracer.readback()
    assert np.array_equal(rgba0, together[0][0]) and np.array_equal(counts0, together[0][1])
    # and pt_configure returns the renderer to one scene
    mesh, cam, w, h = scenes[1]
    tracer.configure(w, h, mesh)
    tracer.set_camera(cam)
    tracer.set_params(params)
    tracer.set_environment(env)
    tracer.render(0)
    rgba1, counts1, _ = tracer.readback()
    assert np.array_equal(rgba1, alone[1][0]) and np.array_equal(counts1, alone[1][1])


def test_batch_argument_errors(tracer):
    from lsystemeditor_b200.pathtracer import PathTracerError
    scenes = _scenes()[:2]
    tracer.batch_configure([(w, h) for _, _, w, h in scenes])
    with pytest.raises(PathTracerError):
        tracer.batch_set_mesh(2, scenes[0][0])
    with pytest.raises(PathTracerError):
        tracer.batch_set_camera(-1, scenes[0][1])
    with pytest.raises(PathTracerError):
        tracer.batch_configure([(16, 16), (0, 8)])
    tracer.batch_configure([(w, h) for _, _, w, h in scenes])
    tracer.batch_set_mesh(0, scenes[0][0])
    with pytest.raises(PathTracerError, match="scene 1"):
        tracer.render(1)  # scene 1 has no mesh yet


def test_batch_per_lane_kernels(tracer):
    """The per-lane closest-hit and shadow kernels with the slot-ordered
    next-bounce queue: every scene still equals its render alone, at a path
    capacity small enough that a batch runs in many generations of slots that
    cross scene boundaries."""
    scenes = _scenes()
    params = default_params(background_r=0.2, background_g=0.2, background_b=0.25, max_path_depth=5,
                            min_samples=4, max_samples_per_pixel=24, relative_error_threshold=0.3,
                            emitter_mis=1)
    tracer.set_extend_mode(2)
    tracer.set_tuning(4096, 0)
    try:
        alone = _plain(tracer, scenes, params, None)
        together = _batched(tracer, scenes, params, None)
    finally:
        tracer.set_tuning(0, 0)
        tracer.set_extend_mode(0)
    for k, ((ra, ca, va), (rb, cb, vb)) in enumerate(zip(alone, together)):
        assert np.array_equal(ca, cb), f"scene {k}: sample counts differ"
        assert np.array_equal(ra, rb), f"scene {k}: image differs"
