"""The emitter MIS estimator on the GPU (pt_render_params.emitter_mis = 1, an
extension with no reference counterpart; the reference estimator is mode 0).

* Parity: with the reference sampler the GPU draws its uniforms and the FP32
  oracle, switched to the same mode, replays them: per-channel relative RMSE
  <= 1e-3 at equal spp, on the material zoo (opaque vertices take part; glass,
  thin and subsurface vertices keep the reference estimator) and on config 0.
* Same expectation as the reference estimator, in RGB and spectral mode: the
  image's mean luminance of both modes agrees within 4.5 standard errors over
  independent seed batches, and MIS mode's batch-to-batch spread is smaller.
* The adjoint replays the reference estimator only, and says so.
"""
import numpy as np
import pytest

from lsystemeditor_b200.records import default_params
from tests.helpers import rel_rmse, zoo_camera, zoo_scene

pytestmark = pytest.mark.gpu

IMAGE_REL_RMSE = 1.0e-3


def _pair(tracer, oracle, mesh, camera, params, w, h, waves, stride):
    tracer.configure(w, h, mesh)
    tracer.set_camera(camera)
    tracer.set_params(params)
    tape = tracer.rng_tape(0, waves, stride)
    tracer.reset_accumulation()
    tracer.render(waves)
    rgba, counts, _ = tracer.readback()
    sc = oracle.scene(mesh).set_emitter_mis(True)
    st = sc.render(camera, params, w, h, waves, seed_base=1, tape=tape, tape_stride=stride)
    assert st["tape_errors"] == 0
    return rgba.reshape(-1, 4), st


def test_emitter_mis_parity_material_zoo(tracer, oracle):
    mesh = zoo_scene()
    w, h, spp = 48, 40, 8
    params = default_params(background_r=0.05, background_g=0.05, background_b=0.08, max_path_depth=8,
                            min_samples=spp, max_samples_per_pixel=spp, emitter_mis=1)
    rgba, st = _pair(tracer, oracle, mesh, zoo_camera(w, h), params, w, h, spp, 200)
    err = rel_rmse(rgba[:, :3], st["acc"][:, :3])
    assert np.all(err <= IMAGE_REL_RMSE), f"relative RMSE {err}"


def test_emitter_mis_parity_config0(tracer, oracle, config0):
    w = h = 64
    spp = 16
    cam = config0.camera.copy()
    cam["aspect"] = 1.0
    params = config0.params.copy()
    params["min_samples"] = params["max_samples_per_pixel"] = spp
    params["emitter_mis"] = 1
    rgba, st = _pair(tracer, oracle, config0.mesh, cam, params, w, h, spp, 160)
    err = rel_rmse(rgba[:, :3], st["acc"][:, :3])
    assert np.all(err <= IMAGE_REL_RMSE), f"relative RMSE {err}"
    assert rgba[:, :3].mean() > 1e-3


@pytest.mark.parametrize("nw", [0, 4])
def test_emitter_mis_keeps_the_expectation(tracer, config0, nw):
    """Both modes over 8 independent seed batches (hash seeds): the image's mean
    luminance agrees within 4.5 standard errors, and on the pixels lit by the
    small light (not seeing it directly) the per-pixel batch-to-batch variance
    of MIS mode is far lower."""
    w = h = 64
    spp, batches = 64, 8
    cam = config0.camera.copy()
    cam["aspect"] = 1.0
    tracer.configure(w, h, config0.mesh)
    tracer.set_camera(cam)
    lum = np.array([0.2126, 0.7152, 0.0722])
    imgs = {}
    for mode in (0, 1):
        vals = []
        for b in range(batches):
            p = config0.params.copy()
            p["min_samples"] = p["max_samples_per_pixel"] = spp
            p["emitter_mis"] = mode
            p["spectral_wavelengths"] = nw
            p["seed_mode"] = 1
            p["seed_value"] = 77 + 1000 * mode + b
            tracer.set_params(p)
            tracer.reset_accumulation()
            tracer.render(0)
            rgba, _, _ = tracer.readback()
            vals.append(rgba[..., :3].reshape(-1, 3).astype(np.float64) @ lum)
        imgs[mode] = np.array(vals)  # (batches, pixels)
    means = {m: imgs[m].mean(axis=1) for m in imgs}
    m0, m1 = means[0].mean(), means[1].mean()
    se = np.sqrt(means[0].var(ddof=1) / batches + means[1].var(ddof=1) / batches)
    assert abs(m0 - m1) <= 4.5 * se, f"mean luminance {m0} (reference) vs {m1} (MIS), se {se}"
    pix_mean = 0.5 * (imgs[0].mean(0) + imgs[1].mean(0))
    lit = (pix_mean > 1e-3) & (pix_mean < 1.0)  # lit geometry, not the emitter itself
    assert lit.sum() > 100
    v0, v1 = imgs[0].var(axis=0, ddof=1)[lit], imgs[1].var(axis=0, ddof=1)[lit]
    assert np.median(v1 / np.maximum(v0, 1e-30)) < 0.25, "MIS mode did not lower the per-pixel variance"


def test_backward_rejects_emitter_mis(tracer, config0):
    from lsystemeditor_b200.pathtracer import PathTracerError
    tracer.configure(16, 16, config0.mesh)
    p = config0.params.copy()
    p["emitter_mis"] = 1
    tracer.set_params(p)
    with pytest.raises(PathTracerError):
        tracer.backward(np.zeros((16, 16, 3), np.float32), 1)
    tracer.set_params(config0.params)
