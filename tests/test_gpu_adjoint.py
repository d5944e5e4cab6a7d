"""Differentiable rendering: the path-replay adjoint (pt_backward).

* Against the FP64 host oracle's path-replay gradient on the same random
  numbers (GPU tape): every gradient entry agrees within 2e-3 of the largest
  entry of its parameter kind (FP32 vs FP64 arithmetic and the FP32 difference
  quotients of roughness / metallic).
* Against Richardson-extrapolated central differences of the rendered loss
  with the same seeds: for base colour, sheen and emission the estimator is a
  smooth function of those parameters (sampling does not depend on them;
  Russian roulette switched off), so they agree up to the FP32 rounding of the
  rendered image (relative 1e-3 plus an absolute 1e-3).
* Through torch.autograd: Adam steps on the branch materials' base colours
  reduce an L2 image loss against a target rendered from other colours.
"""
import numpy as np
import pytest

from lsystemeditor_b200.scene import config3_scene, diff_materials
from tests.diff_render import PARAMS, apply_theta, theta_of

pytestmark = pytest.mark.gpu


def _setup(tracer, w, h, spp, depth=6, rr_min=3, seed=3):
    spec = config3_scene(width=w, height=h, spp=spp, seed=seed, max_depth=depth)
    p = spec.params.copy()
    p["russian_roulette_min_depth"] = rr_min
    # a grey sky lights the scene through environment next-event estimation (the
    # area light is reached by BSDF sampling only, its NEE shadow ray always
    # hitting the light itself)
    p["background_r"] = p["background_g"] = p["background_b"] = 0.4
    tracer.configure(w, h, spec.mesh)
    tracer.set_camera(spec.camera)
    tracer.set_params(p)
    return spec, p


def _render(tracer, mats, spp):
    tracer.set_materials(mats)
    tracer.reset_accumulation()
    tracer.render(spp)
    rgba, counts, _ = tracer.readback()
    assert np.all(counts == spp)
    return rgba[..., :3].astype(np.float64)


def test_adjoint_matches_fp64_oracle(tracer, oracle):
    w, h, spp, stride = 40, 40, 4, 120
    spec, params = _setup(tracer, w, h, spp)
    mats = spec.mesh.materials
    target = _render(tracer, apply_theta(mats, theta_of(mats) * 0.9), spp)
    img = _render(tracer, mats, spp)
    d_image = (2.0 * (img - target)).astype(np.float32)
    g_gpu, ms = tracer.backward(d_image, spp)
    tape = tracer.rng_tape(0, spp, stride)
    sc = oracle.scene(spec.mesh)
    g_orc, underruns = sc.backward(spec.camera, params, w, h, spp, tape, stride, d_image, 16)
    assert underruns == 0
    M = len(mats)
    a, b = g_gpu[:M].astype(np.float64), g_orc[:M]
    assert np.abs(b).max() > 0
    for j, name in enumerate(PARAMS):
        scale = np.abs(b[:, j]).max()
        if scale == 0:
            assert np.all(a[:, j] == 0), name
            continue
        err = np.abs(a[:, j] - b[:, j]).max() / scale
        assert err < 2e-3, f"{name}: max error {err:.2e} of max |grad| {scale:.3e}\n{a[:, j]}\n{b[:, j]}"


@pytest.mark.parametrize("name", ["r", "g", "b", "sheen", "emission"])
def test_adjoint_matches_finite_differences(tracer, name):
    w, h, spp = 64, 64, 8
    spec, params = _setup(tracer, w, h, spp, depth=5, rr_min=64)  # no Russian roulette
    mats = spec.mesh.materials
    rng = np.random.default_rng(5)
    target = rng.uniform(0.0, 0.3, (h, w, 3))
    j = PARAMS.index(name)

    def loss(theta):
        img = _render(tracer, apply_theta(mats, theta), spp)
        return float(((img - target) ** 2).sum()), img

    theta = theta_of(mats)
    l0, img = loss(theta)
    g, _ = tracer.backward((2.0 * (img - target)).astype(np.float32), spp)

    def central(m, step):
        tp, tm = theta.copy(), theta.copy()
        tp[m, j] += step
        tm[m, j] -= step
        dx = float(np.float32(tp[m, j])) - float(np.float32(tm[m, j]))  # float32 material record
        return (loss(tp)[0] - loss(tm)[0]) / dx

    # Richardson-extrapolated central differences.  The image is accumulated in
    # FP32, which puts a noise floor of a few 1e-3 (absolute) on a difference
    # quotient of this loss at steps ~1e-2, so the steps are as large as the
    # parameter's range allows; the FP64 oracle test pins the gradient itself.
    mats_to_check = [9] if name == "emission" else ([0, 3, 6] if name == "sheen" else [0, 3, 6, 8])
    for m in mats_to_check:
        x = theta[m, j]
        step = 0.5 if name == "emission" else min(0.05, x / 4.0, (1.0 - x) / 4.0)
        fd = (4.0 * central(m, step) - central(m, 2.0 * step)) / 3.0
        assert abs(g[m, j] - fd) <= 1e-3 * abs(fd) + 1e-3, (name, m, g[m, j], fd)


@pytest.mark.parametrize("name", ["roughness", "metallic"])
def test_adjoint_matches_finite_differences_in_expectation(tracer, name):
    """Roughness and metallic change how directions and lobes are sampled, so the
    fixed-seed estimate is not a smooth function of them and the difference
    quotient of one render is not their gradient.  For a loss linear in the image
    (weights w), the path-replay gradient (sampling detached) and a central
    difference of two renders with common random numbers are both unbiased
    estimates of d E[loss] / d theta (the difference up to O(step^2)).  Over K
    independent seed batches (hash seeds) their means must agree within four
    combined standard errors plus 2%, and the gradient must be resolved."""
    w = h = 32
    spp, K, m, step = 16, 24, 8, 0.05
    spec, params = _setup(tracer, w, h, spp, depth=5, rr_min=64)  # no Russian roulette
    mats = spec.mesh.materials.copy()
    mats[m]["roughness"] = 0.5   # the ground: half the image, away from the parameter bounds
    mats[m]["metallic"] = 0.2
    j = PARAMS.index(name)
    wgt = np.random.default_rng(11).uniform(0.5, 1.5, (h, w, 3))
    theta = theta_of(mats)
    tp, tm = theta.copy(), theta.copy()
    tp[m, j] += step
    tm[m, j] -= step
    dx = float(np.float32(tp[m, j])) - float(np.float32(tm[m, j]))
    grads, fds = [], []
    for k in range(K):
        p = params.copy()
        p["seed_mode"] = 1
        p["seed_value"] = 1000 + k
        tracer.set_params(p)
        _render(tracer, mats, spp)
        g, _ = tracer.backward(wgt.astype(np.float32), spp)
        grads.append(float(g[m, j]))
        lp = float((wgt * _render(tracer, apply_theta(mats, tp), spp)).sum())
        lm = float((wgt * _render(tracer, apply_theta(mats, tm), spp)).sum())
        fds.append((lp - lm) / dx)
    grads, fds = np.array(grads), np.array(fds)
    se = np.sqrt(grads.var(ddof=1) / K + fds.var(ddof=1) / K)
    gm, fm = grads.mean(), fds.mean()
    assert abs(gm) > 4.0 * grads.std(ddof=1) / np.sqrt(K), f"{name}: gradient not resolved ({gm} +- {grads.std()})"
    assert abs(gm - fm) <= 4.0 * se + 0.02 * abs(fm), f"{name}: path replay {gm:.4f} vs difference {fm:.4f} (se {se:.4f})"


def test_torch_autograd_reduces_loss(tracer):
    """Adam on the branch materials' base colours through torch.autograd
    (Russian roulette off, so the fixed-seed loss is smooth in them)."""
    torch = pytest.importorskip("torch")
    from tests.diff_render import RenderImage
    w, h, spp = 48, 48, 8
    spec, params = _setup(tracer, w, h, spp, depth=5, rr_min=64)
    truth = spec.mesh.materials
    target = torch.from_numpy(_render(tracer, truth, spp).astype(np.float32))
    init = truth.copy()
    wrong = diff_materials(np.random.default_rng(99), 8)
    for c in ("r", "g", "b"):
        init[c][:8] = wrong[c]
    theta = torch.tensor(theta_of(init), dtype=torch.float64, requires_grad=True)
    mask = torch.zeros_like(theta)
    mask[:8, 0:3] = 1.0
    opt = torch.optim.Adam([theta], lr=2e-2)
    losses = []
    for _ in range(15):
        opt.zero_grad()
        img = RenderImage.apply(theta, tracer, truth, spp)
        loss = ((img.double() - target.double()) ** 2).sum()
        loss.backward()
        assert theta.grad is not None and torch.isfinite(theta.grad).all()
        theta.grad *= mask
        opt.step()
        with torch.no_grad():
            theta[:, 0:3].clamp_(0.0, 1.0)
        losses.append(float(loss))
    assert losses[-1] < 0.5 * losses[0], losses


def test_recorded_samples_give_the_replayed_gradient(tracer):
    """pt_record_samples: the adjoint reads each sample's radiance kept by the
    forward render instead of replaying the path a first time; the gradient is
    the same (up to the FP32 rounding differences of the two kernels)."""
    w, h, spp = 48, 40, 6
    spec, params = _setup(tracer, w, h, spp)
    mats = spec.mesh.materials
    target = np.full((h, w, 3), 0.1)
    img = _render(tracer, mats, spp)
    d_image = (2.0 * (img - target)).astype(np.float32)
    g_replay, ms_replay = tracer.backward(d_image, spp)
    tracer.record_samples(spp)
    img2 = _render(tracer, mats, spp)
    assert np.array_equal(img, img2)
    g_rec, ms_rec = tracer.backward(d_image, spp)
    M = len(mats)
    scale = np.abs(g_replay[:M]).max(axis=0)
    err = np.abs(g_rec[:M] - g_replay[:M]) / np.maximum(scale, 1e-30)
    assert err.max() < 1e-4, err.max()
    # a render with other parameters invalidates the record: back to the replay
    p2 = params.copy()
    p2["max_path_depth"] = 3
    tracer.set_params(p2)
    tracer.render(spp)
    tracer.set_params(params)
    g_again, _ = tracer.backward(d_image, spp)
    assert np.allclose(g_again[:M], g_replay[:M], rtol=0, atol=1e-4 * scale.max())
    tracer.record_samples(0)
