"""The FP64 oracle's path-replay gradient (orc64_backward) against central
finite differences of its own FP64 render on the same random numbers (a
seeded tape).  With Russian roulette off, the estimator is a smooth function
of base colour, sheen and emission (sampling does not depend on them), so the
two agree to ~1e-8 relative.  CPU only."""
import numpy as np
import pytest

from lsystemeditor_b200.scene import config3_scene
from tests.diff_render import PARAMS, apply_theta, theta_of


@pytest.fixture(scope="module")
def case(oracle):
    w, h, spp, stride = 16, 16, 4, 100
    spec = config3_scene(width=w, height=h, spp=spp, seed=4, max_depth=4)
    params = spec.params.copy()
    params["russian_roulette_min_depth"] = 64
    # a grey sky lights the scene through environment next-event estimation (the
    # area light is reached by BSDF sampling only)
    params["background_r"] = params["background_g"] = params["background_b"] = 0.4
    rng = np.random.default_rng(11)
    tape = rng.uniform(1e-7, 1.0, (spp, w * h, stride)).astype(np.float32)
    target = rng.uniform(0.0, 0.2, (w * h, 3))
    return spec, params, w, h, spp, stride, tape, target


def _loss(oracle, spec, params, w, h, spp, stride, tape, target, mats):
    mesh = spec.mesh
    mesh_m = type(mesh)(mesh.positions, mesh.normals, mesh.uvs, mesh.material_ids, mats, mesh.textures)
    st = oracle.scene(mesh_m).render(spec.camera, params, w, h, spp, tape=tape, tape_stride=stride, fp64=True)
    img = st["acc"][:, :3]
    return float(((img - target) ** 2).sum()), img


@pytest.mark.parametrize("name,mat", [("r", 2), ("g", 5), ("b", 8), ("sheen", 5), ("emission", 9)])
def test_oracle_gradient_matches_finite_differences(oracle, case, name, mat):
    spec, params, w, h, spp, stride, tape, target = case
    mats = spec.mesh.materials
    theta = theta_of(mats)
    l0, img = _loss(oracle, spec, params, w, h, spp, stride, tape, target, mats)
    d_image = (2.0 * (img - target)).astype(np.float32)
    g, underruns = oracle.scene(spec.mesh).backward(spec.camera, params, w, h, spp, tape, stride, d_image, 10)
    assert underruns == 0
    j = PARAMS.index(name)
    step = 1e-4
    tp, tm = theta.copy(), theta.copy()
    tp[mat, j] += step
    tm[mat, j] -= step
    # the step actually taken: the material record stores float32
    dx = float(np.float32(tp[mat, j])) - float(np.float32(tm[mat, j]))
    fd = (_loss(oracle, spec, params, w, h, spp, stride, tape, target, apply_theta(mats, tp))[0] -
          _loss(oracle, spec, params, w, h, spp, stride, tape, target, apply_theta(mats, tm))[0]) / dx
    assert abs(g[mat, j] - fd) <= 2e-5 * abs(fd) + 1e-9, (name, mat, g[mat, j], fd)
    assert abs(fd) > 1e-8
