"""Pins the CPU oracle (this project's restatement) to the reference's own code
compiled for the host (oracle/_ref): every comparison is bit-exact.  Skipped
where the reference tree is not available; tests/test_golden.py carries the
same pins as committed fixtures.
"""
import numpy as np
import pytest

from lsystemeditor_b200.records import PARAMS_DTYPE, default_material, default_params, look_at_camera
from tests.helpers import material_zoo, rays_through_bounds, random_soup, sky, zoo_camera, zoo_scene


def test_record_sizes_match_reference(ref):
    from lsystemeditor_b200.records import CAMERA_DTYPE, MATERIAL_DTYPE, TEXTURE_DTYPE
    assert ref.fn("sizeof_material")() == MATERIAL_DTYPE.itemsize == 96
    assert ref.fn("sizeof_texture")() == TEXTURE_DTYPE.itemsize == 64
    assert ref.fn("sizeof_camera")() == CAMERA_DTYPE.itemsize == 80
    assert ref.fn("sizeof_params")() == 44
    assert ref.fn("sizeof_bvh_node")() == 48


def test_bvh_and_emissive_list_identical(ref, oracle):
    mesh = zoo_scene(n_per_mat=80)
    a, b = oracle.scene(mesh), ref.scene(mesh)
    assert a.bvh_node_count() == b.bvh_node_count() == 2 * mesh.triangle_count - 1
    ia, ca = a.emissive()
    ib, cb = b.emissive()
    assert np.array_equal(ia, ib) and np.array_equal(ca, cb)


@pytest.mark.parametrize("seed", [0, 1])
def test_traversal_bit_exact(ref, oracle, seed):
    mesh = random_soup(2000, seed=seed)
    o, d = rays_through_bounds(mesh, 20_000, seed=seed + 10)
    rng = np.random.default_rng(seed)
    d[:500, rng.integers(0, 3, 500)] = 0.0  # degenerate direction components (quirk Q1)
    tmin = np.where(rng.uniform(size=len(o)) < 0.7, 0.0, 0.3).astype(np.float32)
    ra = oracle.scene(mesh).trace(o, d, tmin)
    rb = ref.scene(mesh).trace(o, d, tmin)
    for k in ra:
        assert np.array_equal(ra[k], rb[k]), k


def _random_frames(rng, n):
    nrm = rng.normal(size=(n, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3)).astype(np.float32)
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3)).astype(np.float32)
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    return nrm, wo, wi


def test_bsdf_bit_exact(ref, oracle):
    rng = np.random.default_rng(3)
    zoo = material_zoo()
    nrm, wo, wi = _random_frames(rng, 400)
    for i in range(400):
        m = zoo[i % len(zoo)]
        eta = 1.0 if i % 3 else float(m["ior"])
        dbg = 0 if i % 7 else (1 << (i % 5))
        u1, u2 = rng.uniform(size=2)
        assert np.array_equal(oracle.brdf_eval(nrm[i], wo[i], m, eta, wi[i], dbg),
                              ref.brdf_eval(nrm[i], wo[i], m, eta, wi[i], dbg))
        assert oracle.brdf_pdf(nrm[i], wo[i], m, eta, wi[i], dbg) == ref.brdf_pdf(nrm[i], wo[i], m, eta, wi[i], dbg)
        sa = oracle.brdf_sample(nrm[i], wo[i], m, eta, u1, u2, dbg)
        sb = ref.brdf_sample(nrm[i], wo[i], m, eta, u1, u2, dbg)
        for k in sa:
            assert np.array_equal(sa[k], sb[k]), (i, k)
        ta = oracle.brdf_sample_transmit(nrm[i], wo[i], m, eta, u1, u2, dbg)
        tb = ref.brdf_sample_transmit(nrm[i], wo[i], m, eta, u1, u2, dbg)
        for k in ta:
            assert np.array_equal(ta[k], tb[k]), (i, k)
        assert np.array_equal(oracle.brdf_apply_throughput([1, 0.5, 0.25], nrm[i], wo[i], m, eta, u1, u2),
                              ref.brdf_apply_throughput([1, 0.5, 0.25], nrm[i], wo[i], m, eta, u1, u2))
        assert np.array_equal(oracle.lobe_weights(m), ref.lobe_weights(m))


def test_textures_bit_exact(ref, oracle):
    mesh = zoo_scene(n_per_mat=10)
    rng = np.random.default_rng(5)
    for i in range(300):
        m = mesh.materials[i % len(mesh.materials)]
        u, v = rng.uniform(-1.5, 2.5, size=2)
        assert np.array_equal(oracle.resolve_material(m, u, v, mesh.textures),
                              ref.resolve_material(m, u, v, mesh.textures))


def test_lights_and_camera_bit_exact(ref, oracle):
    params = default_params(environment_intensity=1.7)
    rng = np.random.default_rng(6)
    img = sky(48, 24)
    ea, eb = oracle.env(img), ref.env(img)
    for x, y in zip(ea.tables(), eb.tables()):
        assert np.array_equal(x, y)
    for _ in range(300):
        u1, u2 = rng.uniform(size=2)
        da, pa = ea.sample(params, u1, u2)
        db, pb = eb.sample(params, u1, u2)
        assert np.array_equal(da, db) and pa == pb
        d = rng.normal(size=3).astype(np.float32)
        assert ea.pdf(params, d) == eb.pdf(params, d)
        assert np.array_equal(ea.eval(params, d), eb.eval(params, d))
    mesh = zoo_scene(n_per_mat=20)
    sa, sb = oracle.scene(mesh), ref.scene(mesh)
    for _ in range(200):
        u = rng.uniform(size=3)
        ra, rb = sa.sample_emissive(*u), sb.sample_emissive(*u)
        assert ra[0] == rb[0] and all(np.array_equal(x, y) for x, y in zip(ra[1:4], rb[1:4])) and ra[4] == rb[4]
    for cam in (look_at_camera((1, 2, 5), (0, 0, 0)),
                look_at_camera((1, 2, 5), (0, 0, 0), aperture_radius=0.2, focus_distance=4.0)):
        for _ in range(100):
            args = rng.uniform(size=4)
            oa, da = oracle.camera_ray(cam, *args)
            ob, db = ref.camera_ray(cam, *args)
            assert np.array_equal(oa, ob) and np.array_equal(da, db)


def test_adaptive_predicate_bit_exact(ref, oracle):
    rng = np.random.default_rng(7)
    for _ in range(2000):
        n = int(rng.integers(0, 64))
        mean = float(rng.choice([0.0, 1e-6, rng.uniform(0, 2)]))
        m2 = float(rng.uniform(0, 1.0) * n * mean * mean)
        mn = int(rng.integers(1, 32))
        thr = float(rng.uniform(0.001, 0.5))
        assert oracle.is_converged(n, mean, m2, mn, thr) == ref.is_converged(n, mean, m2, mn, thr)


@pytest.mark.parametrize("case", ["fixed", "adaptive", "environment"])
def test_render_bit_exact(ref, oracle, case):
    mesh = zoo_scene(n_per_mat=120, seed=11)
    w, h = 32, 24
    env = None
    if case == "fixed":
        waves = 6
        params = default_params(background_r=0.05, background_g=0.05, background_b=0.08, max_path_depth=8,
                                min_samples=waves, max_samples_per_pixel=waves)
    elif case == "adaptive":
        waves = 40
        params = default_params(background_r=0.3, background_g=0.3, background_b=0.3, max_path_depth=5,
                                min_samples=8, max_samples_per_pixel=40, relative_error_threshold=0.3)
    else:
        waves = 4
        params = default_params(max_path_depth=6, min_samples=waves, max_samples_per_pixel=waves,
                                environment_intensity=1.2)
        env = sky(32, 16)
    cam = zoo_camera(w, h)
    ea = oracle.env(env) if env is not None else None
    eb = ref.env(env) if env is not None else None
    sa = oracle.scene(mesh).render(cam, params, w, h, waves, env=ea)
    sb = ref.scene(mesh).render(cam, params, w, h, waves, env=eb)
    for k in ("acc", "counts", "lum_mean", "m2", "converged"):
        assert np.array_equal(sa[k], sb[k]), k
    # the same with a tape (the form the GPU parity tests use)
    rng = np.random.default_rng(12)
    tape = rng.uniform(1e-7, 1.0, (waves, w * h, 160)).astype(np.float32)
    ta = oracle.scene(mesh).render(cam, params, w, h, waves, tape=tape, tape_stride=160, env=ea)
    tb = ref.scene(mesh).render(cam, params, w, h, waves, tape=tape, tape_stride=160, env=eb)
    assert ta["tape_errors"] == tb["tape_errors"] == 0
    assert np.array_equal(ta["acc"], tb["acc"]) and np.array_equal(ta["counts"], tb["counts"])


def test_config0_render_bit_exact(ref, oracle, config0):
    w = h = 48
    cam = config0.camera.copy()
    cam["aspect"] = 1.0
    params = config0.params.copy()
    params["min_samples"] = params["max_samples_per_pixel"] = 4
    sa = oracle.scene(config0.mesh).render(cam, params, w, h, 4)
    sb = ref.scene(config0.mesh).render(cam, params, w, h, 4)
    assert np.array_equal(sa["acc"], sb["acc"])
