"""Known-answer and property checks carried over from the reference's own
tests (PathTracerLib/tests/*), run against the CPU oracle.  The same
functions run on the GPU in tests/test_gpu_parity.py."""
import math

import numpy as np

from lsystemeditor_b200.records import MATERIAL_DTYPE, TEXTURE_DTYPE, default_material, default_params
from lsystemeditor_b200.scene import HostMesh

N_UP = np.array([0.0, 0.0, 1.0], np.float32)
WO = np.array([0.2, 0.1, 1.0], np.float32) / np.linalg.norm([0.2, 0.1, 1.0])
WO_INSIDE = np.array([0.2, 0.1, -1.0], np.float32) / np.linalg.norm([0.2, 0.1, -1.0])


def glass(**kw):
    return default_material(r=1.0, g=1.0, b=1.0, roughness=0.0, transmission=1.0, ior=1.5, **kw)


def one_triangle():
    pos = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32)
    nrm = np.array([[[0, 0, 1]] * 3], np.float32)
    uv = np.array([[[0, 0], [1, 0], [0, 1]]], np.float32)
    return HostMesh(pos, nrm, uv, np.zeros(1, np.uint32), np.array([default_material()], MATERIAL_DTYPE),
                    np.zeros(0, TEXTURE_DTYPE))


# --- PathTracerMeshUvTests.cpp:264-287 -------------------------------------
def test_interpolates_uv_at_hit(oracle):
    # The reference test calls meshAccelRayTriangle directly with d = (0, 0, -1).  Through the
    # traversal such a ray falls under quirk Q1, so the same hit point is reached with a
    # slightly tilted ray.
    d = np.array([1e-3, 1e-3, -1.0], np.float32)
    o = np.array([0.25, 0.25, 0.0], np.float32) - d
    r = oracle.scene(one_triangle()).trace([o], [d], 0.0, 10.0)
    assert r["hit"][0]
    assert abs(r["uv"][0, 0] - 0.25) < 1e-5 and abs(r["uv"][0, 1] - 0.25) < 1e-5


# --- quirk Q1 (MeshAccelIntersectCore.h:125-128 with :32-44) ------------------
def test_zero_direction_component_quirk(oracle):
    """A zero reciprocal turns each slab test into "origin inside the box on the other axes"."""
    sc = oracle.scene(one_triangle())
    # straight down onto the triangle: the origin's z (1) is outside the box's z range [0, 0] -> miss
    assert not sc.trace([[0.25, 0.25, 1.0]], [[0.0, 0.0, -1.0]], 0.0)["hit"][0]
    # the same ray tilted by 1e-3: an ordinary hit
    assert sc.trace([[0.25, 0.25, 1.0]], [[1e-3, 1e-3, -1.0]], 0.0)["hit"][0]
    # origin on the triangle's plane: inside the box -> tested and hit at t = 0 ...
    assert sc.trace([[0.25, 0.25, 0.0]], [[0.0, 0.0, -1.0]], 0.0)["hit"][0]
    # ... but any tMin > 0 fails every slab test
    assert not sc.trace([[0.25, 0.25, 0.0]], [[0.0, 0.0, -1.0]], 1e-3)["hit"][0]


# --- PathTracerProceduralTextureTests.cpp:52-131 -------------------------------
def grid(ar, ag, ab, br, bg, bb, freq, thick):
    t = np.zeros((), TEXTURE_DTYPE)
    t["kind"] = 2
    t["p0"] = [freq, freq, thick, 0.0]
    t["p1"] = [ar, ag, ab, 0.0]
    t["p2"] = [br, bg, bb, 0.0]
    return t


def test_texture_grid_and_stripe(oracle):
    bank = np.zeros(3, TEXTURE_DTYPE)
    bank[1] = grid(1, 0, 0, 0, 1, 0, 4.0, 0.05)
    bank[2]["kind"] = 3
    bank[2]["p0"] = [2.0, 0.5, 0.25, 1.0]
    m = default_material(albedo_tex=1)
    assert np.allclose(oracle.resolve_material(m, 0.3, 0.3, bank)[:3], [1, 0, 0], atol=1e-5)  # off the lines
    assert np.allclose(oracle.resolve_material(m, 0.0, 0.0, bank)[:3], [0, 1, 0], atol=1e-5)  # on the lines
    split = np.zeros(2, TEXTURE_DTYPE)
    split[1]["kind"] = 2
    split[1]["p0"] = [20.0, 2.0, 0.05, 0.0]
    split[1]["p1"] = [1, 0, 0, 0]
    split[1]["p2"] = [0, 1, 0, 0]
    assert abs(oracle.resolve_material(m, 0.03, 0.02, split)[1] - 1.0) < 1e-5
    s = default_material(roughness_tex=2)
    assert abs(oracle.resolve_material(s, 0.0, 0.0, bank)[3] - 0.25) < 1e-5   # stripe on (u1d = u)
    assert abs(oracle.resolve_material(s, 0.4, 0.0, bank)[3] - 1.0) < 1e-5    # stripe off
    inline = default_material(r=0.2, g=0.3, b=0.4, roughness=0.7)
    assert np.allclose(oracle.resolve_material(inline, 0.25, 0.75, None)[[0, 1, 2, 3]], [0.2, 0.3, 0.4, 0.7])


# --- PathTracerAdaptiveSamplingTests.cpp:17-52 ---------------------------------
def test_adaptive_convergence_predicate(oracle):
    assert oracle.is_converged(16, 1.0, 0.0001, 16, 0.02)
    assert not oracle.is_converged(16, 1.0, 0.25, 16, 0.02)
    assert not oracle.is_converged(8, 1.0, 0.0001, 16, 0.02)
    assert not oracle.is_converged(32, 0.0, 0.0, 32, 0.005)
    assert not oracle.is_converged(64, 1.0e-6, 1.0e-8, 32, 0.02)


# --- PathTracerExposureTests.cpp:104-144 ---------------------------------------
def test_solid_environment_pdf_and_radiance(oracle):
    p = default_params(background_r=1.0, background_g=1.0, background_b=1.0, environment_intensity=2.0)
    d, pdf = oracle.env_sample_solid(p, 0.3, 0.6)
    assert abs(pdf - 1.0 / (4.0 * 3.14159265)) < 1e-6
    assert abs(oracle.env_pdf_solid(p, [0, 1, 0]) - 1.0 / (4.0 * 3.14159265)) < 1e-6
    assert np.allclose(oracle.env_eval_solid(p, [0, 1, 0]), [2.0, 2.0, 2.0], atol=1e-6)
    assert abs(np.linalg.norm(d) - 1.0) < 1e-5


def test_environment_pdf_includes_resolution(oracle):
    """The lat-long pdf carries the width*height solid-angle factor (PathTracerExposureTests.cpp:104-116)."""
    img = np.ones((8, 16, 3), np.float32)
    e = oracle.env(img)
    p = default_params()
    d, pdf = e.sample(p, 0.5, 0.5)
    # a uniform map weighted by sin(theta) samples the sphere uniformly: pdf ~ 1/(4 pi); without
    # the width*height factor it would be smaller by W*H = 128
    assert abs(pdf - 1.0 / (4 * np.pi)) * 4 * np.pi < 0.02


# --- PathTracerPrincipledBrdfTests.cpp:80-389 -----------------------------------
def test_transmissive_sample_throughput_near_one(oracle):
    s = oracle.brdf_sample(N_UP, WO, glass(), 1.0, 0.6, 0.5)
    assert s["valid"] and s["transmitted"]
    t = oracle.brdf_apply_throughput([1, 1, 1], N_UP, WO, glass(), 1.0, 0.6, 0.5)
    assert abs(t[0] - 1.0) < 0.15
    s = oracle.brdf_sample(N_UP, WO, glass(), 1.0, 0.99, 0.5)
    assert s["valid"] and not s["transmitted"]
    t = oracle.brdf_apply_throughput([1, 1, 1], N_UP, WO, glass(), 1.0, 0.99, 0.5)
    assert abs(t[0] - 1.0) < 0.15


def test_thin_and_subsurface_and_metal_samples(oracle):
    thin = default_material(r=0.2, g=0.8, b=0.1, roughness=0.5, transmission=1.0, thin=1.0)
    s = oracle.brdf_sample(N_UP, WO, thin, 1.0, 0.6, 0.5)
    assert s["valid"] and s["transmitted"] and abs(np.dot(s["direction"], -WO) - 1.0) < 0.01
    sss = default_material(r=0.9, g=0.85, b=0.7, roughness=0.85, subsurface=0.8, diffuse_roughness=0.85,
                           scatter_radius_r=0.05, scatter_radius_g=0.04, scatter_radius_b=0.02)
    s = oracle.brdf_sample(N_UP, WO, sss, 1.0, 0.95, 0.25)
    assert s["valid"] and s["direction"][2] > 0 and s["subsurface"]
    metal = default_material(r=0.9, g=0.9, b=0.9, roughness=0.3, metallic=1.0)
    s = oracle.brdf_sample(N_UP, WO, metal, 1.0, 0.5, 0.5)
    assert s["valid"] and s["direction"][2] > 0
    w = oracle.lobe_weights(metal)
    assert w[0] < 0.01 and w[2] < 0.01 and w[3] < 0.01


def test_lobe_weights_and_env_nee_skip(oracle):
    w = oracle.lobe_weights(glass())
    assert w[2] >= 0.99 and w[1] < 0.01


def test_forced_refract_reflect_and_debug_flags(oracle):
    s = oracle.brdf_sample_transmit(N_UP, WO, glass(), 1.0, 0.0, 0.5)
    assert s["valid"] and s["transmitted"] and abs(s["next_eta"] - 1.5) < 0.01 and s["direction"][2] < 0
    s = oracle.brdf_sample_transmit(N_UP, WO, glass(), 1.0, 1.0, 0.5)
    assert s["valid"] and not s["transmitted"] and abs(s["next_eta"] - 1.0) < 0.01 and s["direction"][2] > 0
    s = oracle.brdf_sample_transmit(N_UP, WO, glass(), 1.0, 0.0, 0.5, debug=1 << 1)  # kDisableRefract
    assert s["valid"] and not s["transmitted"] and s["direction"][2] > 0
    s = oracle.brdf_sample_transmit(N_UP, WO, glass(), 1.0, 1.0, 0.5, debug=1 << 2)  # kDisableReflect
    assert s["valid"] and s["transmitted"] and abs(s["next_eta"] - 1.5) < 0.01
    s = oracle.brdf_sample(N_UP, WO, glass(), 1.0, 0.5, 0.5, debug=1 << 0)           # kForceTransmitLobeOnly
    assert s["valid"] and (s["transmitted"] or s["direction"][2] > 0)


def test_glass_medium_enter_and_exit(oracle):
    enter = oracle.brdf_sample_transmit(N_UP, WO, glass(), 1.0, 0.0, 0.5)
    assert enter["transmitted"] and abs(enter["next_eta"] - 1.5) < 0.01
    leave = oracle.brdf_sample_transmit(N_UP, WO_INSIDE, glass(), enter["next_eta"], 0.0, 0.5)
    assert leave["transmitted"] and abs(leave["next_eta"] - 1.0) < 0.01
    water = default_material(r=1, g=1, b=1, roughness=0.0, transmission=1.0, ior=1.33)
    e = oracle.brdf_sample_transmit(N_UP, WO, water, 1.0, 0.0, 0.5)
    assert e["transmitted"] and abs(e["next_eta"] - 1.33) < 0.01


def test_rough_metal_energy_compensation_visible(oracle):
    metal = default_material(r=0.9, g=0.9, b=0.9, roughness=0.85, metallic=1.0)
    s = oracle.brdf_sample(N_UP, WO, metal, 1.0, 0.3, 0.6)
    assert s["valid"]
    f = oracle.brdf_eval(N_UP, WO, metal, 1.0, s["direction"])
    assert f[0] > 0.01


def test_diffuse_throughput_range(oracle):
    m = default_material(r=0.8, g=0.8, b=0.8, roughness=0.5)
    for u1 in (0.1, 0.3, 0.5, 0.7, 0.9):
        for u2 in (0.2, 0.5, 0.8):
            t = oracle.brdf_apply_throughput([1, 1, 1], N_UP, WO, m, 1.0, u1, u2)
            assert 0.0 <= t[0] < 1.5
