"""Spectral mode, host side (no GPU needed).

* The colour-matching data the renderer's response table is built from agrees
  with the reference's own tables (Spectral/SpectralCore.h:42-115, recorded by
  tests/golden/make_golden.py): the CIE 1931 2-degree functions to 1e-6.  The
  D65 illuminant is the CIE standard table; the reference's D65 table departs
  from it by up to 4.3% at some wavelengths (580 nm, 690-780 nm), so it is only
  checked to 5%.
* The XYZ -> linear sRGB matrix (derived from the sRGB primaries and white
  point) agrees with the reference's spectralLinearSrgbFromXyz to 5e-4.
* The response table is exactly the stated function of that data, and a flat
  spectrum of 1 maps to RGB (1, 1, 1).
* The uplift reproduces every colour it is given (the spectrum of its
  coefficients, integrated against the response in FP64).
* The oracle's spectrum evaluation is the reference's rgb2specEvalCoefficients
  bit for bit; hero wavelengths are evenly spaced.
* A grey scene renders (oracle, FP32) to the same image in spectral and RGB
  mode up to Monte Carlo noise of the wavelength draw.
"""
import numpy as np
import pytest

from lsystemeditor_b200.pathtracer import PathTracer
from lsystemeditor_b200.records import MATERIAL_DTYPE, default_material, default_params, look_at_camera
from lsystemeditor_b200.scene import HostMesh, quad_mesh
from tests.golden.make_golden import OUT, spectral_inputs
from tests.helpers import random_soup


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(OUT))


@pytest.fixture(scope="module")
def tables():
    return PathTracer.spectral_source_tables()


def test_cmf_matches_reference(golden, tables):
    cie, _ = tables
    ref = golden["spec_cie"]
    assert cie.shape == ref.shape == (41, 4)
    assert np.max(np.abs(cie[:, :3] - ref[:, :3])) <= 1e-6


def test_d65_close_to_reference(golden, tables):
    cie, _ = tables
    ref = golden["spec_cie"].astype(np.float64)
    mine = cie[:, 3].astype(np.float64) / cie[18, 3]
    theirs = ref[:, 3] / ref[18, 3]
    rel = np.abs(mine / theirs - 1.0)
    assert rel.max() <= 0.05, rel.max()
    assert np.median(rel) <= 5e-3


def test_xyz_to_srgb_matches_reference(golden, tables):
    _, m = tables
    _, xyz, _, _ = spectral_inputs()
    mine = xyz.astype(np.float64) @ m.astype(np.float64).T
    ref = golden["spec_srgb"].astype(np.float64)
    assert np.max(np.abs(mine - ref)) <= 5e-4 * np.max(np.abs(ref))


def _response_fp64(cie, m):
    lam = np.arange(401, dtype=np.float64)
    j = np.minimum(lam // 10, 39).astype(int)
    w = (lam - 10 * j) / 10.0
    v = cie[j].astype(np.float64) * (1 - w)[:, None] + cie[j + 1].astype(np.float64) * w[:, None]
    xyz = v[:, :3] * v[:, 3:4]
    resp = xyz @ m.astype(np.float64).T
    wt = np.ones(401)
    wt[0] = wt[-1] = 0.5
    return resp / (wt[:, None] * resp).sum(0)


def test_response_table(tables):
    resp = PathTracer.spectral_response()
    cie, m = tables
    assert resp.shape == (401, 3)
    # m is the float copy of the FP64 matrix the table was built with
    assert np.max(np.abs(resp - _response_fp64(cie, m))) <= 2e-6
    wt = np.ones(401)
    wt[0] = wt[-1] = 0.5
    assert np.allclose((wt[:, None] * resp.astype(np.float64)).sum(0), 1.0, atol=1e-6)


def _spectrum(coef, lam):
    c = coef.astype(np.float64)
    x = c[:, 0:1] * lam * lam + c[:, 1:2] * lam + c[:, 2:3]
    return c[:, 3:4] * (0.5 + x / (2.0 * np.sqrt(1.0 + x * x)))


def test_uplift_round_trip():
    g = np.linspace(0.0, 1.0, 5)
    cols = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    cols = np.concatenate([cols, [[0.35, 0.22, 0.12], [0.1, 0.4, 0.08], [0.999, 0.5, 0.001], [2.0, 1.0, 0.5],
                                  [30.0, 10.0, 2.0], [-1.0, 0.5, 0.2]]]).astype(np.float32)
    coef = PathTracer.spectral_uplift(cols)
    resp = PathTracer.spectral_response().astype(np.float64)
    lam = 380.0 + np.arange(401, dtype=np.float64)
    s = _spectrum(coef, lam)
    wt = np.ones(401)
    wt[0] = wt[-1] = 0.5
    rgb = (s * wt) @ resp
    want = np.maximum(cols.astype(np.float64), 0.0)
    err = np.abs(rgb - want) / np.maximum(1.0, want.max(1, keepdims=True))
    assert err.max() <= 2e-5, (err.max(), cols[err.max(1).argmax()])
    # reflectance spectra of colours in [0, 1] stay in [0, 1]
    inside = (cols >= 0).all(1) & (cols <= 1).all(1)
    assert s[inside].min() >= 0.0 and s[inside].max() <= 1.0 + 1e-6
    # greys are exact constants
    grey = np.isclose(cols[:, 0], cols[:, 1]) & np.isclose(cols[:, 1], cols[:, 2]) & inside
    assert np.all(coef[grey, :3] == 0) and np.allclose(coef[grey, 3], 2 * cols[grey, 0])


def test_oracle_sigmoid_matches_reference(golden, oracle):
    _, _, coef, lam = spectral_inputs()
    ref = golden["spec_sigmoid"]
    mine = np.array([oracle.spec_eval([c[0], c[1], c[2], 1.0], float(l)) for c, l in zip(coef, lam)], np.float32)
    assert np.array_equal(mine, ref)


@pytest.mark.parametrize("nw", [4, 8])
def test_hero_wavelengths_evenly_spaced(oracle, nw):
    rng = np.random.default_rng(4)
    for seed in rng.integers(0, 2 ** 32, 64, dtype=np.uint64):
        lam = np.array([oracle.hero_lambda(int(seed), k, nw) for k in range(nw)])
        assert lam.min() >= 380.0 and lam.max() < 780.0
        d = np.sort((lam - lam[0]) % 400.0)
        assert np.allclose(np.diff(d), 400.0 / nw, atol=1e-3)


def _grey_scene():
    soup = random_soup(300, seed=9, extent=2.0, size=0.6, materials=3)
    greys = [0.2, 0.5, 0.8]
    soup.materials = np.array([default_material(r=v, g=v, b=v, roughness=0.5) for v in greys], MATERIAL_DTYPE)
    ground = quad_mesh((0, -2.5, 0), (10, 0, 0), (0, 0, -10), default_material(r=0.6, g=0.6, b=0.6, roughness=1.0),
                       normal=(0, 1, 0))
    light = quad_mesh((0, 3.5, 0), (2, 0, 0), (0, 0, 2), default_material(r=1, g=1, b=1, emission=6.0),
                      normal=(0, -1, 0))
    return HostMesh.concat([soup, ground, light])


def test_grey_scene_spectral_matches_rgb(oracle):
    from tests.helpers import spectral_inputs as scene_spectral
    w, h, spp = 24, 20, 48
    mesh = _grey_scene()
    cam = look_at_camera((0.0, 1.0, 8.0), (0.0, 0.0, 0.0), fov_y_deg=45.0, aspect=w / h)
    params = default_params(background_r=0.3, background_g=0.3, background_b=0.3, max_path_depth=5,
                            min_samples=spp, max_samples_per_pixel=spp)
    sc = oracle.scene(mesh)
    rgb = sc.render(cam, params, w, h, spp)["acc"][:, :3].astype(np.float64)
    sp = scene_spectral(mesh, params, 8)
    spec = sc.render_spectral(cam, params, w, h, spp, sp)["acc"][:, :3].astype(np.float64)
    # same paths (the wavelength draw takes no random numbers); only the
    # wavelength estimate of white differs per sample
    ratio = spec.mean(0) / rgb.mean(0)
    assert np.all(np.abs(ratio - 1.0) <= 0.02), ratio
