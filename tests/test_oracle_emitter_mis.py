"""The emitter MIS estimator (emitter_mis = 1, an extension) has the
reference estimator's expectation and less variance, checked on the FP64
oracle with independent random numbers (no GPU).

The reference's emissive next-event estimate is always shadowed by the
sampled emitter itself (its shadow ray runs to 1e6), so its emitters are
found by BSDF sampling alone, with weight 1.  In MIS mode, at opaque vertices
the shadow ray stops short of the light sample and BSDF-sampled emitter hits
are balance-weighted against next-event estimation, which estimates the same
integral: the per-pixel means must agree within their standard errors, and
the per-sample luminance variance of lit pixels must drop."""
import numpy as np

from lsystemeditor_b200.scene import config0_scene


def _render(oracle, spec, pixels, spp, mis, seed_base):
    sc = oracle.scene(spec.mesh)
    if mis:
        sc.set_emitter_mis(True)
    p = spec.params.copy()
    p["min_samples"] = p["max_samples_per_pixel"] = spp
    return sc.render(spec.camera, p, spec.width, spec.height, spp, seed_base=seed_base, pixels=pixels, fp64=True)


def test_emitter_mis_keeps_the_expectation_and_lowers_variance(oracle):
    spec = config0_scene(width=48, height=48, spp=1024)
    rng = np.random.default_rng(3)
    # pixels that see lit geometry, chosen from a separate low-sample render
    probe = _render(oracle, spec, None, 16, True, 90_000)
    cand = np.nonzero(probe["lum_mean"] > 1e-3)[0]
    pix = np.sort(rng.choice(cand, min(96, len(cand)), replace=False)).astype(np.int32)
    spp = 1024
    a = _render(oracle, spec, pix, spp, False, 1)
    b = _render(oracle, spec, pix, spp, True, 5000)  # independent random numbers
    n = float(spp)
    ma, mb = a["lum_mean"][pix], b["lum_mean"][pix]
    va, vb = a["m2"][pix] / n, b["m2"][pix] / n  # per-sample luminance variance
    lit = (ma > 1e-3) & (mb > 1e-3)
    assert lit.sum() > 30, "too few lit pixels in the sample"
    se = np.sqrt(va / n + vb / n)
    z = (ma - mb) / np.maximum(se, 1e-12)
    # the images agree in expectation: the pooled difference and each pixel within 4.5 standard errors
    assert abs((ma - mb)[lit].sum()) <= 4.5 * np.sqrt((se[lit] ** 2).sum())
    assert np.mean(np.abs(z[lit]) > 4.5) <= 0.02
    # and MIS mode is the better estimator of the small light
    assert np.median(vb[lit] / np.maximum(va[lit], 1e-30)) < 0.5
