"""Generates tests/golden/reference_golden.npz by running the REFERENCE's own
code compiled for the host (oracle/_ref/libptref.so, built from the reference
tree by oracle/Makefile).  Run here, where the reference tree exists:

    python tests/golden/make_golden.py

The fixtures pin the CPU oracle on machines without the reference tree
(tests/test_golden.py).  Inputs are regenerated from the seeds below.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from lsystemeditor_b200.records import default_params, look_at_camera  # noqa: E402
from oracle.bindings import Checker  # noqa: E402
from tests.helpers import material_zoo, rays_through_bounds, random_soup, sky, zoo_camera, zoo_scene  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.npz")


def inputs():
    """Seeded inputs shared by the generator and the test."""
    d = {}
    soup = random_soup(600, seed=21)
    o, dirs = rays_through_bounds(soup, 3000, seed=22)
    rng = np.random.default_rng(23)
    dirs[:200, rng.integers(0, 3, 200)] = 0.0
    tmin = np.where(rng.uniform(size=len(o)) < 0.8, 0.0, 0.2).astype(np.float32)
    d["trace"] = (soup, o, dirs, tmin)
    nrm = rng.normal(size=(256, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(256, 3)).astype(np.float32)
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(256, 3)).astype(np.float32)
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    u = rng.uniform(size=(256, 2)).astype(np.float32)
    d["bsdf"] = (material_zoo(), nrm, wo, wi, u)
    d["env"] = (sky(24, 12, seed=24), rng.uniform(size=(64, 2)).astype(np.float32))
    mesh = zoo_scene(n_per_mat=40, seed=25)
    d["render"] = (mesh, zoo_camera(20, 16),
                   default_params(background_r=0.1, background_g=0.1, background_b=0.12, max_path_depth=6,
                                  min_samples=4, max_samples_per_pixel=12, relative_error_threshold=0.25),
                   20, 16, 12)
    d["camera"] = (look_at_camera((1, 2, 5), (0, 0, 0), aperture_radius=0.2, focus_distance=4.0),
                   rng.uniform(size=(64, 4)).astype(np.float32))
    return d


def compute(chk: Checker):
    d = inputs()
    out = {}
    soup, o, dirs, tmin = d["trace"]
    r = chk.scene(soup).trace(o, dirs, tmin)
    for k, v in r.items():
        out["trace_" + k] = v
    zoo, nrm, wo, wi, u = d["bsdf"]
    ev, pdf, sd, sp, sf = [], [], [], [], []
    for i in range(len(nrm)):
        m = zoo[i % len(zoo)]
        eta = 1.0 if i % 3 else float(m["ior"])
        ev.append(chk.brdf_eval(nrm[i], wo[i], m, eta, wi[i]))
        pdf.append(chk.brdf_pdf(nrm[i], wo[i], m, eta, wi[i]))
        s = chk.brdf_sample(nrm[i], wo[i], m, eta, float(u[i, 0]), float(u[i, 1]))
        sd.append(s["direction"])
        sp.append(s["pdf"])
        sf.append(int(s["valid"]) | int(s["transmitted"]) << 1 | int(s["subsurface"]) << 2)
    out.update(bsdf_eval=np.array(ev), bsdf_pdf=np.array(pdf, np.float32), bsdf_dir=np.array(sd),
               bsdf_spdf=np.array(sp, np.float32), bsdf_flags=np.array(sf, np.int32))
    img, us = d["env"]
    e = chk.env(img)
    marg, row = e.tables()
    p = default_params()
    es = [e.sample(p, float(a), float(b)) for a, b in us]
    out.update(env_marginal=marg, env_row=row, env_dir=np.array([x[0] for x in es]),
               env_pdf=np.array([x[1] for x in es], np.float32))
    mesh, cam, params, w, h, waves = d["render"]
    st = chk.scene(mesh).render(cam, params, w, h, waves)
    out.update(render_acc=st["acc"], render_counts=st["counts"])
    cam2, lu = d["camera"]
    rays = [chk.camera_ray(cam2, *map(float, x)) for x in lu]
    out.update(camera_o=np.array([x[0] for x in rays]), camera_d=np.array([x[1] for x in rays]))
    return out


def spectral_inputs():
    """Seeded inputs of the spectral fixtures."""
    rng = np.random.default_rng(31)
    lam10 = np.arange(380, 781, 10, dtype=np.float32)
    xyz = rng.uniform(0.0, 1.2, size=(32, 3)).astype(np.float32)
    # coefficient triples in nanometre units of the kind the uplift produces
    c0 = rng.uniform(-1e-3, 1e-3, 256)
    peak = rng.uniform(400.0, 700.0, 256)
    c1 = -2.0 * c0 * peak
    c2 = c0 * peak * peak + rng.uniform(-20.0, 20.0, 256)
    coef = np.stack([c0, c1, c2], 1).astype(np.float32)
    lam = rng.uniform(380.0, 780.0, 256).astype(np.float32)
    return lam10, xyz, coef, lam


def compute_spectral(ref):
    """The reference's spectral helpers (reference build only)."""
    lam10, xyz, coef, lam = spectral_inputs()
    return dict(spec_cie=ref.ref_spectral_cie(lam10), spec_srgb=ref.ref_spectral_xyz_to_srgb(xyz),
                spec_sigmoid=ref.ref_spectral_sigmoid(coef, lam))


if __name__ == "__main__":
    ref = Checker("ref")
    np.savez_compressed(OUT, **compute(ref), **compute_spectral(ref))
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
