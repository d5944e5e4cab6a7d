"""Frame-loop graphs and the autotuner (GPU).

* The bounce loop replayed from CUDA graphs (the default) renders exactly what
  the same loop launched kernel by kernel renders (stage profiling turns the
  graphs off), for a plain scene, a spectral render and a batch of views.
* pt_autotune returns knobs from its candidate sets, never a slower probe
  than the configuration it started from, and the image rendered with the
  chosen knobs is bit-identical to the one rendered with the defaults.
"""
import numpy as np
import pytest

from lsystemeditor_b200.pathtracer import PROFILE_STAGE_TIMES, PathTracer
from lsystemeditor_b200.records import default_params
from tests.helpers import spectral_zoo_scene, zoo_camera

pytestmark = pytest.mark.gpu


def _render(t, profile):
    t.set_profiling(PROFILE_STAGE_TIMES if profile else 0)
    t.reset_accumulation()
    t.render(0)
    out = t.readback()[0].copy()
    t.set_profiling(0)
    return out


@pytest.mark.parametrize("nw", [0, 8])
def test_graphs_match_direct_launches(nw):
    mesh = spectral_zoo_scene(n_per_mat=150, seed=8)
    w, h = 64, 48
    params = default_params(background_r=0.1, background_g=0.12, background_b=0.2, max_path_depth=8,
                            min_samples=8, max_samples_per_pixel=24, relative_error_threshold=0.3,
                            spectral_wavelengths=nw)
    with PathTracer(0) as t:
        t.configure(w, h, mesh)
        t.set_camera(zoo_camera(w, h))
        t.set_params(params)
        graphed = _render(t, False)
        direct = _render(t, True)
        assert np.array_equal(graphed, direct)


def test_autotune_keeps_the_image():
    mesh = spectral_zoo_scene(n_per_mat=150, seed=9)
    w, h = 96, 64
    params = default_params(background_r=0.1, background_g=0.12, background_b=0.2, max_path_depth=8,
                            min_samples=16, max_samples_per_pixel=16)
    with PathTracer(0) as t:
        t.configure(w, h, mesh)
        t.set_camera(zoo_camera(w, h))
        t.set_params(params)
        t.render(0)
        before = t.readback()[0].copy()
        tune = t.autotune(waves=4)
        assert tune["path_capacity"] in (1 << 20, 1 << 21, 1 << 22, 1 << 23)
        assert tune["blocks_per_sm"] in (0, 2, 3, 4)
        assert tune["samples_per_launch"] in (0, 4, 16, 64)
        assert tune["trials"] >= 2 and tune["ms_best"] <= tune["ms_default"]
        t.render(0)
        after = t.readback()[0]
        assert np.array_equal(before, after), "the tuned knobs changed the image"
