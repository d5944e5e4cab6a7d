"""pt_set_params enforces the ranges the reference's setters clamp to
(PathTracer.cpp:126-190), so a C++ caller that fills the record directly gets
the same values as one that goes through the setters."""
import numpy as np
import pytest

from lsystemeditor_b200.records import default_params
from tests.helpers import random_soup

pytestmark = pytest.mark.gpu


def test_set_params_clamps_like_the_reference_setters(tracer):
    tracer.configure(8, 8, random_soup(10, seed=1))
    cases = [
        (dict(max_samples_per_pixel=-5, min_samples=0, relative_error_threshold=0.0, russian_roulette_min_depth=-2),
         dict(max_samples_per_pixel=0, min_samples=1, relative_error_threshold=np.float32(0.001),
              russian_roulette_min_depth=0)),
        (dict(max_samples_per_pixel=5_000_000, min_samples=20_000, relative_error_threshold=7.0),
         dict(max_samples_per_pixel=1_000_000, min_samples=10_000, relative_error_threshold=np.float32(1.0))),
        (dict(relative_error_threshold=float("nan")), dict(relative_error_threshold=np.float32(0.001))),
        (dict(max_samples_per_pixel=64, min_samples=8, relative_error_threshold=0.05),
         dict(max_samples_per_pixel=64, min_samples=8, relative_error_threshold=np.float32(0.05))),
    ]
    for given, expect in cases:
        tracer.set_params(default_params(**given))
        got = tracer.params()
        for k, v in expect.items():
            assert got[k] == v, (given, k, got[k], v)
    tracer.set_params(default_params())
