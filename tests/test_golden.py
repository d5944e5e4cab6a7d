"""The CPU oracle reproduces, bit for bit, outputs of the reference's own code
recorded in tests/golden/reference_golden.npz (generator:
tests/golden/make_golden.py).  Runs everywhere; no reference tree needed."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import OUT, compute


@pytest.fixture(scope="module")
def golden():
    assert os.path.exists(OUT), "run tests/golden/make_golden.py where the reference tree exists"
    return dict(np.load(OUT))


@pytest.fixture(scope="module")
def computed(oracle):
    return compute(oracle)


@pytest.mark.parametrize("key", ["trace_hit", "trace_t", "trace_tri", "trace_normal", "trace_uv", "bsdf_eval",
                                 "bsdf_pdf", "bsdf_dir", "bsdf_spdf", "bsdf_flags", "env_marginal", "env_row",
                                 "env_dir", "env_pdf", "render_acc", "render_counts", "camera_o", "camera_d"])
def test_oracle_matches_reference_golden(golden, computed, key):
    assert np.array_equal(np.asarray(computed[key]), golden[key]), key
