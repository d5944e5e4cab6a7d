"""Quality of the GPU BVH build: the treelet SAH reordering (Karras & Aila
2013) lowers the SAH cost of the plain Karras LBVH (30-bit Morton codes sorted
by the library's radix sort), and the hits stay the same (exact-t ties go to
the higher triangle index whatever the tree)."""
import numpy as np
import pytest

from tests.helpers import random_soup, rays_through_bounds

pytestmark = pytest.mark.gpu


def _scenes():
    from lsystemeditor_b200.scene import config0_scene, tree_tubes
    return [("config0", config0_scene().mesh),
            ("tree", tree_tubes(iterations=5, seed=7, sides=16, rings=4).host_mesh()),
            ("soup", random_soup(20000, seed=5, extent=6.0, size=0.4))]


@pytest.mark.parametrize("name,mesh", _scenes(), ids=lambda x: x if isinstance(x, str) else "")
def test_treelet_reordering_lowers_sah_and_keeps_hits(tracer, name, mesh):
    o, d = rays_through_bounds(mesh, 50_000, seed=3)
    costs, hits = [], []
    for passes in (0, 1, 2):
        tracer.set_bvh_options(passes)
        tracer.configure(8, 8, mesh)
        costs.append(tracer.bvh_sah_cost())
        hits.append(tracer.trace_rays(o, d))
    tracer.set_bvh_options(1)
    assert costs[1] < 0.99 * costs[0], f"{name}: treelet SAH {costs[1]:.2f} vs plain LBVH {costs[0]:.2f}"
    assert costs[2] <= costs[1] * 1.001, f"{name}: a second pass raised the SAH ({costs[2]:.2f} > {costs[1]:.2f})"
    for h in hits[1:]:
        for k in ("hit", "tri", "t", "normal", "uv"):
            assert np.array_equal(h[k], hits[0][k]), (name, k)
