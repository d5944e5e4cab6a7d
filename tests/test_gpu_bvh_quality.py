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


def test_coincident_triangles_trace_without_stack_overflow(tracer, oracle):
    """2500 coincident copies of 8 triangles: every Morton key collides, the
    deepest tree the builder makes.  No traversal stack overflows (counted into
    pt_stats.stack_overflows for queries and renders), the hits equal the
    oracle's in hit flag and t, and every hit is the highest-indexed copy (the
    tie rule), also for rays with exact-zero direction components."""
    from lsystemeditor_b200.scene import HostMesh
    base = random_soup(8, seed=1, extent=1.0, size=0.5)
    copies = 2500
    mesh = HostMesh(np.tile(base.positions, (copies, 1, 1)), np.tile(base.normals, (copies, 1, 1)),
                    np.tile(base.uvs, (copies, 1, 1)), np.tile(base.material_ids, copies), base.materials,
                    base.textures)
    tracer.configure(8, 8, mesh)
    before = tracer.stats()["stack_overflows"]
    o, d = rays_through_bounds(mesh, 20_000, seed=4)
    d[:2000, 0] = 0.0  # exact-zero direction components take the reference's slab-test path
    g = tracer.trace_rays(o, d)
    r = oracle.scene(mesh).trace(o, d)
    assert tracer.stats()["stack_overflows"] == before
    assert g["hit"].sum() > 1000
    assert np.array_equal(g["hit"], r["hit"])
    assert np.array_equal(g["t"][g["hit"]], r["t"][r["hit"]])
    assert np.all(g["tri"][g["hit"]] >= 8 * (copies - 1))
