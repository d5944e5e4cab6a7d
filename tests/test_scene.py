"""Scene generator used by the benchmark workloads."""
import numpy as np

from lsystemeditor_b200.scene import bracketed_ol_tree, config0_scene, expand


def test_bracketed_tree_counts():
    tree = bracketed_ol_tree()
    # 5^4 = 625 segments, each an 8-gon tube with two rings and two caps = 32 triangles
    assert tree.triangle_count == 625 * 32


def test_config0_scene_layout():
    spec = config0_scene()
    m = spec.mesh
    assert m.triangle_count == 625 * 32 + 4
    assert len(m.materials) == 3 and float(m.materials[2]["emission"]) == 10.0
    n = np.linalg.norm(m.normals, axis=-1)
    assert np.allclose(n, 1.0, atol=1e-5)
    lo, hi = m.bounds()
    assert hi[1] > 8.0 and abs(lo[1]) < 1e-6  # the root pitch of 90 degrees in single precision
    assert int(spec.params["min_samples"]) == int(spec.params["max_samples_per_pixel"]) == 64
    assert int(spec.params["max_path_depth"]) == 8


def test_expand_is_seeded():
    rules = {"A": lambda a, rng: [("F", ()), ("A", ())] if rng.uniform() < 0.5 else [("A", ()), ("F", ())]}
    a = expand([("A", ())], rules, 8, seed=3)
    b = expand([("A", ())], rules, 8, seed=3)
    assert a == b
