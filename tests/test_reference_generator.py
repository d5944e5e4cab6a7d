"""The scene generator pinned to the reference's own (no GPU).

The reference's L-system evaluator, turtle and Hermite spline
(LSystemLib, Application/src/Procedural/Turtle.cpp, Spline.cpp, compiled
unchanged into oracle/_ref/libptref_gen.so, with the loft of Loft.cpp:108-155
and the root transform restated beside them) generate config 0 from its
grammar in the reference's own syntax; the product's generator (expand ->
turtle -> spline_frames -> root rotation -> loft) must give the same triangles
in the same order: positions within 1e-5 (the reference runs its turtle in
single precision, the product in double), normals within 1e-4, uvs exactly.
A curved segment (rotations between the forward steps of one segment) takes
the refinement path of Spline.cpp: the product's frames match the reference's.
"""
import numpy as np
import pytest

from lsystemeditor_b200 import scene as S

CONFIG0_GRAMMAR = "F(0.1,0.02)\nF(h,r) -> F(h,r)[Yaw(25.7)F(h,r)]F(h,r)[Yaw(0-25.7)F(h,r)]F(h,r)"


@pytest.fixture(scope="module")
def refgen():
    from oracle.bindings import ReferenceGenerator, reference_generator_available
    if not reference_generator_available():
        pytest.skip("reference generator build unavailable (no reference tree where build() ran)")
    return ReferenceGenerator()


def _config0_word():
    def rule(args, _rng):
        h, r = args
        F = ("F", (h, r))
        return [F, ("[", ()), ("Yaw", (25.7,)), F, ("]", ()), F, ("[", ()), ("Yaw", (-25.7,)), F, ("]", ()), F]
    return S.expand([("F", (0.1, 0.02))], {"F": rule}, 4)


def test_config0_tree_matches_the_reference_generator(refgen):
    ref = refgen.build(CONFIG0_GRAMMAR, 4, rotation_deg=(0.0, 90.0, 0.0), sides=8)
    assert ref["positions"].shape[0] == 625 * 32 and ref["skipped"] == 0
    mine = S.bracketed_ol_tree()                  # the product's config-0 tree
    segs, _ = S.reference_tree(_config0_word())
    assert len(segs) == 625
    assert mine.triangle_count == ref["positions"].shape[0]
    assert np.abs(mine.positions - ref["positions"]).max() < 1e-5
    assert np.abs(mine.normals - ref["normals"]).max() < 1e-4
    assert np.array_equal(mine.uvs, ref["uvs"])


def test_config0_scene_tree_is_the_reference_tree(refgen):
    ref = refgen.build(CONFIG0_GRAMMAR, 4, rotation_deg=(0.0, 90.0, 0.0), sides=8)
    spec = S.config0_scene()
    n = ref["positions"].shape[0]
    assert np.abs(spec.mesh.positions[:n] - ref["positions"]).max() < 1e-5


def test_curved_segment_frames_match_the_reference(refgen):
    """One segment with yaw and pitch turns between its forward steps: the spline
    refines the curved spans (samplesPerSpan 4) and transports the frame."""
    grammar = "F(1,0.1) Yaw(30) F(1,0.1) Pitch(20) F(0.5,0.08) Roll(15) Yaw(-40) F(1,0.05)\nX -> X"
    ref = refgen.build(grammar, 0, sides=6)
    word = [("F", (1.0, 0.1)), ("Yaw", (30.0,)), ("F", (1.0, 0.1)), ("Pitch", (20.0,)), ("F", (0.5, 0.08)),
            ("Roll", (15.0,)), ("Yaw", (-40.0,)), ("F", (1.0, 0.05))]
    segs, _ = S.turtle(word)
    framed = S.spline_frames_all(segs)
    assert len(framed) == 1
    f = framed[0]
    rf = ref["frames"]
    assert len(f.points) == len(rf) > 5, "the curved spans were not refined like the reference's"
    assert np.allclose(np.array(f.points), rf[:, 0:3], atol=1e-5)
    assert np.allclose(np.array(f.tangents), rf[:, 3:6], atol=1e-5)
    assert np.allclose(np.array(f.normals), rf[:, 6:9], atol=1e-4)
    assert np.allclose(np.array(f.binormals), rf[:, 9:12], atol=1e-4)
    assert np.allclose(np.array(f.radii), rf[:, 12], atol=1e-6)
    mine = S.loft(framed, 6)
    assert np.abs(mine.positions - ref["positions"]).max() < 1e-5


def test_host_stage_times_are_reported(refgen):
    ref = refgen.build(CONFIG0_GRAMMAR, 4, rotation_deg=(0.0, 90.0, 0.0), sides=8)
    assert set(ref["ms"]) == {"lsystem", "turtle", "spline", "loft"}
    assert all(v >= 0.0 for v in ref["ms"].values()) and ref["symbols"] > 625
