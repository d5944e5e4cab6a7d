"""Procedural ingestion (lsystemeditor_b200.procedural, the host side of the
reference's meshSceneBuild) against the reference's own generator, no GPU.

Two instances of the config-0 grammar with their own root rotations and
translations (ProceduralInstance, ProceduralTypes.h:72-78): the product's
tubes, lofted on the host, must equal the reference generator's meshes of the
two instances (its LSystemLib, turtle and spline compiled unchanged; the root
transform of ProceduralMeshBuilder.cpp:243-253 restated beside them), appended
in instance order as meshSceneBuild appends them.
"""
import numpy as np
import pytest

from lsystemeditor_b200 import procedural as P
from lsystemeditor_b200 import scene as S

CONFIG0_GRAMMAR = "F(0.1,0.02)\nF(h,r) -> F(h,r)[Yaw(25.7)F(h,r)]F(h,r)[Yaw(0-25.7)F(h,r)]F(h,r)"


def _rule(args, _rng):
    h, r = args
    F = ("F", (h, r))
    return [F, ("[", ()), ("Yaw", (25.7,)), F, ("]", ()), F, ("[", ()), ("Yaw", (-25.7,)), F, ("]", ()), F]


INSTANCES = [
    dict(rotation_deg=(0.0, 90.0, 0.0), translation=(0.0, 0.0, 0.0), iterations=3),
    dict(rotation_deg=(35.0, 80.0, 10.0), translation=(2.5, -0.5, 1.25), iterations=2),
]


@pytest.fixture(scope="module")
def refgen():
    from oracle.bindings import ReferenceGenerator, reference_generator_available
    if not reference_generator_available():
        pytest.skip("reference generator build unavailable (no reference tree where build() ran)")
    return ReferenceGenerator()


def _instances():
    return [P.ProceduralInstance(axiom=[("F", (0.1, 0.02))], rules={"F": _rule}, iterations=d["iterations"],
                                 translation=d["translation"], rotation_deg=d["rotation_deg"]) for d in INSTANCES]


def test_two_instances_match_the_reference_generator(refgen):
    sides = 8
    refs = [refgen.build(CONFIG0_GRAMMAR, d["iterations"], rotation_deg=d["rotation_deg"],
                         translation=d["translation"], sides=sides) for d in INSTANCES]
    tubes = P.build_tubes(_instances(), P.ProceduralBuildParams(circular_segments=sides))
    mine = tubes.host_mesh()
    ref_pos = np.concatenate([r["positions"] for r in refs])
    ref_nrm = np.concatenate([r["normals"] for r in refs])
    ref_uv = np.concatenate([r["uvs"] for r in refs])
    assert mine.triangle_count == ref_pos.shape[0] == sum(32 * 5 ** d["iterations"] for d in INSTANCES)
    assert np.abs(mine.positions - ref_pos).max() < 2e-5
    assert np.abs(mine.normals - ref_nrm).max() < 2e-4
    assert np.array_equal(mine.uvs, ref_uv)


def test_translation_moves_the_instance_only():
    base = P.build_tubes([P.ProceduralInstance(word=[("F", (1.0, 0.1)), ("Yaw", (30.0,)), ("F", (1.0, 0.1))])],
                         P.ProceduralBuildParams(circular_segments=6)).host_mesh()
    moved = P.build_tubes([P.ProceduralInstance(word=[("F", (1.0, 0.1)), ("Yaw", (30.0,)), ("F", (1.0, 0.1))],
                                                translation=(3.0, -2.0, 0.5))],
                          P.ProceduralBuildParams(circular_segments=6)).host_mesh()
    assert np.allclose(moved.positions - base.positions, np.array([3.0, -2.0, 0.5], np.float32), atol=1e-5)
    assert np.array_equal(moved.normals, base.normals)
    assert np.array_equal(moved.uvs, base.uvs)


def test_instance_materials_and_errors():
    insts = [P.ProceduralInstance(word=[("F", (1.0, 0.1))], material=0),
             P.ProceduralInstance(word=[("F", (1.0, 0.1))], translation=(1.0, 0.0, 0.0), material=1)]
    bank = np.concatenate([P._default_bank(), P._default_bank()])
    tubes = P.build_tubes(insts, P.ProceduralBuildParams(circular_segments=4, materials=bank))
    assert list(tubes.materials) == [0, 1]
    mesh = tubes.host_mesh()
    assert len(mesh.materials) == 2 and set(np.unique(mesh.material_ids)) == {0, 1}
    with pytest.raises(ValueError):
        P.build_tubes([])
    with pytest.raises(ValueError):
        P.ProceduralInstance().evaluated()
